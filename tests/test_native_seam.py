"""The seam solprop's registry loads as its native backend (``solprop_native``).

``src/solprop/backends/registry.py:386-394`` imports ``NativeBackend`` from
``solprop_native`` and builds it with the problem and request.  Without a GPU: the
package reports and checks its build; and, where the reference checkout is present, the
reference's own registry -- imported from a scratch backport of it -- resolves
``"native"`` to this package's backend for a capillary problem, whose every source
evaluation is then routed to the device library, and refuses by name, as solprop's
``BackendError``, a problem the device path does not execute.
"""

import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
REFERENCE = Path(os.environ.get("SOLPROP_REFERENCE", "/root/reference"))


def test_build_info_and_check():
    import solprop_native

    info = solprop_native.check_build()
    assert "sm_100a" in info.version and info.device_backend == "cuda"
    assert Path(info.library).exists()


@pytest.fixture(scope="module")
def reference():
    if not (REFERENCE / "src" / "solprop").is_dir():
        pytest.skip("the reference checkout is not on this machine")
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    import generate  # the fixture generator: backports the reference and builds problems

    return generate


def test_reference_registry_resolves_the_device_backend(reference):
    import solprop_native
    from solprop.backends import registry
    from solprop.backends.numpy_ref.workspace import NumpyWorkspace

    sim = reference.capillary("cap1_ar", gas="Ar", pressure=1.0, length=0.02,
                              n_t_limits=(200e-9, 4e-6), trange=100e-15, energy=30e-6,
                              fwhm=10e-15, modes=1)
    problem, request = sim.translate(), sim.run_request()
    backend = registry.select("native", problem, request, grid=sim.grid, modes=sim.modes,
                              profiles=sim.profiles)
    assert type(backend).__module__ == "solprop_native" and backend.name == "native"
    assert isinstance(backend, solprop_native.NativeBackend)
    workspace = backend._workspace
    # every source evaluation of the host march goes to the device library
    assert workspace.nonlinear.__func__ is solprop_native._device_nonlinear
    assert NumpyWorkspace.nonlinear is not solprop_native._device_nonlinear
    assert workspace._device.record.n_to == sim.grid.n_to
    assert backend.metadata()["backend"] == "native"
    backend.close()


def test_reference_registry_refuses_by_name(reference):
    from solprop.backends import registry
    from solprop.exceptions import BackendError

    sim = reference.capillary("cap1_ar", gas="Ar", pressure=1.0, length=0.02,
                              n_t_limits=(200e-9, 4e-6), trange=100e-15, energy=30e-6,
                              fwhm=10e-15, modes=1)
    problem, request = sim.translate(), sim.run_request()
    import dataclasses

    # five plasma channels: the device column carries a mixture of four at most
    responses = problem.responses
    five = dataclasses.replace(responses, plasma_channels=responses.plasma_channels * 5,
                               ionisation_table=tuple(responses.ionisation_table) * 5)
    bad = dataclasses.replace(problem, responses=five)
    with pytest.raises(BackendError, match="refused by the B200 backend"):
        registry.select("native", bad, request, grid=sim.grid, modes=sim.modes)
