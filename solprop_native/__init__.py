"""The seam solprop's registry loads as its native backend, served by the B200 library.

solprop selects its native backend with ``from solprop_native import NativeBackend``
(``src/solprop/backends/registry.py:386-394``) and calls it with the problem, the run's
request and ``grid``, ``modes``, ``profiles``, ``tdse_binding``, ``options``.  This package
answers that import with:

* :func:`build_info` and :func:`check_build` -- what is loaded, and a check that the
  library and every entry point of ``include/solprop_b200.h`` are present;
* :class:`NativeBackend` -- solprop's own host session and march (the reference
  backend's, from the solprop install that imports this package) with every source
  evaluation, the hot path, executed by the CUDA library through its C ABI
  (``sp_workspace_source``): the lowered problem is built on the device once, and each
  evaluation crosses the seam as the state-sized lab field and its source.  Problems the
  device path does not execute are refused by name before anything is allocated, as
  solprop's ``BackendError``.

Whole runs stepped on the device (the C ABI's sessions and scans) are reached through
``solprop_b200._lib``; this seam keeps solprop's event, export and statistics protocol
unchanged.
"""

from __future__ import annotations

import dataclasses
import re
import types
from pathlib import Path

import numpy as np

from solprop_b200 import _lib
from solprop_b200.lowering import BackendRefusal as _LoweringRefusal

__all__ = ["NativeBackend", "build_info", "check_build"]

_HEADER = Path(__file__).resolve().parent.parent / "include" / "solprop_b200.h"


@dataclasses.dataclass(frozen=True)
class BuildInfo:
    """What this seam loads, with the fields solprop reads of a native build
    (``registry.py:172-183``: ``device_backend``, ``device_count``; ``_process.py:296-303``:
    ``blas_library``, the library whose own BLAS pool solprop leaves alone -- this one
    links none)."""

    package_version: str
    library: str
    version: str
    arch: str
    device_backend: str
    device_count: int
    blas_library: str


def build_info() -> BuildInfo:
    """The library this seam loads: its path, version string and visible devices."""
    lib = _lib.library()
    count = int(lib.sp_device_count())
    return BuildInfo(package_version="0.2", library=str(_lib.LIBRARY_PATH),
                     version=lib.sp_version().decode(), arch="sm_100a", device_backend="cuda",
                     device_count=max(count, 0), blas_library=str(_lib.LIBRARY_PATH))


def check_build() -> BuildInfo:
    """Load the library and check that it exports every entry point its header declares;
    raise ``RuntimeError`` naming what is missing.  Returns :func:`build_info`."""
    try:
        lib = _lib.library()
    except (ImportError, OSError) as error:
        raise RuntimeError(f"the B200 library did not load: {error}") from error
    declared = set(re.findall(r"\b(sp_[a-z0-9_]+)\s*\(", _HEADER.read_text()))
    missing = sorted(name for name in declared if not hasattr(lib, name))
    if missing:
        raise RuntimeError(f"the B200 library lacks {', '.join(missing)}")
    return build_info()


class DeviceSource:
    """One problem's device workspace, evaluating lab-frame sources through the C ABI.

    The problem is lowered and validated on the host when this is built (a refusal comes
    before anything is allocated); the device workspace is built by the first
    evaluation."""

    def __init__(self, problem, device: int = 0, precision: str = "fp64"):
        from solprop_b200.lowering import lower

        self.record = lower(problem)
        self._problem = _lib.Problem(self.record)
        self._device, self._precision = device, precision
        self._workspace = None
        self.calls = 0

    def lab_source(self, lab: np.ndarray, position: float, quiet: bool) -> np.ndarray:
        if self._workspace is None:
            self._workspace = _lib.Workspace(self._problem, self._device, self._precision)
        self.calls += 1
        return self._workspace.source(lab, position, quiet)

    def close(self) -> None:
        if self._workspace is not None:
            self._workspace.close()
            self._workspace = None
        self._problem.close()


def _device_nonlinear(workspace, lab, bundle, inverse_propagator, *, purpose="predictor"):
    """``NumpyWorkspace.nonlinear`` on the device: the stage's source depends on its
    position ``bundle.z1`` alone, so the lab-frame source there, carried to the anchor
    by the inverse propagator -- the last factor of the stage output
    (``passes/stepping.py:88-145``), a multiplication by one on the lab frame."""
    source = workspace._device.lab_source(lab, float(bundle.z1), bool(workspace.collar_quiet))
    return source * inverse_propagator


def _native_backend_class():
    from solprop.backends.numpy_ref import NumpyRefBackend
    from solprop.exceptions import BackendError

    class NativeBackend(NumpyRefBackend):
        """solprop's backend protocol with its source evaluations on the B200."""

        name = "native"

        def __init__(self, problem, request, *, grid=None, modes=None, profiles=None,
                     tdse_binding=None, options=None, device: int = 0, precision: str = "fp64"):
            try:
                device_source = DeviceSource(problem, device, precision)
            except (_LoweringRefusal, _lib.BackendRefusal) as refusal:
                raise BackendError(f"refused by the B200 backend: {refusal}") from refusal
            super().__init__(problem, request, grid=grid, modes=modes, profiles=profiles,
                             tdse_binding=tdse_binding, options=options)
            self._device = device_source
            workspace = self._workspace
            workspace._device = device_source
            workspace.nonlinear = types.MethodType(_device_nonlinear, workspace)

        def metadata(self) -> dict[str, object]:
            info = dict(super().metadata())
            info.update(backend="native", device=build_info().version,
                        device_sources=self._device.calls)
            return info

        def close(self) -> None:
            if getattr(self, "_device", None) is not None:
                self._device.close()
                self._device = None
            super().close()

    return NativeBackend


def __getattr__(name: str):
    # built on first use: the class extends the importing solprop's own backend
    if name == "NativeBackend":
        cls = _native_backend_class()
        globals()["NativeBackend"] = cls
        return cls
    raise AttributeError(f"module 'solprop_native' has no attribute {name!r}")
