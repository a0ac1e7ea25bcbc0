"""The source evaluation that allocates no device memory, against the allocating one.

``sp_source_noalloc`` serves callers that cannot call cudaMalloc -- code whose device
memory all belongs to a pool or framework, or that must not allocate while it runs --
by keeping every buffer in one fixed array inside the library.  This test calls it
through the C ABI twice in a row, on two different problems (so the second call starts
from the first call's leftovers in the shared array), and checks each result against
``sp_workspace_source_device`` on the same device buffers, at the tolerance of the other
source tests.  It sits in a file of its own that pytest collects last.
"""

import ctypes as C

import numpy as np
import pytest

from tests._cases import golden, record, rel

pytestmark = pytest.mark.gpu

SOURCE_TOL = 1e-10


def _device_copy(torch, array):
    flat = np.ascontiguousarray(array, dtype=np.complex128).view(np.float64).ravel()
    return torch.from_numpy(flat.copy()).to("cuda:0")


def _host(tensor, shape):
    return tensor.cpu().numpy().view(np.complex128).reshape(shape)


@pytest.mark.parametrize("order", [("cap4_he", "cap1_ar"), ("cap1_ar", "config1")])
def test_no_alloc_source_matches_the_workspace_twice_in_a_row(order):
    torch = pytest.importorskip("torch")
    from solprop_b200 import _lib

    lib = _lib.library()
    for call, case in enumerate(order):
        rec = record(case)
        g = golden(case)
        index = call  # a different lab on each call
        lab = g[f"src{index}.lab"]
        z = float(g[f"src{index}.z"])
        shape = (rec.n_modes, rec.n_pol, rec.n_omega)
        problem = _lib.Problem(rec)
        lab_dev = _device_copy(torch, lab)
        out_noalloc = torch.empty_like(lab_dev)
        stream = torch.cuda.current_stream().cuda_stream
        _lib.check(lib.sp_source_noalloc(problem.handle, C.c_void_p(lab_dev.data_ptr()), z, 0,
                                         C.c_void_p(out_noalloc.data_ptr()), C.c_void_p(stream)))
        torch.cuda.synchronize()
        ws = _lib.Workspace(problem, 0)
        out_ws = torch.empty_like(lab_dev)
        ws.source_device(lab_dev.data_ptr(), z, out_ws.data_ptr())
        torch.cuda.synchronize()
        got, want = _host(out_noalloc, shape), _host(out_ws, shape)
        assert np.all(np.isfinite(got))
        assert rel(got, want) < SOURCE_TOL, (case, call)
        # and both against the reference's own value for this lab
        assert rel(got, g[f"src{index}.source"]) < SOURCE_TOL, (case, call)
        ws.close()
        problem.close()


def test_no_alloc_refuses_a_problem_larger_than_its_array():
    from solprop_b200 import _lib

    rec = record("config2")
    rec.n_nodes = 512  # 3 * 512 * 16384 * 8 bytes of node streams alone: past 40 MiB
    rec.synthesis = np.tile(rec.synthesis, (8, 1))
    rec.projection = np.tile(rec.projection, (1, 8))
    problem = _lib.Problem(rec)
    lab = np.zeros(rec.n_cols * rec.n_omega * 2)
    with pytest.raises(_lib.NativeError, match="MiB"):
        _lib.check(_lib.library().sp_source_noalloc(
            problem.handle, C.c_void_p(lab.ctypes.data), 0.0, 0, C.c_void_p(lab.ctypes.data),
            None))


def test_no_alloc_after_a_refusal_leaves_the_callers_stream_usable():
    """A refused call on the caller's own stream, then a good call on it, then more work.

    The entry point lends the caller's stream to its internal view only for the call; a
    refusal part-way through (the problem does not fit the array) must leave nothing of
    it behind.  Free device memory is also unchanged across warm calls: the evaluation
    allocates nothing.
    """
    torch = pytest.importorskip("torch")
    from solprop_b200 import _lib

    lib = _lib.library()
    side = torch.cuda.Stream(device="cuda:0")
    big = record("config2")
    big.n_nodes = 512
    big.synthesis = np.tile(big.synthesis, (8, 1))
    big.projection = np.tile(big.projection, (1, 8))
    too_big = _lib.Problem(big)
    rec = record("cap1_ar")
    g = golden("cap1_ar")
    problem = _lib.Problem(rec)
    shape = (rec.n_modes, rec.n_pol, rec.n_omega)
    with torch.cuda.stream(side):
        lab_dev = _device_copy(torch, g["src1.lab"])
        out = torch.empty_like(lab_dev)
        junk = torch.zeros(big.n_cols * big.n_omega * 2, dtype=torch.float64, device="cuda:0")
    side.synchronize()
    handle = C.c_void_p(side.cuda_stream)
    with pytest.raises(_lib.NativeError, match="MiB"):
        _lib.check(lib.sp_source_noalloc(too_big.handle, C.c_void_p(junk.data_ptr()), 0.0, 0,
                                         C.c_void_p(junk.data_ptr()), handle))
    z = float(g["src1.z"])
    for _ in range(2):  # the first call on a device may resolve the array's address
        _lib.check(lib.sp_source_noalloc(problem.handle, C.c_void_p(lab_dev.data_ptr()), z, 0,
                                         C.c_void_p(out.data_ptr()), handle))
    free_before, _ = torch.cuda.mem_get_info(0)
    _lib.check(lib.sp_source_noalloc(problem.handle, C.c_void_p(lab_dev.data_ptr()), z, 0,
                                     C.c_void_p(out.data_ptr()), handle))
    free_after, _ = torch.cuda.mem_get_info(0)
    assert free_after == free_before
    # the stream still takes work after the calls
    with torch.cuda.stream(side):
        doubled = out * 2.0
    side.synchronize()
    got = _host(out, shape)
    assert rel(got, g["src1.source"]) < SOURCE_TOL
    assert rel(_host(doubled, shape), 2.0 * got) == 0.0
    problem.close()
    too_big.close()
