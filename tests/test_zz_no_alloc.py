"""The allocation-free evaluation, egs_mle_eval_noalloc, against egs_mle_eval.

It serves callers that cannot call cudaMalloc: applications whose device memory
belongs to another allocator (a framework's caching allocator, or a pool sized
once at start-up) and evaluation loops that cannot pay the device-wide
synchronisation of cudaMalloc/cudaFree on every call.  The caller hands over
every large buffer; the entry point keeps its small per-call state in one
static device array.  This test allocates the caller's buffers itself (through
torch) and calls the entry point through the C ABI.

The file is named so that pytest collects it last: a run that stops at the
first failure has then already run every other test.
"""
import ctypes

import numpy as np
import pytest

import exageostatcpp_b200 as egs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LOGLIK_RTOL = 1e-10  # the plain-FP64 log-likelihood tolerance of the parity tests


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_matches_resident_evaluation_on_two_calls():
    torch = pytest.importorskip("torch")
    n, dts = 1500, 320
    x, y, z = O.load_data(n, 3, [1.0, 0.1, 0.5])
    lib = egs.load_library()
    need = ctypes.c_longlong()
    assert lib.egs_mle_noalloc_workspace(n, dts, ctypes.byref(need)) == egs.EGS_OK
    dev = torch.device("cuda:0")
    tx, ty, tz = (torch.tensor(a, dtype=torch.float64, device=dev) for a in (x, y, z))
    work = torch.empty(need.value, dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream()

    p = egs.Problem(n, dts)
    p.set_locations(x, y)
    p.set_observations(z)
    for theta in ([1.0, 0.1, 0.5], [0.8, 0.07, 1.3]):
        th = np.array(theta, dtype=np.float64)
        out = ctypes.c_double()
        rc = lib.egs_mle_eval_noalloc(n, dts, _ptr(tx), _ptr(ty), _ptr(tz),
                                      th.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _ptr(work), need.value,
                                      ctypes.byref(out), ctypes.c_void_p(stream.cuda_stream))
        assert rc == egs.EGS_OK, lib.egs_last_error()
        ref = p.mle_eval(theta)[0]
        assert out.value == pytest.approx(ref, rel=LOGLIK_RTOL, abs=0)
    p.close()
    # the inputs are read only
    assert np.array_equal(tz.cpu().numpy(), z)
    assert np.array_equal(tx.cpu().numpy(), x)


def test_noalloc_call_leaves_device_memory_unchanged():
    # The feature's claim: after a first call (which loads the kernels and looks
    # up the static array), an evaluation takes no device memory of its own.
    # Free device memory is read before and after a second call; a cudaMalloc,
    # cudaMallocAsync or a lazily loaded module anywhere on its path shows up as
    # a drop.
    torch = pytest.importorskip("torch")
    n, dts = 1300, 256
    x, y, z = O.load_data(n, 4, [1.0, 0.08, 0.9])
    lib = egs.load_library()
    need = ctypes.c_longlong()
    assert lib.egs_mle_noalloc_workspace(n, dts, ctypes.byref(need)) == egs.EGS_OK
    dev = torch.device("cuda:0")
    tx, ty, tz = (torch.tensor(a, dtype=torch.float64, device=dev) for a in (x, y, z))
    work = torch.empty(need.value, dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream()
    th = np.array([1.0, 0.08, 0.9], dtype=np.float64)
    values = []
    free = []
    for _ in range(2):
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info(dev)[0])
        out = ctypes.c_double()
        rc = lib.egs_mle_eval_noalloc(n, dts, _ptr(tx), _ptr(ty), _ptr(tz),
                                      th.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _ptr(work), need.value,
                                      ctypes.byref(out), ctypes.c_void_p(stream.cuda_stream))
        assert rc == egs.EGS_OK, lib.egs_last_error()
        torch.cuda.synchronize()
        values.append(out.value)
    free.append(torch.cuda.mem_get_info(dev)[0])
    assert free[2] == free[1], (free, "the second call changed the free device memory")
    assert values[0] == values[1]
    assert values[1] == pytest.approx(O.mle_loglik(x, y, z, th), rel=LOGLIK_RTOL, abs=0)


def test_noalloc_rejects_sizes_beyond_its_limit():
    lib = egs.load_library()
    need = ctypes.c_longlong()
    # 4096 device tiles of 64 rows is the largest problem the static state covers
    assert lib.egs_mle_noalloc_workspace(4096 * 64, 64, ctypes.byref(need)) == egs.EGS_OK
    assert lib.egs_mle_noalloc_workspace(4096 * 64 + 1, 64, ctypes.byref(need)) == egs.EGS_ERR_INVALID
    assert b"4096" in lib.egs_last_error()
    th = np.array([1.0, 0.1, 0.5])
    out = ctypes.c_double()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.egs_mle_eval_noalloc(4096 * 64 + 1, 64, dummy, dummy, dummy,
                                  th.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), dummy, 1 << 40,
                                  ctypes.byref(out), None)
    assert rc == egs.EGS_ERR_INVALID


def test_noalloc_rejects_a_short_workspace():
    torch = pytest.importorskip("torch")
    n, dts = 200, 64
    lib = egs.load_library()
    need = ctypes.c_longlong()
    assert lib.egs_mle_noalloc_workspace(n, dts, ctypes.byref(need)) == egs.EGS_OK
    dev = torch.device("cuda:0")
    buf = torch.zeros(need.value, dtype=torch.float64, device=dev)
    th = np.array([1.0, 0.1, 0.5])
    out = ctypes.c_double()
    rc = lib.egs_mle_eval_noalloc(n, dts, _ptr(buf), _ptr(buf), _ptr(buf),
                                  th.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _ptr(buf), need.value - 1,
                                  ctypes.byref(out), None)
    assert rc == egs.EGS_ERR_INVALID
    assert b"workspace" in lib.egs_last_error()
