"""GPU test of the allocation-free direct evaluation entry point.

PVFMMKernelEvalDeviceNoAllocD serves callers that cannot allocate device
memory when they call it (a framework that owns the device memory pool, or a
loop that must not pay for an allocation): its partial sums live in a fixed
array in the library's device image.  This file is collected last so that a
run stopping at the first failure has already run every other test; it also
passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import pvfmm_b200 as P
from oracle import pvfmm_oracle as O

pytestmark = pytest.mark.gpu


def _bind(lib):
    f = lib.PVFMMKernelEvalDeviceNoAllocD
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_long, ctypes.c_void_p]
    return f


def test_no_alloc_matches_allocating_entry_point_on_two_calls():
    torch = pytest.importorskip("torch")
    lib = P.load_library()
    noalloc = _bind(lib)
    vp = ctypes.c_void_p
    for call, (kid, n_src, n_trg) in enumerate([(6, 20000, 5000), (3, 7000, 30000)]):
        K = O.KERNELS[kid]
        rng = np.random.default_rng(100 + call)
        src = torch.as_tensor(rng.random((n_src, 3)), device="cuda")
        den = torch.as_tensor(rng.uniform(-1, 1, (n_src, K.k0)), device="cuda")
        trg = torch.as_tensor(np.concatenate([rng.random((n_trg - 10, 3)), src[:10].cpu().numpy()]), device="cuda")
        a = torch.zeros((n_trg, K.k1), device="cuda", dtype=torch.float64)
        b = torch.zeros((n_trg, K.k1), device="cuda", dtype=torch.float64)
        stream = torch.cuda.current_stream().cuda_stream
        P.kernel_eval_device(P.FMMKernel(kid), src.data_ptr(), den.data_ptr(), n_src, trg.data_ptr(), a.data_ptr(),
                             n_trg, stream)
        rc = noalloc(kid, vp(src.data_ptr()), vp(den.data_ptr()), n_src, vp(trg.data_ptr()), vp(b.data_ptr()), n_trg,
                     vp(stream))
        assert rc == 0, P.last_error()
        torch.cuda.synchronize()
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.isfinite(b).all()
        np.testing.assert_allclose(b, a, rtol=1e-12, atol=1e-12 * np.abs(a).max())


def test_no_alloc_at_its_scratch_limit():
    # n_trg * k1 = 262144 * 4 = 1 Mi values fills the fixed scratch exactly:
    # the scratch then holds one partial row per value, so the chunk count is
    # forced down to 1 (the allocating path splits the sources into chunks)
    torch = pytest.importorskip("torch")
    lib = P.load_library()
    noalloc = _bind(lib)
    vp = ctypes.c_void_p
    n_src, n_trg = 3000, (1 << 20) // 4
    rng = np.random.default_rng(300)
    src = torch.as_tensor(rng.random((n_src, 3)), device="cuda")
    den = torch.as_tensor(rng.uniform(-1, 1, (n_src, 1)), device="cuda")
    trg = torch.as_tensor(rng.random((n_trg, 3)), device="cuda")
    a = torch.zeros((n_trg, 4), device="cuda", dtype=torch.float64)
    b = torch.full((n_trg, 4), 0.25, device="cuda", dtype=torch.float64)
    a += 0.25
    stream = torch.cuda.current_stream().cuda_stream
    P.kernel_eval_device(P.FMMKernel(6), src.data_ptr(), den.data_ptr(), n_src, trg.data_ptr(), a.data_ptr(), n_trg,
                         stream)
    for _ in range(2):
        c = b.clone()
        rc = noalloc(6, vp(src.data_ptr()), vp(den.data_ptr()), n_src, vp(trg.data_ptr()), vp(c.data_ptr()), n_trg,
                     vp(stream))
        assert rc == 0, P.last_error()
        assert P.last_error() == ""
        torch.cuda.synchronize()
        np.testing.assert_allclose(c.cpu().numpy(), a.cpu().numpy(), rtol=1e-12,
                                   atol=1e-12 * float(a.abs().max()))


def test_no_alloc_empty_call_clears_the_last_error():
    lib = P.load_library()
    noalloc = _bind(lib)
    vp = ctypes.c_void_p
    assert noalloc(99, None, None, 1, None, None, 1, None) != 0   # unknown kernel id sets an error
    assert P.last_error() != ""
    assert noalloc(6, None, None, 0, None, None, 0, None) == 0   # nothing to do: success, error cleared
    assert P.last_error() == ""


def test_no_alloc_rejects_sizes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    lib = P.load_library()
    noalloc = _bind(lib)
    n_trg = (1 << 20) // 4 + 1                      # pot+grad: 4 values per target
    src = torch.zeros((8, 3), device="cuda", dtype=torch.float64)
    trg = torch.zeros((n_trg, 3), device="cuda", dtype=torch.float64)
    out = torch.zeros((n_trg, 4), device="cuda", dtype=torch.float64)
    vp = ctypes.c_void_p
    rc = noalloc(6, vp(src.data_ptr()), vp(src.data_ptr()), 8, vp(trg.data_ptr()), vp(out.data_ptr()), n_trg, None)
    assert rc != 0
    assert "exceeds the fixed scratch" in P.last_error()
