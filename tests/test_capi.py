"""CPU tests of the C interface library (no GPU needed).

* libpvfmm_b200.so loads and exports every function declared in include/pvfmm.h
* the host FP64 operator precompute (Jacobi SVD pseudo-inverses, U2U/D2D,
  V-list spectra) reproduces the oracle's FMM when the oracle runs on it
* argument validation fails loudly (no CPU fallback)
"""
import ctypes
import os
import re

import numpy as np
import pytest

import pvfmm_b200 as P
from oracle import pvfmm_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    src = open(os.path.join(ROOT, "include", "pvfmm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(PVFMM\w+|pvfmm\w+_)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(P.LIB_PATH))
    names = _declared_functions()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    lib = P.load_library()
    for n in _declared_functions():
        assert getattr(lib, n).restype is not None or n.startswith(("PVFMMEval", "PVFMMDestroy", "pvfmm")) \
            or n in ("PVFMMEvalD", "PVFMMEvalF")


@pytest.mark.parametrize("kid,m", [(0, 6), (1, 4), (6, 6)])
def test_library_operators_reproduce_oracle_fmm(kid, m):
    """The oracle on the library's operators agrees with the oracle on its own
    (numpy-SVD) operators far below the FMM truncation error."""
    K = O.KERNELS[kid]
    ops_lib = O.Operators.from_arrays(K, m, P.precomp_operators(P.FMMKernel(kid), m))
    ops_np = O.Operators(K, m)
    rng = np.random.default_rng(12)
    x = rng.random((2500, 3))
    q = rng.uniform(-1, 1, (2500, K.k0))
    a = O.pvfmm_eval(kid, m, 60, x, q, x, ops=ops_lib)
    b = O.pvfmm_eval(kid, m, 60, x, q, x, ops=ops_np)
    ref = O.direct_sum(kid, x, q, x)
    err = O.rel_l2(b, ref)
    assert O.rel_l2(a, b) < 1e-3 * err
    assert abs(O.rel_l2(a, ref) - err) < 1e-2 * err


@pytest.mark.parametrize("kid", [2, 4, 5])
def test_self_expanded_kernel_operators_reproduce_oracle_fmm(kid):
    """Stokes pressure (3->1), Stokes velocity gradient (3->9) and Biot-Savart
    (3->3) expand themselves, with rectangular check->equivalent factors: the
    library's host precompute drives the oracle FMM to the same result as the
    oracle's own operators."""
    K = O.KERNELS[kid]
    ops_lib = O.Operators.from_arrays(K, 4, P.precomp_operators(P.FMMKernel(kid), 4))
    rng = np.random.default_rng(50 + kid)
    x = rng.random((1200, 3))
    f = rng.standard_normal((1200, 3))
    a = O.pvfmm_eval(kid, 4, 60, x, f, x, ops=ops_lib)
    b = O.pvfmm_eval(kid, 4, 60, x, f, x)
    assert O.rel_l2(a, b) < 1e-3 * O.rel_l2(b, O.direct_sum(kid, x, f, x))


def test_stokes_operators_reproduce_oracle_fmm():
    K = O.KERNELS[3]
    ops_lib = O.Operators.from_arrays(K, 4, P.precomp_operators(P.FMMKernel.StokesVelocity, 4))
    rng = np.random.default_rng(13)
    x = rng.random((1200, 3))
    f = rng.standard_normal((1200, 3))
    a = O.pvfmm_eval(3, 4, 60, x, f, x, ops=ops_lib)
    b = O.pvfmm_eval(3, 4, 60, x, f, x)
    ref = O.direct_sum(3, x, f, x)
    assert O.rel_l2(a, b) < 1e-3 * O.rel_l2(b, ref)


def test_pseudo_inverse_factors():
    """UC2UE0 * UC2UE1 is the SVD pseudo-inverse of the equivalent->check
    matrix: M pinv M = M to near machine precision (fmm_pts.txx:478-537)."""
    m = 4
    ops = P.precomp_operators(P.FMMKernel.LaplacePotential, m)
    ns = 6 * (m - 1) ** 2 + 2
    u = ops["usurf"].reshape(ns, 3)
    M = O.LAPLACE.matrix(0.5 + 0.5 * O.RAD0 * u, 0.5 + 0.5 * O.RAD1 * u)
    c2e0 = ops["uc2ue0"].reshape(ns, ns)
    c2e1 = ops["uc2ue1"].reshape(ns, ns)
    R = (M @ c2e0) @ c2e1 @ M
    assert np.linalg.norm(R - M) / np.linalg.norm(M) < 1e-12


def test_unit_surface_matches_reference_surface():
    for m in (4, 6, 8):
        u = P.precomp_operator(P.FMMKernel.LaplacePotential, m, 0, 6).reshape(-1, 3)
        ref = O.surface(m, np.zeros(3), 1.0, 0) * 2 - 1.0     # alpha=1, depth 0: (u+1)*0.5
        np.testing.assert_allclose(u, ref, atol=1e-15)


def test_mixed_precompute_uses_fp32_cutoff():
    a = P.precomp_operator(P.FMMKernel.LaplacePotential, 6, 0, 0)
    b = P.precomp_operator(P.FMMKernel.LaplacePotential, 6, 1, 0)
    # the FP32 cutoff drops the smallest singular values: far smaller entries
    assert np.abs(b).max() < 1e-2 * np.abs(a).max()


def test_invalid_arguments_fail_loudly():
    lib = P.load_library()
    assert not lib.PVFMMCreateContextExD(-1.0, 100, 6, 9, 0)         # not a PVFMMKernel value
    assert "unsupported" in P.last_error()
    assert not lib.PVFMMCreateContextExD(-1.0, 100, 7, 0, 0)         # odd order
    assert P.last_error()
    assert P.precomp_operator.__doc__


def test_invalid_context_pointer_is_rejected():
    lib = P.load_library()
    bogus = (ctypes.c_char * 64)()
    assert lib.PVFMMGetTreeData(ctypes.cast(bogus, ctypes.c_void_p), 0, None, 0) == -1
    assert "invalid" in P.last_error()


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-GPU failure path")
def test_no_gpu_means_no_context():
    with pytest.raises(RuntimeError):
        P.FMMParticleContext(-1, 100, 4, P.FMMKernel.LaplacePotential)


def test_fortran_bindings_pass_every_argument_by_reference():
    """The Fortran entry points (reference src/pvfmm-wrapper.cpp:831-875),
    called as a Fortran program calls them: every argument by reference.
    Without a GPU the context cannot be created: the handle comes back NULL
    with the message set, and an evaluation on it fills the output with NaN."""
    if __import__("torch").cuda.is_available():
        pytest.skip("checks the no-GPU failure path")
    lib = ctypes.CDLL(str(P.LIB_PATH))
    c_i32, c_i64 = ctypes.c_int32, ctypes.c_int64
    ctx = ctypes.c_void_p(1)
    lib.pvfmmcreatecontextd_(ctypes.byref(ctx), ctypes.byref(ctypes.c_double(-1.0)), ctypes.byref(c_i32(100)),
                             ctypes.byref(c_i32(6)), ctypes.byref(c_i32(0)), ctypes.byref(c_i32(0)))
    assert ctx.value is None and P.last_error()
    x = np.random.default_rng(0).random(3 * 10)
    q = np.ones(10)
    out = np.zeros(10)
    lib.pvfmmevald_(x.ctypes.data_as(ctypes.c_void_p), q.ctypes.data_as(ctypes.c_void_p), ctypes.byref(c_i64(10)),
                    x.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(c_i64(10)),
                    ctypes.byref(ctx), ctypes.byref(c_i32(1)))
    assert np.isnan(out).all()
    lib.pvfmmdestroycontextd_(ctypes.byref(ctx))
    assert ctx.value is None
    ctxf = ctypes.c_void_p(1)
    lib.pvfmmcreatecontextf_(ctypes.byref(ctxf), ctypes.byref(ctypes.c_float(-1.0)), ctypes.byref(c_i32(100)),
                             ctypes.byref(c_i32(6)), ctypes.byref(c_i32(0)), ctypes.byref(c_i32(0)))
    assert ctxf.value is None
    lib.pvfmmdestroycontextf_(ctypes.byref(ctxf))
