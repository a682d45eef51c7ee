"""GPU parity tests: libpvfmm_b200 (CUDA, through the C ABI) vs the oracle.

The oracle runs on the library's own FP64 operators (Operators.from_arrays),
so the plain FP64 form must agree with it to round-off: rel-L2 <= 1e-12 on
every output, with an identical octree (Morton ids, leaf flags, point ranges,
parents).  The mixed form (FP32 compute, FP64 pseudo-inverse precompute) is
checked against the same oracle at the mixed-precision tolerance stated per
test.  Large-N cases check size-independent properties instead (linearity,
permutation invariance, determinism, accuracy against an FP64 direct sum on
sampled targets).
"""
import ctypes

import numpy as np
import pytest

import pvfmm_b200 as P
from oracle import pvfmm_oracle as O

pytestmark = pytest.mark.gpu

PLAIN_TOL = 1e-12      # plain FP64 GPU vs oracle (same operators)
MIXED_TOL = 1e-6       # mixed form vs oracle (the accuracy bar of the mixed form)


def points(dist, n, seed):
    rng = np.random.default_rng(seed)
    if dist == "unif":
        return rng.random((n, 3))
    if dist == "gauss":
        c = rng.uniform(0.1, 0.9, (8, 3))
        return np.clip(c[rng.integers(0, 8, n)] + 0.02 * rng.standard_normal((n, 3)), 0, 1)
    if dist == "sphere":
        u = rng.standard_normal((n, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        return 0.5 + np.array([0.45, 0.3, 0.15]) * u
    if dist == "coincident":
        x = rng.random((n, 3))
        x[: n // 2] = x[0]                     # half the points on one spot: tree to max depth
        x[n // 2: n // 2 + 20] = x[n - 1]
        return x
    raise ValueError(dist)


_OPS = {}


def oracle_ops(kid, m, prec=0):
    key = (kid, m, prec)
    if key not in _OPS:
        _OPS[key] = O.Operators.from_arrays(O.KERNELS[kid], m, P.precomp_operators(P.FMMKernel(kid), m, 0))
    return _OPS[key]


def gpu_eval(kid, m, mp, src, den, trg, prec=0, setup=True, ctx=None):
    ctx = ctx or P.FMMParticleContext(-1, mp, m, P.FMMKernel(kid), precision=prec)
    trg_arg = src.reshape(-1) if trg is src else trg.reshape(-1)
    src_arg = src.reshape(-1)
    if trg is src:
        trg_arg = src_arg
    out = ctx.evaluate(src_arg, None if den is None else den.reshape(-1), None, trg_arg, setup)
    return out.reshape(len(trg), -1), ctx


def tree_matches(ctx, fmm):
    N = fmm.tree.nodes
    keys = ctx.tree_data(2).reshape(-1, 4)
    ok = np.array([[n.X, n.Y, n.Z, n.depth] for n in N])
    assert keys.shape == ok.shape, (keys.shape, ok.shape)
    np.testing.assert_array_equal(keys, ok)
    np.testing.assert_array_equal(ctx.tree_data(3), [n.leaf for n in N])
    np.testing.assert_array_equal(ctx.tree_data(5).reshape(-1, 2), [n.trg for n in N])
    np.testing.assert_array_equal(ctx.tree_data(6), [n.parent for n in N])
    if fmm.tree.src_counted:
        np.testing.assert_array_equal(ctx.tree_data(4).reshape(-1, 2), [n.src for n in N])


CASES = [
    # name, kernel, m, n, max_pts, distribution, separate targets
    ("laplace_unif", 0, 6, 3000, 50, "unif", False),
    ("laplace_sep", 0, 6, 3000, 50, "unif", True),
    ("laplace_grad", 1, 6, 3000, 50, "unif", False),
    ("laplace_potgrad_m8", 6, 8, 3000, 60, "unif", False),
    ("stokes", 3, 6, 1500, 50, "unif", False),
    ("stokes_sep_m4", 3, 4, 1500, 40, "gauss", True),
    ("laplace_gauss", 0, 6, 5000, 40, "gauss", False),
    ("laplace_ellipsoid_m4", 0, 4, 4000, 30, "sphere", False),
    ("laplace_coincident_m4", 0, 4, 400, 10, "coincident", False),
]


@pytest.mark.parametrize("name,kid,m,n,mp,dist,sep", CASES, ids=[c[0] for c in CASES])
def test_plain_matches_oracle(name, kid, m, n, mp, dist, sep):
    K = O.KERNELS[kid]
    src = points(dist, n, 1)
    trg = points("unif", n // 2 + 3, 2) * 0.9 + 0.05 if sep else src
    den = np.random.default_rng(3).uniform(-1, 1, (n, K.k0))
    out, ctx = gpu_eval(kid, m, mp, src, den, trg)
    ref, fmm = O.pvfmm_eval(kid, m, mp, src, den, trg, ops=oracle_ops(kid, m), return_fmm=True)
    tree_matches(ctx, fmm)
    assert np.isfinite(out).all()
    assert O.rel_l2(out, ref) < PLAIN_TOL
    assert ctx.launch_count() > 0


@pytest.mark.parametrize("kid,m", [(0, 6), (3, 6), (3, 8), (6, 8)])
def test_mixed_matches_oracle(kid, m):
    """Laplace kernels: the mixed form matches the oracle (FP64-cutoff
    operators) to MIXED_TOL.  Stokes: the mixed form uses the FP32 cutoff in
    the downward pseudo-inverse and projects the upward equivalent densities,
    so it is a different approximation; it must be as accurate as the plain
    FMM against the direct sum."""
    K = O.KERNELS[kid]
    src = points("unif", 3000, 4)
    den = np.random.default_rng(5).uniform(-1, 1, (3000, K.k0))
    out, ctx = gpu_eval(kid, m, 50, src, den, src, prec=P.PRECISION_MIXED)
    ref, fmm = O.pvfmm_eval(kid, m, 50, src, den, src, ops=oracle_ops(kid, m), return_fmm=True)
    tree_matches(ctx, fmm)
    if kid == 3:
        direct = O.direct_sum(kid, src, den, src)
        assert O.rel_l2(out, direct) < 1.5 * O.rel_l2(ref, direct) + 1e-6
    else:
        assert O.rel_l2(out, ref) < MIXED_TOL


def test_float_api_matches_oracle():
    src = points("unif", 3000, 6)
    den = np.random.default_rng(7).uniform(-1, 1, 3000)
    ctx = P.FMMParticleContext(-1, 50, 6, P.FMMKernel.LaplacePotential, dtype=np.float32)
    s32 = src.astype(np.float32).reshape(-1)
    out = ctx.evaluate(s32, den.astype(np.float32), None, s32, True)
    assert out.dtype == np.float32
    ref = O.pvfmm_eval(0, 6, 50, src.astype(np.float32).astype(np.float64), den.astype(np.float32), src.astype(np.float32).astype(np.float64))
    assert O.rel_l2(out, ref) < 5e-5


@pytest.mark.parametrize("kid", [0, 3])
def test_float_api_double_layer_matches_oracle(kid):
    """PVFMMEvalF with single- and double-layer values (FP32 inputs, the mixed
    form) against the FP64 oracle on the same FP32-rounded inputs."""
    K = O.KERNELS[kid]
    src = points("gauss", 3000, 16)
    rng = np.random.default_rng(17)
    den = rng.uniform(-1, 1, (3000, K.k0)).astype(np.float32)
    dl = rng.uniform(-1, 1, (3000, K.k0 + 3)).astype(np.float32)
    ctx = P.FMMParticleContext(-1, 50, 6, P.FMMKernel(kid), dtype=np.float32)
    s32 = src.astype(np.float32).reshape(-1)
    out = ctx.evaluate(s32, den.reshape(-1), dl.reshape(-1), s32, True)
    ctx.close()
    assert out.dtype == np.float32
    s64 = src.astype(np.float32).astype(np.float64)
    # the oracle follows the float interface's FP32 bounding box, mapped
    # coordinates and scales (mapping in FP32 moves close pairs by ~1e-7 of
    # the box, which the 1/r^2 double layer turns into ~1e-4 of the output,
    # in the reference's float interface as much as here)
    ref = O.pvfmm_eval(kid, 6, 50, s64, den, s64, dl_den=dl, real=np.float32)
    direct = O.direct_sum_mapped(kid, s64, den.astype(np.float64), s64, dl_den=dl.astype(np.float64))
    # Laplace: the mixed form's accuracy; Stokes (whose double-layer FMM is far
    # from its direct sum, see the reference pins): as close to the direct sum
    # as the FP64 FMM
    if kid == 0:
        assert O.rel_l2(out, ref) < 1e-5
    else:
        assert O.rel_l2(out, direct) < 1.5 * O.rel_l2(ref, direct) + 1e-5


def test_setup0_reuses_tree_with_new_densities():
    src = points("gauss", 4000, 8)
    rng = np.random.default_rng(9)
    d1, d2 = rng.uniform(-1, 1, 4000), rng.uniform(-1, 1, 4000)
    ctx = P.FMMParticleContext(-1, 40, 6, P.FMMKernel.LaplacePotential)
    a = ctx.evaluate(src.reshape(-1), d1, None, src.reshape(-1), True)
    b = ctx.evaluate(src.reshape(-1), d2, None, src.reshape(-1), False)
    c = P.FMMParticleContext(-1, 40, 6, P.FMMKernel.LaplacePotential).evaluate(src.reshape(-1), d2, None,
                                                                               src.reshape(-1), True)
    np.testing.assert_array_equal(b, c)
    assert O.rel_l2(a, b) > 0.1


def test_null_densities_build_tree_on_targets_only():
    src = points("unif", 2000, 10)
    trg = points("gauss", 1000, 11)
    ctx = P.FMMParticleContext(-1, 30, 4, P.FMMKernel.LaplacePotential)
    out = ctx.evaluate(src.reshape(-1), None, None, trg.reshape(-1), True)
    assert (out == 0).all()
    f = O.FMM(0, 4, 30, ops=oracle_ops(0, 4))
    scale, shift = O.bounding_box_map(src, trg)
    f.setup(O.map_points(src, scale, shift), O.map_points(trg, scale, shift), src_counted=False)
    tree_matches(ctx, f)


def test_empty_inputs():
    lib = P.load_library()
    ctx = P.FMMParticleContext(-1, 30, 4, P.FMMKernel.LaplaceGradient)
    trg = points("unif", 10, 12).reshape(-1)
    out = np.full(30, 7.0)
    src = np.zeros(3)
    lib.PVFMMEvalD(src.ctypes.data_as(ctypes.c_void_p), src.ctypes.data_as(ctypes.c_void_p), None, 0,
                   trg.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p), 10,
                   ctypes.c_void_p(ctx._ptr), 1)
    assert P.last_error() == ""
    assert (out == 0).all()
    out2 = np.full(3, 7.0)
    lib.PVFMMEvalD(trg.ctypes.data_as(ctypes.c_void_p), trg.ctypes.data_as(ctypes.c_void_p), None, 10,
                   trg.ctypes.data_as(ctypes.c_void_p), out2.ctypes.data_as(ctypes.c_void_p), 0,
                   ctypes.c_void_p(ctx._ptr), 1)
    assert (out2 == 7.0).all()


def test_single_point_and_tiny_inputs():
    for n in (1, 2, 7):
        src = points("unif", n, 13 + n)
        den = np.ones(n)
        out, _ = gpu_eval(0, 4, 10, src, den, src)
        ref = O.direct_sum(0, src, den, src)
        np.testing.assert_allclose(out, ref, rtol=1e-12, atol=1e-300)


def test_setup0_with_changed_counts_is_an_error():
    ctx = P.FMMParticleContext(-1, 30, 4, P.FMMKernel.LaplacePotential)
    a = points("unif", 100, 20)
    ctx.evaluate(a.reshape(-1), np.ones(100), None, a.reshape(-1), True)
    b = points("unif", 90, 21)
    with pytest.raises(RuntimeError, match="setup=0"):
        ctx.evaluate(b.reshape(-1), np.ones(90), None, b.reshape(-1), False)


def test_device_entry_point_matches_host_entry_point():
    torch = pytest.importorskip("torch")
    src = points("gauss", 20000, 22)
    den = np.random.default_rng(23).uniform(-1, 1, 20000)
    ctx = P.FMMParticleContext(-1, 64, 6, P.FMMKernel.LaplacePotGrad)
    host = ctx.evaluate(src.reshape(-1), den, None, src.reshape(-1), True)
    ds = torch.as_tensor(src, device="cuda")
    dd = torch.as_tensor(den, device="cuda")
    do = torch.empty((20000, 4), device="cuda", dtype=torch.float64)
    ctx.evaluate_device(ds.data_ptr(), dd.data_ptr(), 20000, ds.data_ptr(), do.data_ptr(), 20000, True,
                        torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(do.cpu().numpy().reshape(-1), host)


# ---------------------------------------------------------------- large N
@pytest.fixture(scope="module")
def big():
    n = 1_000_000
    rng = np.random.default_rng(30)
    c = rng.uniform(0.1, 0.9, (8, 3))
    x = np.clip(c[rng.integers(0, 8, n)] + 0.02 * rng.standard_normal((n, 3)), 0, 1)
    return x, rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)


def _direct_sample(x, q, idx, torch):
    X = torch.as_tensor(x, device="cuda")
    Q = torch.as_tensor(q, device="cuda")
    T = X[torch.as_tensor(idx, device="cuda")]
    out = torch.zeros(len(idx), device="cuda", dtype=torch.float64)
    for a in range(0, len(x), 1 << 15):
        d = T[:, None, :] - X[None, a:a + (1 << 15)]
        r2 = (d * d).sum(-1)
        out += torch.where(r2 > 0, Q[None, a:a + (1 << 15)] * r2.clamp_min(1e-300).rsqrt(),
                           torch.zeros_like(r2)).sum(1)
    return (out / (4 * np.pi)).cpu().numpy()


def test_large_linearity_determinism_and_accuracy(big):
    torch = pytest.importorskip("torch")
    x, q1, q2 = big
    ctx = P.FMMParticleContext(-1, 256, 8, P.FMMKernel.LaplacePotential)
    a = ctx.evaluate(x.reshape(-1), q1, None, x.reshape(-1), True)
    b = ctx.evaluate(x.reshape(-1), q2, None, x.reshape(-1), False)
    c = ctx.evaluate(x.reshape(-1), 2.0 * q1 - 3.0 * q2, None, x.reshape(-1), False)
    assert O.rel_l2(c, 2.0 * a - 3.0 * b) < 1e-13
    a2 = ctx.evaluate(x.reshape(-1), q1, None, x.reshape(-1), True)
    np.testing.assert_array_equal(a, a2)
    idx = np.random.default_rng(31).choice(len(x), 500, replace=False)
    ref = _direct_sample(x, q1, idx, torch)
    assert O.rel_l2(a[idx], ref) < 1e-6


def test_large_permutation_invariance(big):
    x, q1, _ = big
    perm = np.random.default_rng(32).permutation(len(x))
    ctx = P.FMMParticleContext(-1, 256, 8, P.FMMKernel.LaplacePotential)
    a = ctx.evaluate(x.reshape(-1), q1, None, x.reshape(-1), True)
    xp = np.ascontiguousarray(x[perm])
    b = ctx.evaluate(xp.reshape(-1), np.ascontiguousarray(q1[perm]), None, xp.reshape(-1), True)
    assert O.rel_l2(b, a[perm]) < 1e-13


def test_large_mixed_accuracy(big):
    torch = pytest.importorskip("torch")
    x, q1, _ = big
    ctx = P.FMMParticleContext(-1, 256, 8, P.FMMKernel.LaplacePotential, precision=P.PRECISION_MIXED)
    a = ctx.evaluate(x.reshape(-1), q1, None, x.reshape(-1), True)
    idx = np.random.default_rng(33).choice(len(x), 500, replace=False)
    ref = _direct_sample(x, q1, idx, torch)
    assert O.rel_l2(a[idx], ref) < 1e-6


def test_large_mixed_potgrad_every_component(big):
    """Mixed form, pot+grad at 1M points: each of the 4 outputs within 1e-6
    of an FP64 direct sum (the potential is the far-field-dominated one)."""
    torch = pytest.importorskip("torch")
    x, q1, _ = big
    ctx = P.FMMParticleContext(-1, 256, 8, P.FMMKernel.LaplacePotGrad, precision=P.PRECISION_MIXED)
    a = ctx.evaluate(x.reshape(-1), q1, None, x.reshape(-1), True).reshape(-1, 4)
    idx = np.random.default_rng(34).choice(len(x), 500, replace=False)
    X = torch.as_tensor(x, device="cuda")
    Q = torch.as_tensor(q1, device="cuda")
    T = X[torch.as_tensor(idx, device="cuda")]
    ref = torch.zeros((len(idx), 4), device="cuda", dtype=torch.float64)
    for s0 in range(0, len(x), 1 << 15):
        d = T[:, None, :] - X[None, s0:s0 + (1 << 15)]
        r2 = (d * d).sum(-1)
        rinv = torch.where(r2 > 0, r2.clamp_min(1e-300).rsqrt(), torch.zeros_like(r2))
        qr = rinv * Q[None, s0:s0 + (1 << 15)]
        ref[:, 0] += qr.sum(1)
        ref[:, 1:] += (d * (qr * rinv * rinv)[:, :, None]).sum(1)
    ref = (ref / (4 * np.pi)).cpu().numpy()
    for k in range(4):
        assert O.rel_l2(a[idx, k], ref[:, k]) < 1e-6, k


@pytest.mark.parametrize("kid", [0, 1, 2, 3, 4, 5, 6])
def test_kernel_eval_device_matches_direct_sum(kid):
    """PVFMMKernelEvalDeviceD (Kernel<T>::ker_poten on the GPU) accumulates the
    FP64 direct sum into its output."""
    torch = pytest.importorskip("torch")
    K = O.KERNELS[kid]
    rng = np.random.default_rng(40 + kid)
    src = rng.random((3000, 3))
    trg = np.concatenate([rng.random((700, 3)), src[:50]])      # includes r == 0 pairs
    den = rng.uniform(-1, 1, (3000, K.k0))
    ref = O.direct_sum(kid, src, den, trg)
    ds, dd, dt = (torch.as_tensor(a, device="cuda") for a in (src, den, trg))
    out = torch.full((len(trg), K.k1), 0.5, device="cuda", dtype=torch.float64)
    P.kernel_eval_device(P.FMMKernel(kid), ds.data_ptr(), dd.data_ptr(), 3000, dt.data_ptr(), out.data_ptr(), len(trg))
    torch.cuda.synchronize()
    np.testing.assert_allclose(out.cpu().numpy() - 0.5, ref, rtol=1e-11, atol=1e-11 * np.abs(ref).max())


@pytest.mark.parametrize("prec", [P.PRECISION_PLAIN, P.PRECISION_MIXED])
def test_vlist_chunks_give_identical_results(monkeypatch, prec):
    """The V-list runs its target parents in chunks when the output spectra
    do not fit in device memory; every parent's products are independent of
    the chunking, so the results are bit-identical."""
    src = points("gauss", 20000, 31)
    den = np.random.default_rng(32).uniform(-1, 1, 20000)
    whole, ctx = gpu_eval(6, 6, 40, src, den, src, prec=prec)
    ctx.close()
    monkeypatch.setenv("PVFMM_B200_VLIST_CHUNK", "100")
    chunked, ctx = gpu_eval(6, 6, 40, src, den, src, prec=prec)
    assert ctx.tree_stats()["n_vtrg"] > 300
    ctx.close()
    assert np.array_equal(whole, chunked)


def test_tree_build_writes_stay_in_bounds_on_a_count_mismatch():
    """The tree build checks its per-level internal-node and leaf counts only
    at its final synchronisation; until then the kernels that write by scan
    rank skip ranks beyond the buffers' capacities.  The library's self-check
    runs them with more flagged entries than capacity and checks a guard band
    after each buffer."""
    lib = P.load_library()
    f = lib.PVFMMB200CheckBoundedWrites
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_long, ctypes.c_long]
    for n, cap in [(1000, 600), (4096, 0), (300, 300)]:
        assert f(n, cap) == 0, P.last_error()


def test_tcgen05_hadamard_agrees_with_mma_sync_hadamard(monkeypatch):
    """The mixed form's V-list products on the 5th-generation tensor cores
    (tcgen05, TMEM accumulators, tiles of Morton-consecutive targets with their
    source unions staged in shared memory) and on the warp-level MMA path give
    the same FMM result to well within the mixed form's accuracy (both carry
    each product to ~2^-22 with a 3-term TF32 split; only the accumulation
    order inside the tensor cores differs)."""
    src = points("gauss", 40000, 41)
    den = np.random.default_rng(42).uniform(-1, 1, 40000)
    monkeypatch.setenv("PVFMM_B200_HADAMARD", "tcgen05")
    a, ctx = gpu_eval(6, 8, 128, src, den, src, prec=P.PRECISION_MIXED)
    assert ctx.tree_stats()["n_vtrg"] > 200
    ctx.close()
    monkeypatch.setenv("PVFMM_B200_HADAMARD", "mma")
    b, ctx = gpu_eval(6, 8, 128, src, den, src, prec=P.PRECISION_MIXED)
    ctx.close()
    for k in range(4):
        assert O.rel_l2(a[:, k], b[:, k]) < 1e-7, k


@pytest.mark.parametrize("kid", [0, 6])
def test_fp64_tensor_core_hadamard_agrees_with_simt(monkeypatch, kid):
    """The plain form's scalar V-list products on the FP64 tensor cores
    (mma.sync m8n8k4 .f64) and in FP64 SIMT give the same FMM result to FP64
    rounding."""
    K = O.KERNELS[kid]
    src = points("gauss", 30000, 45)
    den = np.random.default_rng(46).uniform(-1, 1, (30000, K.k0))
    monkeypatch.setenv("PVFMM_B200_HADAMARD", "simt")
    a, ctx = gpu_eval(kid, 8, 60, src, den, src, prec=P.PRECISION_PLAIN)
    assert ctx.tree_stats()["n_vtrg"] > 100
    ctx.close()
    monkeypatch.delenv("PVFMM_B200_HADAMARD")
    b, ctx = gpu_eval(kid, 8, 60, src, den, src, prec=P.PRECISION_PLAIN)
    ctx.close()
    for k in range(K.k1):
        assert O.rel_l2(b[:, k], a[:, k]) < 1e-12, k


@pytest.mark.parametrize("prec", [P.PRECISION_MIXED, P.PRECISION_PLAIN])
@pytest.mark.parametrize("kid", [3, 2, 4, 5])
def test_tensor_core_hadamard_of_vector_expansions_agrees_with_simt(monkeypatch, kid, prec):
    """The V-list products of the 3-component expansions (Stokes velocity,
    pressure, velocity gradient; Biot-Savart) on the tensor cores (mixed: TF32
    3-term split, plain: FP64; K = 48, streamed operator fragments) and in SIMT
    give the same FMM result: to FP64 rounding in the plain form (2e-13 apart:
    624-term sums in different orders, amplified by the downward
    pseudo-inverse), within the mixed
    form's accuracy in the mixed one (3e-7 apart on this case: both round each
    product to FP32 accuracy, the SIMT kernel in FP32 FMA chains over 624
    terms, the tensor cores through the split products and fresh
    accumulators)."""
    K = O.KERNELS[kid]
    src = points("gauss", 20000, 43)
    den = np.random.default_rng(44).uniform(-1, 1, (20000, K.k0))
    monkeypatch.setenv("PVFMM_B200_HADAMARD3", "simt")
    a, ctx = gpu_eval(kid, 6, 40, src, den, src, prec=prec)
    assert ctx.tree_stats()["n_vtrg"] > 100
    ctx.close()
    monkeypatch.delenv("PVFMM_B200_HADAMARD3")
    b, ctx = gpu_eval(kid, 6, 40, src, den, src, prec=prec)
    ctx.close()
    tol = 1e-6 if prec == P.PRECISION_MIXED else 1e-12
    for k in range(K.k1):
        assert O.rel_l2(b[:, k], a[:, k]) < tol, k


@pytest.mark.parametrize("prec,kid", [(P.PRECISION_PLAIN, 6), (P.PRECISION_MIXED, 6), (P.PRECISION_PLAIN, 3),
                                      (P.PRECISION_MIXED, 3)])
def test_vlist_frequency_slabs_match_the_whole_spectrum(monkeypatch, prec, kid):
    """When the source parents' spectra do not fit in device memory the V-list
    runs in slabs of kz: each slab's forward DFT rows, products and inverse-DFT
    contribution in turn (the transforms are linear).  The result equals the
    one-slab evaluation to rounding."""
    K = O.KERNELS[kid]
    src = points("gauss", 20000, 51)
    den = np.random.default_rng(52).uniform(-1, 1, (20000, K.k0))
    whole, ctx = gpu_eval(kid, 6, 40, src, den, src, prec=prec)
    ctx.close()
    monkeypatch.setenv("PVFMM_B200_VLIST_SLABS", "5")
    sliced, ctx = gpu_eval(kid, 6, 40, src, den, src, prec=prec)
    ctx.close()
    # plain: FP64 rounding only (2e-13 for Stokes); mixed: the slabs' FP32 inverse DFTs round
    # differently from one whole transform (measured 2e-7), within its bar
    tol = 1e-12 if prec == P.PRECISION_PLAIN else 1e-6
    assert O.rel_l2(sliced.reshape(-1), whole.reshape(-1)) < tol


def test_double_layer_setup0_and_rejections():
    """setup=0 with new double-layer values equals a fresh setup=1; a setup=0
    call must pass the same densities as its setup; kernels without a
    double-layer kernel reject dl_den with a message and NaN outputs."""
    rng = np.random.default_rng(77)
    src = points("gauss", 3000, 78)
    trg = points("unif", 1000, 79)
    sl = rng.uniform(-1, 1, 3000)
    dl1 = rng.uniform(-1, 1, 3000 * 4)
    dl2 = rng.uniform(-1, 1, 3000 * 4)
    s, t = src.reshape(-1), trg.reshape(-1)
    ctx = P.FMMParticleContext(-1, 40, 6, P.FMMKernel.LaplacePotential)
    ctx.evaluate(s, sl, dl1, t, True)
    again = ctx.evaluate(s, sl, dl2, t, False)
    fresh = P.FMMParticleContext(-1, 40, 6, P.FMMKernel.LaplacePotential)
    want = fresh.evaluate(s, sl, dl2, t, True)
    assert O.rel_l2(again, want) < 1e-14
    with pytest.raises(RuntimeError, match="same densities"):
        ctx.evaluate(s, None, dl2, t, False)
    ctx.close()
    fresh.close()
    g = P.FMMParticleContext(-1, 40, 6, P.FMMKernel.LaplaceGradient)
    with pytest.raises(RuntimeError, match="double-layer"):
        g.evaluate(s, sl, dl1, t, True)
    g.close()
