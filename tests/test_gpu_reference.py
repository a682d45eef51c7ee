"""GPU parity against the reference's own particle FMM (fixtures
tests/golden/reference_*.npz, written by the reference compiled from its
sources; see tests/test_reference_pins.py for how they were made and why two
cases carry wider bars).

The plain FP64 CUDA path must build the reference's octree (the same Morton
ids, leaf flags and points per leaf) and reproduce its outputs to 1e-12
relative L2; the mixed form must stay within its accuracy bar (1e-6) of the
reference.  The FP64 translation products (translate.cu) are checked against
an FP64 product on the host.
"""
import ctypes
import glob
import os

import numpy as np
import pytest

import pvfmm_b200 as P
from oracle import pvfmm_oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
GPU_KERNELS = {0, 1, 2, 3, 4, 5}
FIXTURES = sorted(f for f in glob.glob(os.path.join(GOLDEN, "reference_*.npz"))
                  if "config1" not in f and not os.path.basename(f).startswith(("reference_periodic_", "reference_bc_"))
                  and int(np.load(f)["kernel"]) in GPU_KERNELS)
TOL = {"reference_laplace_coincident_m4.npz": 1e-7, "reference_stokes_vel_gauss_m6.npz": 1e-11,
       "reference_stokes_dl_m4.npz": 1e-11, "reference_stokes_sldl_gauss_m4.npz": 1e-10}


def gpu_eval(kid, m, mp, src, den, trg, prec=P.PRECISION_PLAIN, dl=None):
    ctx = P.FMMParticleContext(-1, mp, m, P.FMMKernel(kid), precision=prec)
    s = np.ascontiguousarray(src).reshape(-1)
    t = s if trg is None else np.ascontiguousarray(trg).reshape(-1)
    d = None if den is None else np.ascontiguousarray(den).reshape(-1)
    d2 = None if dl is None else np.ascontiguousarray(dl).reshape(-1)
    out = ctx.evaluate(s, d, d2, t, True)
    return out, ctx


def fixture_densities(z):
    """(sl_den, dl_den) of a fixture; an empty array or a missing one is NULL."""
    den = z["den"] if len(z["den"]) else None
    dl = z["dl"] if "dl" in z.files and len(z["dl"]) else None
    return den, dl


def check_tree(ctx, nodes):
    keys = ctx.tree_data(2).reshape(-1, 4)
    leaf = ctx.tree_data(3)
    src = ctx.tree_data(4).reshape(-1, 2)
    trg = ctx.tree_data(5).reshape(-1, 2)
    ours = {tuple(int(v) for v in k): i for i, k in enumerate(keys)}
    ref = {tuple(int(v) for v in r[:4]): r for r in nodes}
    assert set(ours) == set(ref), (len(ours), len(ref))
    for k, i in ours.items():
        r = ref[k]
        assert bool(leaf[i]) == bool(r[4]), k
        if leaf[i]:
            assert int(trg[i][1] - trg[i][0]) == int(r[6]), k
            assert int(src[i][1] - src[i][0]) == int(r[5]), k


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(f)[10:-4] for f in FIXTURES])
def test_plain_matches_reference(path):
    z = np.load(path)
    kid, m, mp = int(z["kernel"]), int(z["m"]), int(z["max_pts"])
    trg = z["trg"] if len(z["trg"]) else None
    den, dl = fixture_densities(z)
    out, ctx = gpu_eval(kid, m, mp, z["src"], den, trg, dl=dl)
    check_tree(ctx, z["nodes"])
    err = O.rel_l2(out.reshape(-1), z["out"].reshape(-1))
    assert err < TOL.get(os.path.basename(path), 1e-12), err
    assert ctx.launch_count() > 0
    ctx.close()


@pytest.mark.parametrize("name", ["laplace_unif_m6", "laplace_gauss_m8", "laplace_sep_m6", "laplace_grad_unif_m6"])
def test_mixed_within_bar_of_reference(name):
    z = np.load(os.path.join(GOLDEN, f"reference_{name}.npz"))
    kid, m, mp = int(z["kernel"]), int(z["m"]), int(z["max_pts"])
    trg = z["trg"] if len(z["trg"]) else None
    out, ctx = gpu_eval(kid, m, mp, z["src"], z["den"], trg, prec=P.PRECISION_MIXED)
    ref = z["out"].reshape(len(out.reshape(-1)) // z["out"].shape[-1], -1)
    o = out.reshape(ref.shape)
    for k in range(ref.shape[1]):
        assert O.rel_l2(o[:, k], ref[:, k]) < 1e-6, k
    ctx.close()


def test_potgrad_matches_reference_potential_and_gradient():
    zp = np.load(os.path.join(GOLDEN, "reference_laplace_unif_m6.npz"))
    zg = np.load(os.path.join(GOLDEN, "reference_laplace_grad_unif_m6.npz"))
    out, ctx = gpu_eval(6, 6, 50, zp["src"], zp["den"], None)
    out = out.reshape(-1, 4)
    ref = np.concatenate([zp["out"].reshape(-1, 1), zg["out"].reshape(-1, 3)], axis=1)
    for k in range(4):
        assert O.rel_l2(out[:, k], ref[:, k]) < 1e-12, k
    ctx.close()


def test_config1_matches_reference_on_every_target():
    """100,000 uniform points, Laplace potential, m=6, 300 points per leaf:
    the plain form against the reference's output on all targets."""
    z = np.load(os.path.join(GOLDEN, "reference_config1.npz"))
    x = np.random.default_rng(1).random((100000, 3))
    q = np.random.default_rng(2).uniform(-1, 1, 100000)
    assert np.array_equal(x[:4], z["x_first"]) and np.array_equal(q[:4], z["q_first"])
    assert x.sum() == z["x_sum"] and q.sum() == z["q_sum"]
    out, ctx = gpu_eval(0, 6, 300, x, q, None)
    assert ctx.tree_stats()["n_nodes"] == int(z["n_nodes"])
    assert O.rel_l2(out.reshape(-1), z["out"]) < 1e-12
    ctx.close()


def _translate_check():
    lib = P.load_library()
    f = lib.PVFMMB200TranslateGemmCheck
    f.restype = ctypes.c_int
    vp = ctypes.c_void_p
    f.argtypes = [ctypes.c_long, ctypes.c_int, ctypes.c_int, vp, ctypes.c_long, vp, vp, vp, ctypes.c_long, vp, vp,
                  ctypes.c_int, ctypes.c_int]
    return f


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


@pytest.mark.parametrize("M,N,K,gather,scatter,scale,acc,ksplit", [
    (1000, 296, 296, False, False, False, False, 1),     # S2U / D2T pseudo-inverse products
    (777, 296, 2368, False, True, False, False, 1),      # U2U: 8 children per row, rows scattered to parents
    (777, 296, 2368, False, True, False, False, 8),      # U2U with K split per child
    (3, 296, 2368, False, True, True, True, 8),          # split K with scaling and accumulation, few rows
    (333, 2368, 296, True, False, False, True, 1),       # D2D: parents gathered, children accumulated
    (1500, 296, 296, True, False, True, False, 1),       # D2T first product: gathered, scaled by 2^-depth
    (65, 152, 10, False, False, False, False, 1),        # ragged tiles in every direction
    (64 * 65536 + 70, 8, 4, False, False, False, False, 1),   # more than one launch of row tiles
])
def test_translate_products_match_fp64_host_products(M, N, K, gather, scatter, scale, acc, ksplit):
    f = _translate_check()
    rng = np.random.default_rng(M + N + K)
    a_rows = M + 50 if gather else M
    c_rows = M + 40 if scatter else M
    A = rng.standard_normal((a_rows, K))
    B = rng.standard_normal((K, N))
    C = rng.standard_normal((c_rows, N)) if acc else np.zeros((c_rows, N))
    arows = rng.permutation(a_rows)[:M].astype(np.int32) if gather else None
    crows = rng.permutation(c_rows)[:M].astype(np.int32) if scatter else None
    depth = rng.integers(0, 20, a_rows).astype(np.int32) if scale else None
    want = C.copy()
    Ag = A[arows] if gather else A
    prod = Ag @ B
    if scale:
        prod *= np.ldexp(1.0, -depth[arows] if gather else -depth)[:, None]
    if scatter:
        want[crows] = prod + (C[crows] if acc else 0)
    else:
        want = prod + (C if acc else 0)
    got = C.copy()
    rc = f(M, N, K, _p(A), a_rows, _p(arows), _p(B), _p(got), c_rows, _p(crows), _p(depth), 1 if acc else 0, ksplit)
    assert rc == 0, P.last_error()
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err < 1e-14 * max(1, K / 64), err


@pytest.mark.parametrize("name", ["stokes_press_m4", "stokes_grad_m4", "biot_savart_m4", "stokes_vel_m4"])
def test_mixed_self_expanding_kernels_as_accurate_as_plain(name):
    """The mixed form of the kernels with 3-component expansions (Stokes
    velocity, pressure, velocity gradient, Biot-Savart) against an FP64 direct
    sum: as accurate as the plain form (the m=4 truncation error dominates)."""
    z = np.load(os.path.join(GOLDEN, f"reference_{name}.npz"))
    kid, m, mp = int(z["kernel"]), int(z["m"]), int(z["max_pts"])
    src, den = z["src"], z["den"]
    out, ctx = gpu_eval(kid, m, mp, src, den, None, prec=P.PRECISION_MIXED)
    ctx.close()
    direct = O.direct_sum(kid, src, den, src).reshape(-1)
    err_plain = O.rel_l2(z["out"].reshape(-1), direct)
    assert O.rel_l2(out.reshape(-1), direct) < 1.5 * err_plain + 1e-6


DL_CASES = ["laplace_dl_unif_m6", "laplace_sldl_gauss_m6", "stokes_dl_m4", "stokes_sldl_gauss_m4"]


@pytest.mark.parametrize("name", DL_CASES)
def test_mixed_double_layer_as_accurate_as_plain(name):
    """Double-layer sources in the mixed form (FP32 near field with hi/lo
    coordinates) against the direct sum the reference's frame defines: as
    accurate as the reference's FP64 FMM, to within 1e-6.  (For Stokes the
    reference's own FMM is 0.15-0.4 from the direct sum: the v1 v1 + v2 v2
    of its n.f adds a point-source flow r/r^3, whose net flux Stokeslet
    equivalent surfaces cannot carry; the bar is relative to that.)"""
    z = np.load(os.path.join(GOLDEN, f"reference_{name}.npz"))
    kid, m, mp = int(z["kernel"]), int(z["m"]), int(z["max_pts"])
    src = z["src"]
    den, dl = fixture_densities(z)
    trg = z["trg"] if len(z["trg"]) else None
    out, ctx = gpu_eval(kid, m, mp, src, den, trg, prec=P.PRECISION_MIXED, dl=dl)
    ctx.close()
    t = src if trg is None else trg
    direct = O.direct_sum_mapped(kid, src, den, t, dl_den=dl).reshape(-1)
    err_plain = O.rel_l2(z["out"].reshape(-1), direct)
    assert O.rel_l2(out.reshape(-1), direct) < 1.5 * err_plain + 1e-6
