"""CPU tests of the oracle (the numpy restatement of PVFMM's particle FMM).

The reference has no unit tests or golden vectors for this path; its own
checks are (a) FMM vs. direct sum in the examples
(examples/include/utils.txx:7-109, examples/src/example1.cpp:102-140) and
(b) direct kernel formulas in julia/test/reference_comparison.jl:32-103.
These tests pin the oracle against both, against the reference's own
Morton-id code (golden vectors from src/mortonid.cpp compiled from source),
and against committed golden fixtures of the oracle itself.
"""
import math
import os

import numpy as np
import pytest

from oracle import pvfmm_oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


# --- kernels vs the reference's Julia direct formulas (up to the PVFMM scale factor)
def _julia_laplace(src, q, trg):
    out = np.zeros(len(trg))
    for t, xt in enumerate(trg):
        r = xt - src
        r2 = (r * r).sum(1)
        m = r2 > 1e-24
        out[t] = (q[m] / np.sqrt(r2[m])).sum()
    return out


def _julia_grad(src, q, trg):
    out = np.zeros((len(trg), 3))
    for t, xt in enumerate(trg):
        r = xt - src
        r2 = (r * r).sum(1)
        m = r2 > 1e-24
        out[t] = ((-q[m] / (r2[m] * np.sqrt(r2[m])))[:, None] * r[m]).sum(0)
    return out


def _julia_stokes(src, f, trg):
    out = np.zeros((len(trg), 3))
    for t, xt in enumerate(trg):
        r = xt - src
        r2 = (r * r).sum(1)
        m = r2 > 1e-24
        invr = 1 / np.sqrt(r2[m])
        invr3 = invr ** 3
        out[t] = (invr[:, None] * f[m] + ((r[m] * f[m]).sum(1) * invr3)[:, None] * r[m]).sum(0)
    return out


def test_kernels_match_reference_formulas():
    rng = np.random.default_rng(11)
    src = rng.random((40, 3))
    trg = rng.random((35, 3)) + 1.5
    q = rng.uniform(-1, 1, 40)
    f = rng.standard_normal((40, 3))
    np.testing.assert_allclose(O.LAPLACE.eval(src, q, trg)[:, 0], _julia_laplace(src, q, trg) / (4 * math.pi),
                               rtol=1e-13)
    # PVFMM's laplace_grad returns +r q / r^3 / 4pi, i.e. minus the gradient (kernel.txx:1316-1330)
    np.testing.assert_allclose(O.LAPLACE_GRAD.eval(src, q, trg), -_julia_grad(src, q, trg) / (4 * math.pi),
                               rtol=1e-13)
    np.testing.assert_allclose(O.STOKES.eval(src, f.reshape(-1), trg), _julia_stokes(src, f, trg) / (8 * math.pi),
                               rtol=1e-13)
    pg = O.LAPLACE_PG.eval(src, q, trg)
    np.testing.assert_allclose(pg[:, 0], O.LAPLACE.eval(src, q, trg)[:, 0], rtol=1e-14)
    np.testing.assert_allclose(pg[:, 1:], O.LAPLACE_GRAD.eval(src, q, trg), rtol=1e-14)


def test_self_interaction_is_masked():
    x = np.array([[0.3, 0.4, 0.5], [0.3, 0.4, 0.5], [0.6, 0.1, 0.2]])
    out = O.LAPLACE.eval(x, np.array([1.0, 2.0, 3.0]), x[:1])
    assert np.isfinite(out).all()
    np.testing.assert_allclose(out[0, 0], 3.0 / np.linalg.norm(x[0] - x[2]) / (4 * math.pi))


# --- FMM vs direct sum (the reference examples' self-check)
@pytest.mark.parametrize("kid,m,tol", [(0, 4, 1e-3), (0, 6, 2e-5), (0, 8, 5e-7), (1, 6, 1e-4), (3, 4, 1e-2),
                                       (6, 6, 1e-4)])
def test_fmm_matches_direct_sum(kid, m, tol):
    rng = np.random.default_rng(3)
    K = O.KERNELS[kid]
    n = 2500
    x = rng.random((n, 3))
    q = rng.uniform(-1, 1, (n, K.k0))
    out = O.pvfmm_eval(kid, m, 60, x, q, x)
    ref = O.direct_sum(kid, x, q, x)
    assert O.rel_l2(out, ref) < tol


def test_error_decreases_with_order():
    rng = np.random.default_rng(5)
    x = rng.random((2500, 3))
    q = rng.uniform(-1, 1, 2500)
    ref = O.direct_sum(0, x, q, x)
    errs = [O.rel_l2(O.pvfmm_eval(0, m, 60, x, q, x), ref) for m in (4, 6, 8)]
    assert errs[0] > 10 * errs[1] > 100 * errs[2] * 0.1


def test_separate_targets_and_scaling():
    """Sources and targets in different boxes: exercises the bounding-box map
    and the output scaling by scale_x^trg_scal (pvfmm-wrapper.cpp:458-541)."""
    rng = np.random.default_rng(9)
    src = rng.random((1500, 3)) * 3.0 - 1.0
    trg = rng.random((700, 3)) * 2.0 + 0.5
    q = rng.uniform(-1, 1, 1500)
    for kid, tol in [(0, 5e-5), (1, 5e-4)]:
        out = O.pvfmm_eval(kid, 6, 50, src, q, trg)
        ref = O.direct_sum(kid, src, q, trg)
        assert O.rel_l2(out, ref) < tol


# --- tree properties
def _tree(x, max_pts=40):
    f = O.FMM(0, 4, max_pts)
    f.setup(x, x)
    return f.tree


def test_tree_is_2to1_balanced_and_partitions_points():
    rng = np.random.default_rng(2)
    c = rng.uniform(0.2, 0.8, (3, 3))
    x = np.clip(c[rng.integers(0, 3, 3000)] + 0.01 * rng.standard_normal((3000, 3)), 0, 0.999)
    T = _tree(x)
    N = T.nodes
    leaves = [n for n in N if n.leaf]
    assert sum(n.n_trg for n in leaves) == 3000
    for n in N:
        if not n.leaf:
            assert sum(N[n.child0 + c].n_trg for c in range(8)) == n.n_trg
    # 2:1: every leaf's colleague-level neighbour region is covered by leaves at depth >= d-1
    by_key = {(n.X, n.Y, n.Z, n.depth): n for n in N}
    for n in leaves:
        w = O.TWO30 >> n.depth
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    X, Y, Z = n.X + dx * w, n.Y + dy * w, n.Z + dz * w
                    if not (0 <= X < O.TWO30 and 0 <= Y < O.TWO30 and 0 <= Z < O.TWO30):
                        continue
                    # the node containing (X,Y,Z) at depth >= n.depth-1 must exist
                    d = n.depth - 1
                    if d < 0:
                        continue
                    pm = ~((O.TWO30 >> d) - 1)
                    assert (X & pm, Y & pm, Z & pm, d) in by_key


def test_leaf_counts_respect_max_points():
    rng = np.random.default_rng(4)
    x = rng.random((4000, 3))
    T = _tree(x, max_pts=50)
    for n in T.nodes:
        if n.leaf:
            assert n.n_src + n.n_trg <= 50 or n.depth >= O.MAX_DEPTH - 1


def test_coincident_points_reach_max_depth():
    x = np.full((40, 3), 0.3)
    x[20:] = 0.7
    T = _tree(x, max_pts=10)
    assert T.depth == O.MAX_DEPTH - 1


# --- Morton order vs the reference's own mortonid.cpp (golden vectors)
def test_morton_order_matches_reference_golden():
    path = os.path.join(GOLDEN, "mortonid_ref.npz")
    g = np.load(path)
    xyz, depth, order = g["xyz"], g["depth"], g["order"]
    hi, lo = O.interleave_key(xyz[:, 0], xyz[:, 1], xyz[:, 2], depth)
    ours = np.lexsort((lo, hi))
    np.testing.assert_array_equal(ours, order)
    # point ids from coordinates: floor(c * 2^30)
    np.testing.assert_array_equal(O.morton_coords(g["coords"]), g["coord_ids"])
    # Children() and NbrList()
    np.testing.assert_array_equal(_children(g["child_of"]), g["children"])
    for ids, nb in zip(g["nbr_of"], g["nbrs"]):
        ref = [tuple(r) for r in nb if r[3] >= 0]
        assert O.nbr_list(*[int(v) for v in ids]) == ref


def _children(ids):
    out = []
    for X, Y, Z, d in ids:
        w = O.TWO30 >> (d + 1)
        for c in range(8):
            out.append((X + w * (c & 1), Y + w * ((c >> 1) & 1), Z + w * ((c >> 2) & 1), d + 1))
    return np.array(out)


# --- committed golden fixtures of the oracle
@pytest.mark.parametrize("name", ["laplace_m4", "stokes_m4", "laplace_potgrad_m6", "stokes_press_m4",
                                  "stokes_grad_m4", "biot_savart_m4"])
def test_oracle_golden_fixture(name):
    g = np.load(os.path.join(GOLDEN, f"oracle_{name}.npz"))
    out, fmm = O.pvfmm_eval(int(g["kernel"]), int(g["m"]), int(g["max_pts"]), g["src"], g["den"], g["trg"],
                            return_fmm=True)
    np.testing.assert_array_equal(np.array(fmm.tree.leaf_keys()), g["leaf_keys"])
    np.testing.assert_allclose(out, g["out"], rtol=0, atol=1e-12 * np.abs(g["out"]).max())
