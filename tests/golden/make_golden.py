"""Generates the golden fixtures under tests/golden/.

mortonid_ref.npz   outputs of the reference's own Morton-id code
                   (src/mortonid.cpp, include/mortonid.txx), compiled from the
                   reference sources by oracle/ref_mortonid/build.sh: point ids,
                   the stable sort order under MortonId::operator<, Children()
                   and NbrList().  Needs the reference tree (this container).
oracle_*.npz       small FMM cases of the oracle (inputs, leaf ids, outputs),
                   regression pins of the oracle itself.
reference_*.npz    the reference's own particle FMM (src/pvfmm-wrapper.cpp and
                   the templates it instantiates, built from the reference
                   sources by oracle/ref_fmm/build.sh) through its C interface
                   PVFMMCreateContextDWorld / PVFMMEvalD, free space: inputs,
                   outputs, and the octree (Morton ids, leaf flags, points per
                   leaf) and interaction lists (U0, U1, U2, W, X, V1) it built.
reference_config1.npz   the reference's output on the 100,000-point uniform
                   Laplace case (m=6, 300 points per leaf); the inputs are
                   regenerated from their seeds (checksums kept).

Run:  python tests/golden/make_golden.py [--force]   (existing oracle_*.npz and
reference_*.npz are kept unless --force).  The reference tree is read from
$PVFMM_REFERENCE (its build scripts' default otherwise).
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import pvfmm_oracle as O  # noqa: E402


def morton_golden():
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libmortonid_ref.so")
    subprocess.run(["bash", os.path.join(ROOT, "oracle", "ref_mortonid", "build.sh")], check=True)
    lib = ctypes.CDLL(lib_path)
    rng = np.random.default_rng(2024)
    # point coordinates, including edge values
    c = rng.random((3000, 3))
    c[:8] = [[0, 0, 0], [1 - 2 ** -53, 0.5, 0.25], [0.5, 0.5, 0.5], [2 ** -30, 2 ** -31, 0],
             [0.999999999, 0.000000001, 0.5], [0.75, 0.25, 0.125], [1 - 2 ** -31, 1 - 2 ** -30, 2 ** -29], [0.3, 0.3, 0.3]]
    c = np.ascontiguousarray(c)
    pid = np.zeros((len(c), 4), dtype=np.int64)
    lib.ref_point_ids(c.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(len(c)), pid.ctypes.data_as(ctypes.c_void_p))
    # node ids at random depths (coordinates truncated to the depth), with
    # duplicates and ancestor/descendant pairs
    n = 4000
    d = rng.integers(0, 31, n)
    X = rng.integers(0, 1 << 30, (n, 3))
    X[n // 2:] = X[: n // 2]                  # shared coordinates at other depths
    for i in range(n):
        X[i] &= ~((1 << (30 - d[i])) - 1)
    ids = np.ascontiguousarray(np.concatenate([X, d[:, None]], axis=1).astype(np.int64))
    order = np.zeros(n, dtype=np.int64)
    lib.ref_sort(ids.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(n), order.ctypes.data_as(ctypes.c_void_p))
    sub = ids[ids[:, 3] < 30][:300].copy()
    ch = np.zeros((len(sub) * 8, 4), dtype=np.int64)
    lib.ref_children(sub.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(len(sub)), ch.ctypes.data_as(ctypes.c_void_p))
    sub2 = np.ascontiguousarray(ids[ids[:, 3] > 0][:300])
    nb = np.zeros((len(sub2) * 27, 4), dtype=np.int64)
    lib.ref_nbrs(sub2.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(len(sub2)), nb.ctypes.data_as(ctypes.c_void_p))
    np.savez_compressed(os.path.join(HERE, "mortonid_ref.npz"), coords=c, coord_ids=pid[:, :3],
                        xyz=ids[:, :3], depth=ids[:, 3], order=order, child_of=sub, children=ch,
                        nbr_of=sub2, nbrs=nb.reshape(len(sub2), 27, 4))


def oracle_golden(force=False):
    cases = {
        "laplace_m4": (0, 4, 40, 1200, False),
        "stokes_m4": (3, 4, 40, 600, False),
        "laplace_potgrad_m6": (6, 6, 50, 1500, True),
        "stokes_press_m4": (2, 4, 40, 600, False),
        "stokes_grad_m4": (4, 4, 40, 600, True),
        "biot_savart_m4": (5, 4, 40, 600, False),
    }
    for name, (kid, m, mp, n, sep) in cases.items():
        if not force and os.path.exists(os.path.join(HERE, f"oracle_{name}.npz")):
            continue
        rng = np.random.default_rng(100 + kid + m)
        K = O.KERNELS[kid]
        src = rng.random((n, 3))
        trg = rng.random((n // 2, 3)) * 0.8 + 0.1 if sep else src
        den = rng.uniform(-1, 1, (n, K.k0))
        out, fmm = O.pvfmm_eval(kid, m, mp, src, den, trg, return_fmm=True)
        np.savez_compressed(os.path.join(HERE, f"oracle_{name}.npz"), kernel=kid, m=m, max_pts=mp, src=src, den=den,
                            trg=trg, out=out, leaf_keys=np.array(fmm.tree.leaf_keys()))


def points(dist, n, seed):
    """Seeded point sets of the reference-pinned cases (also used by tests)."""
    rng = np.random.default_rng(seed)
    if dist == "unif":
        return rng.random((n, 3))
    if dist == "gauss":        # 8 isotropic Gaussians, sigma 0.02, clipped to the unit cube
        c = rng.uniform(0.1, 0.9, (8, 3))
        return np.clip(c[rng.integers(0, 8, n)] + 0.02 * rng.standard_normal((n, 3)), 0, 1)
    if dist == "sphere":       # ellipsoid surface, semi-axes (0.45, 0.3, 0.15)
        u = rng.standard_normal((n, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        return 0.5 + np.array([0.45, 0.3, 0.15]) * u
    if dist == "coincident":   # half the points on one spot: a tree to the maximum depth
        x = rng.random((n, 3))
        x[: n // 2] = x[0]
        x[n // 2: n // 2 + 20] = x[n - 1]
        return x
    raise ValueError(dist)


# name: (kernel id of the C interface, m, max points per leaf, distribution,
# n, separate targets, input seed)
REFERENCE_CASES = {
    "laplace_unif_m6": (0, 6, 50, "unif", 3000, False, 1),
    "laplace_grad_unif_m6": (1, 6, 50, "unif", 3000, False, 1),   # same inputs: pot + grad
    "laplace_gauss_m6": (0, 6, 50, "gauss", 5000, False, 2),
    "laplace_gauss_m8": (0, 8, 120, "gauss", 8000, False, 3),
    "laplace_sphere_m4": (0, 4, 40, "sphere", 4000, False, 4),
    "laplace_coincident_m4": (0, 4, 60, "coincident", 3000, False, 5),
    "laplace_sep_m6": (0, 6, 50, "unif", 3000, True, 6),
    "stokes_vel_m4": (3, 4, 60, "unif", 3000, False, 7),
    "stokes_vel_gauss_m6": (3, 6, 80, "gauss", 3000, False, 8),
    "stokes_press_m4": (2, 4, 60, "unif", 2000, False, 9),
    "stokes_grad_m4": (4, 4, 60, "unif", 2000, False, 10),
    "biot_savart_m4": (5, 4, 60, "unif", 2000, False, 11),
    # double-layer sources (dl_den: k0 + 3 values per point), alone or with
    # single-layer densities on the same points
    "laplace_dl_unif_m6": (0, 6, 50, "unif", 3000, False, 12, "dl"),
    "laplace_sldl_gauss_m6": (0, 6, 50, "gauss", 4000, True, 13, "sldl"),
    "stokes_dl_m4": (3, 4, 60, "unif", 2000, False, 14, "dl"),
    "stokes_sldl_gauss_m4": (3, 4, 60, "gauss", 2000, True, 15, "sldl"),
}
KDIM = {0: (1, 1), 1: (1, 3), 2: (3, 1), 3: (3, 3), 4: (3, 9), 5: (3, 3)}


def case_spec(name):
    """(kernel, m, max_pts, distribution, n, separate targets, seed, layers),
    layers "sl" (single layer), "dl" (double layer) or "sldl" (both)."""
    spec = REFERENCE_CASES[name]
    return spec if len(spec) == 8 else spec + ("sl",)


def reference_case_inputs(name):
    """src, sl_den (None when not passed), trg (None: the sources), dl_den
    (None when not passed)."""
    kid, m, mp, dist, n, sep, seed, layers = case_spec(name)
    src = points(dist, n, seed)
    trg = points("unif", n // 2, seed + 100) * 0.8 + 0.1 if sep else None
    den = np.random.default_rng(seed + 200).uniform(-1, 1, (n, KDIM[kid][0])) if "sl" in layers else None
    dl = None
    if "dl" in layers:
        dl = np.random.default_rng(seed + 300).uniform(-1, 1, (n, KDIM[kid][0] + 3))
    return src, den, trg, dl


# The reference's C++ interface (PtFMM_CreateTree with a separate
# double-layer point set): kernel, m, max_pts, seed
CPP_DL_CASES = {"laplace_dl_m6": (0, 6, 50, 21), "stokes_dl_m4": (3, 4, 60, 22)}


def cpp_dl_inputs(name):
    """Single-layer points (uniform), double-layer points (denser towards a
    corner), targets (uniform), all in [0,1)^3, and their values."""
    kid, _, _, seed = CPP_DL_CASES[name]
    rng = np.random.default_rng(seed)
    k0 = KDIM[kid][0]
    sl = rng.random((2000, 3))
    dl = rng.random((1500, 3)) ** 2
    trg = rng.random((1000, 3))
    return sl, rng.uniform(-1, 1, (2000, k0)), dl, rng.uniform(-1, 1, (1500, k0 + 3)), trg


def config1_inputs():
    """Laplace potential, 100,000 points i.i.d. uniform in [0,1)^3 (PCG64
    seed 1), densities uniform [-1,1] (seed 2)."""
    x = np.random.default_rng(1).random((100000, 3))
    q = np.random.default_rng(2).uniform(-1, 1, 100000)
    return x, q


def reference_golden(force=False):
    from oracle.ref_fmm import refpvfmm as R
    if not R.available():
        subprocess.run(["bash", os.path.join(ROOT, "oracle", "ref_fmm", "build.sh")], check=True)
    for name in REFERENCE_CASES:
        kid, m, mp = case_spec(name)[:3]
        path = os.path.join(HERE, f"reference_{name}.npz")
        if not force and os.path.exists(path):
            continue
        src, den, trg, dl = reference_case_inputs(name)
        out, tree, lists = R.ref_eval(kid, m, mp, src, den, trg, dl=dl)
        extra = {} if dl is None else {"dl": dl}     # an empty den means sl_den = NULL
        np.savez_compressed(path, kernel=kid, m=m, max_pts=mp, src=src,
                            den=np.zeros((0, KDIM[kid][0])) if den is None else den,
                            trg=np.zeros((0, 3)) if trg is None else trg, out=out,
                            nodes=tree[:, :7].astype(np.int32), lists=lists[:, :4].astype(np.int32), **extra)
    for name, (kid, m, mp, seed) in CPP_DL_CASES.items():
        path = os.path.join(HERE, f"refcpp_{name}.npz")
        if not force and os.path.exists(path):
            continue
        sl, sd, dl, dd, trg = cpp_dl_inputs(name)
        out = R.ref_ptfmm_eval(kid, m, mp, sl, sd, dl, dd, trg)
        np.savez_compressed(path, kernel=kid, m=m, max_pts=mp, sl=sl, sd=sd, dl=dl, dd=dd, trg=trg, out=out)
    path = os.path.join(HERE, "reference_config1.npz")
    if force or not os.path.exists(path):
        x, q = config1_inputs()
        out, tree, _ = R.ref_eval(0, 6, 300, x, q)
        np.savez_compressed(path, out=out.reshape(-1), x_sum=x.sum(), q_sum=q.sum(), x_first=x[:4], q_first=q[:4],
                            n_nodes=len(tree), n_leaves=int(tree[:, 4].sum()))


if __name__ == "__main__":
    if os.path.isdir(os.environ.get("PVFMM_REFERENCE", "/root/reference")):
        morton_golden()
        reference_golden(force="--force" in sys.argv)
    oracle_golden(force="--force" in sys.argv)
    print("golden fixtures written to", HERE)
