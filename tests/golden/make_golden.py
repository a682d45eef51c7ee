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
reference_periodic_*.npz   the same, periodic (box_size > 0), from the
                   reference's default build (PVFMM_EXTENDED_BC) and, for the
                   lattice_* cases, from its build without that option
                   (oracle/_ref/libpvfmm_ref_avx2_lattice.so).
reference_bc_*.npz the periodic boundary operator (BC_Type entry 3 of the
                   reference's precompute file) through M V and M^T V for
                   seeded V.
refcppbc_*.npz     the reference's C++ interface (PtFMM_CreateTree,
                   PtFMM_Evaluate) with BoundaryType Periodic.

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
    if dist == "corner":       # two clusters across the periodic faces (corner and an edge), the rest uniform
        x = rng.random((n, 3))
        k = n // 3
        x[:k] = 0.03 * rng.standard_normal((k, 3))                      # around (0, 0, 0)
        x[k:2 * k] = np.array([0.5, 1.0, 0.0]) + 0.03 * rng.standard_normal((k, 3))
        return x                                                          # wrapped by the periodic map
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


# Periodic boundaries (box_size > 0): kernel, m, max_pts, distribution, n
# sources, separate targets, seed, box size, lattice (False: the reference's
# default build, the 5x5x5-image boundary operator; True: the build without
# PVFMM_EXTENDED_BC, the lattice sum).  The points are scaled to the box and
# a tenth of them moved by whole periods, so that the wrap is exercised.
PERIODIC_CASES = {
    "laplace_unif_m6": (0, 6, 50, "unif", 3000, False, 31, 2.0, False),
    "laplace_grad_unif_m6": (1, 6, 50, "unif", 3000, False, 31, 2.0, False),
    "laplace_gauss_m6": (0, 6, 50, "gauss", 4000, False, 32, 1.0, False),
    "laplace_sep_m6": (0, 6, 50, "unif", 3000, True, 33, 1.0, False),
    "laplace_small_m6": (0, 6, 50, "unif", 300, False, 34, 1.0, False),
    "stokes_vel_m4": (3, 4, 60, "unif", 2000, False, 35, 1.0, False),
    # clusters across the faces: adaptive leaves whose U, W and X lists wrap
    "laplace_corner_m6": (0, 6, 40, "corner", 4000, False, 39, 1.0, False),
    "stokes_vel_corner_m4": (3, 4, 40, "corner", 3000, True, 40, 1.0, False),
    "lattice_laplace_corner_m6": (0, 6, 40, "corner", 4000, False, 41, 1.0, True),
    "lattice_laplace_unif_m6": (0, 6, 50, "unif", 3000, False, 36, 1.0, True),
    "lattice_laplace_grad_gauss_m6": (1, 6, 50, "gauss", 3000, False, 37, 1.0, True),
    "lattice_stokes_vel_m4": (3, 4, 60, "unif", 2000, False, 38, 1.5, True),
}
# periodic boundary operators pinned through their action on seeded vectors:
# kernel, m, lattice
PERIODIC_OPERATORS = {"laplace_m6": (0, 6, False), "stokes_vel_m4": (3, 4, False),
                      "lattice_laplace_m6": (0, 6, True), "lattice_laplace_grad_m6": (1, 6, True),
                      "lattice_stokes_vel_m4": (3, 4, True)}


def periodic_case_inputs(name):
    """src, sl_den, trg (None: the sources) of a periodic case, in box units."""
    kid, m, mp, dist, n, sep, seed, box, lattice = PERIODIC_CASES[name]
    rng = np.random.default_rng(seed + 500)
    src = points(dist, n, seed) * box
    shift = rng.integers(-2, 3, (n, 3)) * box
    src = src + np.where(rng.random((n, 1)) < 0.1, shift, 0.0)
    trg = points("unif", n // 2, seed + 100) * box if sep else None
    den = np.random.default_rng(seed + 200).uniform(-1, 1, (n, KDIM[kid][0]))
    return src, den, trg


def periodic_operator_probe(kid, m):
    """The seeded vectors (n x 4) the operator fixtures multiply."""
    n = (6 * (m - 1) ** 2 + 2) * KDIM[kid][0]
    return np.random.default_rng(1000 + kid * 16 + m).standard_normal((n, 4))


def _periodic_case(name):
    from oracle.ref_fmm import refpvfmm as R
    kid, m, mp, dist, n, sep, seed, box, lattice = PERIODIC_CASES[name]
    src, den, trg = periodic_case_inputs(name)
    out, tree, lists = R.ref_eval(kid, m, mp, src, den, trg, box_size=box, lattice=lattice)
    np.savez_compressed(os.path.join(HERE, f"reference_periodic_{name}.npz"), kernel=kid, m=m, max_pts=mp, src=src,
                        den=den, trg=np.zeros((0, 3)) if trg is None else trg, out=out, box=box, lattice=lattice,
                        nodes=tree[:, :7].astype(np.int32))


def _periodic_operator(name):
    import struct
    from oracle.ref_fmm import refpvfmm as R
    kid, m, lattice = PERIODIC_OPERATORS[name]
    ctx = R.RefContext(kid, m, 50, box_size=1.0, lattice=lattice)
    ctx.close()
    # the reference's precompute file holds BC_Type entry 3 (BoundaryType PXYZ == Periodic)
    d = R._lattice_dir[0] if lattice else os.environ["PVFMM_DIR"]
    kname = {0: "laplace", 1: "laplace_grad", 3: "stokes_vel"}[kid]
    b = open(os.path.join(d, f"Precomp_{kname}_m{m}.data"), "rb").read()
    pos, M = 8, None
    for t in range(16):
        cnt = struct.unpack_from("i", b, pos)[0]
        pos += 4
        for j in range(cnt):
            n1, n2 = struct.unpack_from("ii", b, pos)
            pos += 8
            if t == 15 and j == 3:
                M = np.frombuffer(b, dtype=np.float64, count=n1 * n2, offset=pos).reshape(n1, n2)
            pos += 8 * n1 * n2
    V = periodic_operator_probe(kid, m)
    np.savez_compressed(os.path.join(HERE, f"reference_bc_{name}.npz"), kernel=kid, m=m, lattice=lattice,
                        MtV=M.T @ V, MV=M @ V, norm=np.linalg.norm(M))


# The reference's C++ interface with periodic boundaries (coordinates in
# [0,1)^3 as given): kernel, m, max_pts, seed, double-layer points, lattice,
# BoundaryType (3 PXYZ == Periodic, 2 PXY, 1 PX)
CPP_PERIODIC_CASES = {"laplace_m6": (0, 6, 50, 51, False, False, 3), "stokes_vel_m4": (3, 4, 60, 52, False, False, 3),
                      "laplace_dl_m6": (0, 6, 50, 53, True, False, 3),
                      "lattice_laplace_m6": (0, 6, 50, 54, False, True, 3),
                      "px_laplace_m6": (0, 6, 50, 55, False, False, 1),
                      "pxy_laplace_m6": (0, 6, 50, 56, False, False, 2),
                      "pxy_stokes_vel_m4": (3, 4, 60, 57, False, False, 2),
                      "lattice_px_laplace_m6": (0, 6, 50, 58, False, True, 1),
                      "lattice_pxy_stokes_vel_m4": (3, 4, 60, 59, False, True, 2)}


def cpp_periodic_inputs(name):
    """Single-layer points (clustered across the periodic faces), their
    values, double-layer points and values (empty unless the case has them),
    targets (uniform); all in [0,1)^3."""
    kid, _, _, seed, with_dl, _, _ = CPP_PERIODIC_CASES[name]
    rng = np.random.default_rng(seed)
    k0 = KDIM[kid][0]
    sl = points("corner", 2000, seed) % 1.0
    dl = rng.random((1200 if with_dl else 0, 3))
    trg = rng.random((1000, 3))
    return sl, rng.uniform(-1, 1, (2000, k0)), dl, rng.uniform(-1, 1, (len(dl), k0 + 3)), trg


def _cpp_periodic_case(name):
    from oracle.ref_fmm import refpvfmm as R
    kid, m, mp, _, _, lattice, bndry = CPP_PERIODIC_CASES[name]
    sl, sd, dl, dd, trg = cpp_periodic_inputs(name)
    out = R.ref_ptfmm_eval(kid, m, mp, sl, sd, dl, dd, trg, lattice=lattice, bndry=bndry)
    np.savez_compressed(os.path.join(HERE, f"refcppbc_{name}.npz"), kernel=kid, m=m, max_pts=mp, lattice=lattice,
                        bndry=bndry, sl=sl, sd=sd, dl=dl, dd=dd, trg=trg, out=out)


def periodic_golden(force=False):
    """One process per fixture: the two reference builds are not loaded into
    one process."""
    for name in PERIODIC_CASES:
        if force or not os.path.exists(os.path.join(HERE, f"reference_periodic_{name}.npz")):
            subprocess.run([sys.executable, os.path.abspath(__file__), "--periodic-case", name], check=True)
    for name in PERIODIC_OPERATORS:
        if force or not os.path.exists(os.path.join(HERE, f"reference_bc_{name}.npz")):
            subprocess.run([sys.executable, os.path.abspath(__file__), "--periodic-operator", name], check=True)
    for name in CPP_PERIODIC_CASES:
        if force or not os.path.exists(os.path.join(HERE, f"refcppbc_{name}.npz")):
            subprocess.run([sys.executable, os.path.abspath(__file__), "--cpp-periodic-case", name], check=True)


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
    if "--periodic-case" in sys.argv:
        _periodic_case(sys.argv[sys.argv.index("--periodic-case") + 1])
        sys.exit(0)
    if "--periodic-operator" in sys.argv:
        _periodic_operator(sys.argv[sys.argv.index("--periodic-operator") + 1])
        sys.exit(0)
    if "--cpp-periodic-case" in sys.argv:
        _cpp_periodic_case(sys.argv[sys.argv.index("--cpp-periodic-case") + 1])
        sys.exit(0)
    if os.path.isdir(os.environ.get("PVFMM_REFERENCE", "/root/reference")):
        morton_golden()
        reference_golden(force="--force" in sys.argv)
        periodic_golden(force="--force" in sys.argv)
    oracle_golden(force="--force" in sys.argv)
    print("golden fixtures written to", HERE)
