"""Generates the golden fixtures under tests/golden/.

mortonid_ref.npz   outputs of the reference's own Morton-id code
                   (src/mortonid.cpp, include/mortonid.txx), compiled from the
                   reference sources by oracle/ref_mortonid/build.sh: point ids,
                   the stable sort order under MortonId::operator<, Children()
                   and NbrList().  Needs the reference tree (this container).
oracle_*.npz       small FMM cases of the oracle (inputs, leaf ids, outputs),
                   regression pins of the oracle itself.

Run:  python tests/golden/make_golden.py [--force]   (existing oracle_*.npz are
kept unless --force)
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


if __name__ == "__main__":
    if os.path.isdir("/root/reference"):
        morton_golden()
    oracle_golden(force="--force" in sys.argv)
    print("golden fixtures written to", HERE)
