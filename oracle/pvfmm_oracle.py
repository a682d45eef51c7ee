"""CPU oracle for PVFMM particle-FMM evaluation (test infrastructure only).

This module is a plain numpy restatement of the particle FMM path of PVFMM
(dmalhotra/pvfmm).  It is the checker for the CUDA library in ``pvfmm_b200``:
only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it, and nothing in the product calls it.

Every stage cites the reference code it follows:

* points -> unit box, density/output scaling: ``src/pvfmm-wrapper.cpp:458-541``
* Morton ids and their order: ``include/mortonid.txx:25-53, 107-118``
* refinement rule: ``include/fmm_node.txx:63-98``, ``include/mpi_node.txx:79-105``,
  the context's seed grid ``src/pvfmm-wrapper.cpp:416-432``
* 2:1 balance: ``include/mpi_tree.txx:745-943`` (``balanceOctree``)
* colleagues / interaction lists: ``include/mpi_tree.txx:1136-1256``,
  ``include/interac_list.txx:98-279``
* X/W <-> U reassignment by ``Nsrf``: ``include/fmm_pts.txx:4629, 4929, 5295, 5325``
* surfaces and operators: ``include/fmm_pts.txx:54-160, 453-764``
* S2U / U2U / V (FFT) / X / W / U / D2D / D2T: ``include/fmm_pts.txx:2275-2637,
  2689-2858, 3249-3759, 3989-5737``; driver order ``include/fmm_tree.txx:237-738``
* kernels: ``include/kernel.txx:1270-1364``

Parity status.  The reference cannot be built in this container (its SCTL
submodule, MPI and FFTW are absent), so the full FMM output of the oracle is
pinned against the reference's own self-check (FMM vs. direct sum,
``examples/include/utils.txx:7-109``) rather than against reference output.
The Morton ordering is pinned bit-exactly against the reference's own
``src/mortonid.cpp`` compiled from source (``oracle/ref_mortonid``).  Kernel
normalisations are pinned against the direct formulas of the reference's
Julia comparison test (``julia/test/reference_comparison.jl:32-103``).
Full-FMM parity against reference output: unpinned.
"""
from __future__ import annotations

import bisect
import math
import time
from dataclasses import dataclass, field

import numpy as np

MAX_DEPTH = 30          # PVFMM_MAX_DEPTH, include/pvfmm_common.hpp:29
RAD0 = 1.05             # PVFMM_RAD0, include/pvfmm_common.hpp:33
RAD1 = 2.95             # PVFMM_RAD1, include/pvfmm_common.hpp:34
TWO30 = 1 << MAX_DEPTH
# Scale exponents of the expansion kernels: K(x/2) = 2^(src+trg) K(x)
# (include/kernel.txx:64-196).  Every kernel here is homogeneous, so the
# reference's solve gives src = 0 and trg = the kernel's degree (KernelFn.deg).
EXP_SRC_SCAL = 0.0

# PVFMMKernel enum, include/pvfmm.h:21-28 (+ extension value 6 for pot+grad)
LAPLACE_POTENTIAL = 0
LAPLACE_GRADIENT = 1
STOKES_PRESSURE = 2
STOKES_VELOCITY = 3
STOKES_VELOCITY_GRAD = 4
BIOT_SAVART_POTENTIAL = 5
LAPLACE_POTGRAD = 6


# ----------------------------------------------------------------------------
# Kernels (include/kernel.txx:1270-1364)
# ----------------------------------------------------------------------------
@dataclass(frozen=True)
class KernelFn:
    """One kernel function: k0 source dims -> k1 target dims, homogeneous of
    degree ``deg``: K(x/2) = 2^deg K(x)."""
    name: str
    k0: int
    k1: int
    flops: int
    deg: float = 1.0

    def matrix(self, src: np.ndarray, trg: np.ndarray) -> np.ndarray:
        """BuildMatrix layout (include/kernel.txx:1059-1135):
        M[i*k0+j, t*k1+k] = K_jk(trg_t - src_i); r == 0 contributes 0."""
        src = np.asarray(src, dtype=np.float64).reshape(-1, 3)
        trg = np.asarray(trg, dtype=np.float64).reshape(-1, 3)
        r = trg[None, :, :] - src[:, None, :]            # (ns, nt, 3)
        r2 = np.einsum("ijk,ijk->ij", r, r)
        with np.errstate(divide="ignore"):
            rinv = np.where(r2 > 0, 1.0 / np.sqrt(np.where(r2 > 0, r2, 1.0)), 0.0)
        ns, nt = r2.shape
        if self.name == "laplace":
            K = (rinv / (4 * math.pi))[:, None, :, None]            # (ns,1,nt,1)
        elif self.name == "laplace_grad":
            rinv3 = rinv ** 3
            K = (r * (rinv3 / (4 * math.pi))[:, :, None])[:, None, :, :]   # (ns,1,nt,3)
        elif self.name == "laplace_potgrad":
            rinv3 = rinv ** 3
            K = np.empty((ns, 1, nt, 4))
            K[:, 0, :, 0] = rinv / (4 * math.pi)
            K[:, 0, :, 1:] = r * (rinv3 / (4 * math.pi))[:, :, None]
        elif self.name == "stokes_vel":
            rinv2 = rinv * rinv
            K = np.empty((ns, 3, nt, 3))
            for j in range(3):
                for k in range(3):
                    K[:, j, :, k] = rinv * ((1.0 if j == k else 0.0) + r[:, :, j] * r[:, :, k] * rinv2)
            K /= 8 * math.pi
        elif self.name == "stokes_press":        # kernel.txx:1366-1378: (r . f) / r^3 / (4 pi)
            K = (r * (rinv ** 3 / (4 * math.pi))[:, :, None]).transpose(0, 2, 1)[:, :, :, None]   # (ns,3,nt,1)
        elif self.name == "stokes_grad":         # kernel.txx:1404-1432
            # u[3a+b] = (r_b f_a - f_b r_a + (r.f)(delta_ab - 3 r_a r_b / r^2)) / r^3 / (8 pi)
            rinv2, rinv3 = rinv * rinv, rinv ** 3
            K = np.zeros((ns, 3, nt, 9))
            for j in range(3):
                for a in range(3):
                    for b in range(3):
                        v = r[:, :, j] * ((1.0 if a == b else 0.0) - 3 * r[:, :, a] * r[:, :, b] * rinv2)
                        if j == a:
                            v = v + r[:, :, b]
                        if j == b:
                            v = v - r[:, :, a]
                        K[:, j, :, 3 * a + b] = v * rinv3
            K /= 8 * math.pi
        elif self.name == "biot_savart":         # kernel.txx:1492-1505: (f x r) / r^3 / (4 pi)
            rinv3 = rinv ** 3 / (4 * math.pi)
            K = np.zeros((ns, 3, nt, 3))
            for j in range(3):
                for k in range(3):
                    for l in range(3):
                        eps = (j - k) * (k - l) * (l - j) / 2          # Levi-Civita symbol e_jlk
                        if eps:
                            K[:, j, :, k] += -eps * r[:, :, l] * rinv3
        else:
            raise ValueError(self.name)
        return K.reshape(ns * self.k0, nt * self.k1)

    def eval(self, src: np.ndarray, den: np.ndarray, trg: np.ndarray) -> np.ndarray:
        """Direct sum: returns (n_trg, k1) = sum_src K(trg - src) den."""
        src = np.asarray(src, dtype=np.float64).reshape(-1, 3)
        trg = np.asarray(trg, dtype=np.float64).reshape(-1, 3)
        den = np.asarray(den, dtype=np.float64).reshape(-1)
        if src.shape[0] == 0 or trg.shape[0] == 0:
            return np.zeros((trg.shape[0], self.k1))
        return (den @ self.matrix(src, trg)).reshape(-1, self.k1)


@dataclass(frozen=True)
class DblKernelFn:
    """A double-layer kernel: each source carries k0 + 3 values (a density and
    a normal), and the kernel is bilinear in them, so it has no matrix form.
    ``eval`` follows the reference's uKerEval for the kernel literally,
    including which source value it reads as which quantity."""
    name: str
    k0: int             # values per source point (k0 of the kernel + 3)
    k1: int
    flops: int

    def eval(self, src: np.ndarray, val: np.ndarray, trg: np.ndarray, chunk: int = 256) -> np.ndarray:
        src = np.asarray(src, dtype=np.float64).reshape(-1, 3)
        trg = np.asarray(trg, dtype=np.float64).reshape(-1, 3)
        val = np.asarray(val, dtype=np.float64).reshape(-1, self.k0)
        out = np.zeros((trg.shape[0], self.k1))
        if src.shape[0] == 0 or trg.shape[0] == 0:
            return out
        for a in range(0, trg.shape[0], chunk):
            r = trg[a:a + chunk, None, :] - src[None, :, :]            # (nt, ns, 3)
            r2 = np.einsum("ijk,ijk->ij", r, r)
            with np.errstate(divide="ignore"):
                rinv = np.where(r2 > 0, 1.0 / np.sqrt(np.where(r2 > 0, r2, 1.0)), 0.0)
            rinv3 = rinv ** 3
            if self.name == "laplace_dbl":
                # kernel.txx:1299-1311: u += (r . f[0:3]) f[3] / r^3, scale 1/(4 pi)
                rdn = np.einsum("ijk,jk->ij", r, val[:, 0:3])
                out[a:a + chunk, 0] = (rdn * rinv3) @ val[:, 3] / (4 * math.pi)
            elif self.name == "stokes_sym_dip":
                # kernel.txx:1437-1456: f = v[0:3], n = v[3:6],
                # n_dot_f = v0 v3 + v1 v1 + v2 v2 (as the reference computes it),
                # u_k += r_k (n_dot_f - 3 (r.n)(r.f) / r^2) / r^3, scale -1/(8 pi)
                rdf = np.einsum("ijk,jk->ij", r, val[:, 0:3])
                rdn = np.einsum("ijk,jk->ij", r, val[:, 3:6])
                ndf = val[:, 0] * val[:, 3] + val[:, 1] * val[:, 1] + val[:, 2] * val[:, 2]
                common = (ndf[None, :] - 3.0 * rdn * rdf * rinv * rinv) * rinv3
                out[a:a + chunk] = np.einsum("ijk,ij->ik", r, common) * (-1.0 / (8 * math.pi))
            else:
                raise ValueError(self.name)
        return out


LAPLACE = KernelFn("laplace", 1, 1, 9)
LAPLACE_GRAD = KernelFn("laplace_grad", 1, 3, 16)
LAPLACE_PG = KernelFn("laplace_potgrad", 1, 4, 18)
STOKES = KernelFn("stokes_vel", 3, 3, 29)
STOKES_PRESS = KernelFn("stokes_press", 3, 1, 16, deg=2.0)
STOKES_GRAD = KernelFn("stokes_grad", 3, 9, 94, deg=2.0)
BIOT_SAVART = KernelFn("biot_savart", 3, 3, 24, deg=2.0)
LAPLACE_DBL = DblKernelFn("laplace_dbl", 4, 1, 17)
STOKES_DBL = DblKernelFn("stokes_sym_dip", 6, 3, 35)


@dataclass(frozen=True)
class Kernel:
    """pvfmm::Kernel<T> with its sub-kernels (include/kernel.hpp:27-136).

    ``src_scal``/``trg_scal`` are the scale exponents detected by
    Kernel::Initialize (include/kernel.txx:64-196): K(x/2) = 2^(s_i+t_j) K(x).
    ``dbl`` holds the double-layer kernels of the source->check sub-kernels
    (s2m, s2l) and of the source->target one (s2t); None where the reference's
    sub-kernel has none (its EvalListPts asserts one is there,
    fmm_pts.txx:4362).
    """
    name: str
    k0: int
    k1: int
    s2t: KernelFn          # also m2t, l2t
    exp: KernelFn          # s2m, s2l, m2m, m2l, l2l
    src_scal: tuple
    trg_scal: tuple
    dbl: tuple = (None, None)


KERNELS = {
    # LaplaceKernel<T>::potential(), include/kernel.txx:1333-1338
    LAPLACE_POTENTIAL: Kernel("laplace", 1, 1, LAPLACE, LAPLACE, (0.0,), (1.0,), (LAPLACE_DBL, LAPLACE_DBL)),
    # LaplaceKernel<T>::gradient(), include/kernel.txx:1339-1344
    # (its s2m/s2l sub-kernels are the potential kernel, with a double layer;
    # its s2t kernel has none)
    LAPLACE_GRADIENT: Kernel("laplace_grad", 1, 3, LAPLACE_GRAD, LAPLACE, (0.0,), (2.0, 2.0, 2.0), (LAPLACE_DBL, None)),
    # StokesKernel<T>::velocity(), include/kernel.txx:1475-1479
    STOKES_VELOCITY: Kernel("stokes_vel", 3, 3, STOKES, STOKES, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0),
                            (STOKES_DBL, STOKES_DBL)),
    # extension: potential + gradient in one pass (expansions use the potential)
    LAPLACE_POTGRAD: Kernel("laplace_potgrad", 1, 4, LAPLACE_PG, LAPLACE, (0.0,), (1.0, 2.0, 2.0, 2.0)),
    # StokesKernel<T>::pressure() / vel_grad(), BiotSavartKernel<T>::potential()
    # (include/kernel.txx:1480-1491, 1508-1511): no separate expansion kernels,
    # so the kernel itself is expanded (kernel.txx:894-901)
    STOKES_PRESSURE: Kernel("stokes_press", 3, 1, STOKES_PRESS, STOKES_PRESS, (0.0,) * 3, (2.0,)),
    STOKES_VELOCITY_GRAD: Kernel("stokes_grad", 3, 9, STOKES_GRAD, STOKES_GRAD, (0.0,) * 3, (2.0,) * 9),
    BIOT_SAVART_POTENTIAL: Kernel("biot_savart", 3, 3, BIOT_SAVART, BIOT_SAVART, (0.0,) * 3, (2.0,) * 3),
}


# ----------------------------------------------------------------------------
# Morton ids (include/mortonid.txx)
# ----------------------------------------------------------------------------
def morton_coords(c: np.ndarray) -> np.ndarray:
    """MortonId(coord): x = floor(c * 2^30) per axis (mortonid.txx:39-53)."""
    c = np.asarray(c)
    scaled = np.floor(c * c.dtype.type(TWO30))
    return scaled.astype(np.int64).astype(np.uint64)


def interleave_key(X, Y, Z, depth) -> tuple[np.ndarray, np.ndarray]:
    """Sort key equal to the reference's MortonId order (mortonid.txx:107-118):
    the most significant differing coordinate bit decides, z before y before x
    at the same bit; equal coordinates order by depth.  Returned as
    (hi: bits 29..9 interleaved, 63 bits) and (lo: bits 8..0 interleaved << 5 | depth)."""
    X = np.asarray(X, dtype=np.uint64)
    Y = np.asarray(Y, dtype=np.uint64)
    Z = np.asarray(Z, dtype=np.uint64)
    hi = np.zeros(X.shape, dtype=np.uint64)
    lo = np.zeros(X.shape, dtype=np.uint64)
    one = np.uint64(1)
    for b in range(29, 8, -1):
        bb = np.uint64(b)
        hi = (hi << np.uint64(3)) | (((Z >> bb) & one) << np.uint64(2)) | (((Y >> bb) & one) << one) | ((X >> bb) & one)
    for b in range(8, -1, -1):
        bb = np.uint64(b)
        lo = (lo << np.uint64(3)) | (((Z >> bb) & one) << np.uint64(2)) | (((Y >> bb) & one) << one) | ((X >> bb) & one)
    lo = (lo << np.uint64(5)) | np.asarray(depth, dtype=np.uint64)
    return hi, lo


def key_int(X: int, Y: int, Z: int, depth: int) -> int:
    hi, lo = interleave_key(np.array([X]), np.array([Y]), np.array([Z]), np.array([depth]))
    return (int(hi[0]) << 32) | int(lo[0])


def nbr_list(X: int, Y: int, Z: int, depth: int) -> list:
    """MortonId::NbrList at the node's own depth, non-periodic
    (src/mortonid.cpp:15-55): the 3^3 same-depth cells around (X,Y,Z) that lie
    in the unit box, in the order x fastest, then y, then z."""
    w = TWO30 >> depth
    out = []
    for i in range(27):
        x, y, z = X + (i % 3 - 1) * w, Y + ((i // 3) % 3 - 1) * w, Z + (i // 9 - 1) * w
        if 0 <= x < TWO30 and 0 <= y < TWO30 and 0 <= z < TWO30:
            out.append((x, y, z, depth))
    return out


def node_end_key(X: int, Y: int, Z: int, depth: int) -> int:
    """A key larger than every point key inside node (X,Y,Z,depth) and smaller
    than every key after the node's subtree in Morton order."""
    w = TWO30 >> depth
    return key_int(X + w - 1, Y + w - 1, Z + w - 1, 31)


# ----------------------------------------------------------------------------
# Bounding box rescale (src/pvfmm-wrapper.cpp:458-541)
# ----------------------------------------------------------------------------
def bounding_box_map(src_pos: np.ndarray, trg_pos: np.ndarray, real=np.float64):
    """Returns (scale_x, shift_x[3]) mapping both point sets into [0,1)^3."""
    real = np.dtype(real).type
    eps = real(np.finfo(real).eps) * real(64)

    def one_box(x):
        x = np.asarray(x, dtype=real).reshape(-1, 3)
        mn = x.min(axis=0).astype(np.float64)
        mx = x.max(axis=0).astype(np.float64)
        s = real(1) / real(mx[0] - mn[0] + 2 * eps)
        for k in range(3):
            s = min(s, real(1.0 / (mx[k] - mn[k] + 2 * eps)))
        if not np.isfinite(s * 0.0):
            s = real(1)
        sh = np.array([real(-mn[k] * s + eps) for k in range(3)], dtype=real)
        return real(s), sh

    s0, x0 = one_box(src_pos)
    s1, x1 = one_box(trg_pos)
    c0 = [real((real(0.5) - x0[k]) / s0) for k in range(3)]
    c1 = [real((real(0.5) - x1[k]) / s1) for k in range(3)]
    sc = real(0)
    for k in range(3):
        sc = max(sc, real(abs(c0[k] - c1[k])))
    sc = real(1) / (sc + real(1) / s0 + real(1) / s1)
    shift = np.array([real(0.5) - (c0[k] + c1[k]) * sc / real(2) for k in range(3)], dtype=real)
    return sc, shift


def map_points(pos: np.ndarray, scale, shift, real=np.float64) -> np.ndarray:
    """x*scale+shift, then wrapped into [0,1) (pvfmm-wrapper.cpp:582-586)."""
    real = np.dtype(real).type
    c = np.asarray(pos, dtype=real).reshape(-1, 3) * real(scale) + np.asarray(shift, dtype=real)
    c = c.astype(real)
    while True:
        neg = c < 0
        if not neg.any():
            break
        c[neg] += real(1)
    while True:
        big = c >= 1
        if not big.any():
            break
        c[big] -= real(1)
    return c


# ----------------------------------------------------------------------------
# Tree (refine + 2:1 balance + colleagues + lists)
# ----------------------------------------------------------------------------
@dataclass
class Node:
    X: int
    Y: int
    Z: int
    depth: int
    leaf: bool = True
    parent: int = -1
    child0: int = -1        # index of child 0; children are child0..child0+7
    path: int = 0           # Path2Node: octant index within parent
    src: tuple = (0, 0)     # [lo, hi) into the sorted sources
    trg: tuple = (0, 0)     # [lo, hi) into the sorted targets
    colleagues: list = field(default_factory=lambda: [-1] * 27)

    @property
    def n_src(self):
        return self.src[1] - self.src[0]

    @property
    def n_trg(self):
        return self.trg[1] - self.trg[0]


def seed_grid_coords(max_pts: int, real=np.float64) -> np.ndarray:
    """The context's initial tree points (pvfmm-wrapper.cpp:416-432), np = 1."""
    real = np.dtype(real).type
    NN = int(math.ceil(math.pow(float(real(max_pts)), 1.0 / 3.0)))
    i = np.arange(NN ** 3)
    c = np.stack([(real((i // 1) % NN) + real(0.5)) / real(NN),
                  (real((i // NN) % NN) + real(0.5)) / real(NN),
                  (real((i // (NN * NN)) % NN) + real(0.5)) / real(NN)], axis=1)
    return c.astype(real)


def sorted_keys(coords: np.ndarray):
    """Morton-sort points (SortScatterIndex, parUtils.txx:527); equal keys keep
    input order.  Returns (perm, list of python-int keys in sorted order)."""
    M = morton_coords(coords)
    hi, lo = interleave_key(M[:, 0], M[:, 1], M[:, 2], np.full(len(M), MAX_DEPTH))
    perm = np.lexsort((lo, hi))
    keys = [(int(h) << 32) | int(l) for h, l in zip(hi[perm], lo[perm])]
    return perm, keys


class Tree:
    """Single-rank particle octree with PVFMM's refinement and balance."""

    def __init__(self, src_keys, trg_keys, grid_keys, max_pts, max_depth=MAX_DEPTH,
                 src_counted=True, src_weight=None):
        """``src_weight``: how many point sets the source positions stand for
        (the single-layer src_coord and the double-layer surf_coord each count
        in SubdivCond and pt_cnt[0], fmm_node.txx:81-92, fmm_pts.txx:1332-1333);
        0 when the call passes neither density."""
        self.max_pts = max_pts
        self.max_depth = max_depth
        self.src_keys = src_keys
        self.trg_keys = trg_keys
        self.grid_keys = grid_keys
        self.src_weight = (1 if src_counted else 0) if src_weight is None else int(src_weight)
        self.src_counted = self.src_weight > 0
        refined = self._refine()
        self.internal = self._balance(refined)
        self._build_nodes()

    # --- point counts -----------------------------------------------------
    @staticmethod
    def _range(keys, X, Y, Z, d):
        lo = bisect.bisect_left(keys, key_int(X, Y, Z, d))
        hi = bisect.bisect_left(keys, node_end_key(X, Y, Z, d))
        return lo, hi

    def _subdiv(self, X, Y, Z, d) -> bool:
        """FMM_Node::SubdivCond (fmm_node.txx:63-98) for a leaf."""
        if d >= self.max_depth - 1:
            return False
        g = self._range(self.grid_keys, X, Y, Z, d)
        if g[1] - g[0] > self.max_pts:              # MPI_Node::SubdivCond on pt_coord
            return True
        s = self._range(self.src_keys, X, Y, Z, d) if self.src_counted else (0, 0)
        t = self._range(self.trg_keys, X, Y, Z, d)
        return self.src_weight * (s[1] - s[0]) + (t[1] - t[0]) > self.max_pts

    def _refine(self):
        """RefineTree (mpi_tree.txx:403-492): the coarsest tree in which no
        leaf satisfies SubdivCond.  Returns {depth: set of internal (X,Y,Z)}."""
        internal = {}
        level = [(0, 0, 0)]
        d = 0
        while level:
            nxt = []
            for (X, Y, Z) in level:
                if self._subdiv(X, Y, Z, d):
                    internal.setdefault(d, set()).add((X, Y, Z))
                    w = TWO30 >> (d + 1)
                    for c in range(8):
                        nxt.append((X + w * (c & 1), Y + w * ((c >> 1) & 1), Z + w * ((c >> 2) & 1)))
            level = nxt
            d += 1
        return internal

    @staticmethod
    def _balance(internal):
        """balanceOctree (mpi_tree.txx:745-943), non-periodic: the closure of
        the internal-node set under X(level l) -> parent(NbrList(X, l))."""
        if not internal:
            return {}
        S = {d: set(v) for d, v in internal.items()}
        dmax = max(S)
        for l in range(dmax, 0, -1):
            pmask = ~((TWO30 >> (l - 1)) - 1)
            tgt = S.setdefault(l - 1, set())
            for (X, Y, Z) in S.get(l, ()):
                for (x, y, z, _) in nbr_list(X, Y, Z, l):
                    tgt.add((x & pmask, y & pmask, z & pmask))
        return S

    def _build_nodes(self):
        nodes: list[Node] = [Node(0, 0, 0, 0)]
        level_start = [0]
        lookup = [{(0, 0, 0): 0}]
        d = 0
        cur = [0]
        while True:
            S = self.internal.get(d, set())
            nxt = []
            for i in cur:
                n = nodes[i]
                if (n.X, n.Y, n.Z) in S:
                    n.leaf = False
            # children of internal nodes, in Morton order of the parents
            parents = [i for i in cur if not nodes[i].leaf]
            if not parents:
                break
            level_start.append(len(nodes))
            lk = {}
            w = TWO30 >> (d + 1)
            for p in parents:
                P = nodes[p]
                P.child0 = len(nodes)
                for c in range(8):
                    ch = Node(P.X + w * (c & 1), P.Y + w * ((c >> 1) & 1), P.Z + w * ((c >> 2) & 1), d + 1,
                              parent=p, path=c)
                    lk[(ch.X, ch.Y, ch.Z)] = len(nodes)
                    nxt.append(len(nodes))
                    nodes.append(ch)
            lookup.append(lk)
            cur = nxt
            d += 1
        self.nodes = nodes
        self.level_start = level_start + [len(nodes)]
        self.lookup = lookup
        for n in nodes:
            n.src = self._range(self.src_keys, n.X, n.Y, n.Z, n.depth) if self.src_counted else (0, 0)
            n.trg = self._range(self.trg_keys, n.X, n.Y, n.Z, n.depth)
        # SetColleagues (mpi_tree.txx:1136-1256): same-level neighbours, index
        # ((z+1)*3+(y+1))*3+(x+1); free space: no wrap.
        for n in nodes:
            w = TWO30 >> n.depth
            lk = lookup[n.depth]
            for ci in range(27):
                dx, dy, dz = ci % 3 - 1, (ci // 3) % 3 - 1, ci // 9 - 1
                x, y, z = n.X + dx * w, n.Y + dy * w, n.Z + dz * w
                n.colleagues[ci] = lk.get((x, y, z), -1) if (0 <= x < TWO30 and 0 <= y < TWO30 and 0 <= z < TWO30) else -1

    def leaf_keys(self) -> list:
        """Leaf Morton ids (x, y, z, depth) in Morton order (preorder)."""
        leaves = [n for n in self.nodes if n.leaf]
        leaves.sort(key=lambda n: key_int(n.X, n.Y, n.Z, n.depth))
        return [(n.X, n.Y, n.Z, n.depth) for n in leaves]

    @property
    def depth(self) -> int:
        return max(n.depth for n in self.nodes)


# ----------------------------------------------------------------------------
# Interaction lists (interac_list.txx:98-279, fmm_tree.txx:301-352)
# ----------------------------------------------------------------------------
def raw_lists(tree: Tree) -> dict:
    """The reference's interaction lists before any reassignment
    (InteracList::BuildList, interac_list.txx:98-279), built for every node
    with targets in its subtree (FMM_Tree::BuildInteracLists,
    fmm_tree.txx:301-352): ``{list name: {owner node: [member nodes]}}`` with
    lists U0 (adjacent coarser leaves, leaf owners), U1 (leaf colleagues incl.
    self, leaf owners), U2 (adjacent children of non-leaf colleagues, leaf
    owners), W (non-adjacent children of non-leaf colleagues, leaf owners),
    X (non-adjacent coarser leaves: leaf colleagues of the parent) and V1
    (non-leaf colleagues except self, non-leaf owners).  Members are kept
    whether or not they hold sources."""
    N = tree.nodes
    out = {k: {} for k in ("U0", "U1", "U2", "W", "X", "V1")}
    for ti, T in enumerate(N):
        if T.n_trg == 0:
            continue
        L = {k: [] for k in out}
        if T.leaf:
            for ci in range(27):
                c = T.colleagues[ci]
                if c < 0:
                    continue
                if N[c].leaf:
                    L["U1"].append(c)
                    continue
                C = N[c]
                for j in range(8):
                    rel = [(ci % 3) * 4 - 4 + (2 if j & 1 else 0) - 1,
                           ((ci // 3) % 3) * 4 - 4 + (2 if j & 2 else 0) - 1,
                           (ci // 9) * 4 - 4 + (2 if j & 4 else 0) - 1]
                    L["U2" if max(abs(r) for r in rel) <= 3 else "W"].append(C.child0 + j)
        if T.parent >= 0:
            par, p2n = N[T.parent], T.path
            for ci in range(27):
                c = par.colleagues[ci]
                if c >= 0 and N[c].leaf:
                    rel = [(ci % 3) * 4 - 4 - (2 if p2n & 1 else 0) + 1,
                           ((ci // 3) % 3) * 4 - 4 - (2 if p2n & 2 else 0) + 1,
                           (ci // 9) * 4 - 4 - (2 if p2n & 4 else 0) + 1]
                    if max(abs(r) for r in rel) <= 3:
                        if T.leaf:
                            L["U0"].append(c)
                    else:
                        L["X"].append(c)
        if not T.leaf:
            for ci in range(27):
                c = T.colleagues[ci]
                if ci != 13 and c >= 0 and not N[c].leaf:
                    L["V1"].append(c)
        for k, v in L.items():
            if v:
                out[k][ti] = v
    return out


def build_lists(tree: Tree, nsrf: int):
    """Per-target-node lists after the Nsrf reassignment:

    ``p2p[t]``   source leaves evaluated point-to-point into leaf t (U0, U1, U2,
                 plus X when t has <= Nsrf targets, plus W leaves with <= Nsrf
                 sources; fmm_pts.txx:5262-5345)
    ``x[t]``     source leaves -> downward check surface of t (fmm_pts.txx:4629)
    ``w[t]``     source nodes (upward equivalent surface) -> targets of leaf t
                 (fmm_pts.txx:4929)
    ``v1[t]``    (source parent, colleague index) pairs for non-leaf t (V1 list)
    Built from the reference's raw lists (raw_lists); only sources with points
    are kept.
    """
    N = tree.nodes
    raw = raw_lists(tree)
    p2p, xl, wl, v1 = {}, {}, {}, {}
    for ti, T in enumerate(N):
        if T.n_trg == 0:
            continue
        U = raw["U1"].get(ti, []) + raw["U2"].get(ti, []) + raw["U0"].get(ti, [])
        P = [s for s in U if N[s].n_src > 0]
        Xk, Wk = [], []
        for s in raw["X"].get(ti, []):
            if N[s].n_src == 0:
                continue
            if T.leaf and T.n_trg <= nsrf:
                P.append(s)
            else:
                Xk.append(s)
        for s in raw["W"].get(ti, []):
            S = N[s]
            if S.n_src == 0:
                continue
            if S.leaf and S.n_src * tree.src_weight <= nsrf:     # pt_cnt[0] counts both layers
                P.append(s)
            else:
                Wk.append(s)
        if T.leaf:
            p2p[ti] = P
            wl[ti] = Wk
        xl[ti] = Xk
        V = [(c, T.colleagues.index(c)) for c in raw["V1"].get(ti, []) if N[c].n_src > 0]
        if V:
            v1[ti] = V
    return p2p, xl, wl, v1


# ----------------------------------------------------------------------------
# Surfaces and operators (fmm_pts.txx:54-160, 453-764)
# ----------------------------------------------------------------------------
def surface(p: int, c, alpha: float, depth: int) -> np.ndarray:
    """surface() (fmm_pts.txx:54-97): n = 6(p-1)^2+2 points on a cube."""
    n = 6 * (p - 1) * (p - 1) + 2
    co = np.zeros((n, 3))
    co[0] = [-1.0, -1.0, -1.0]
    cnt = 1
    for i in range(p - 1):
        for j in range(p - 1):
            co[cnt] = [-1, (2 * (i + 1) - p + 1) / (p - 1), (2 * j - p + 1) / (p - 1)]
            cnt += 1
    for i in range(p - 1):
        for j in range(p - 1):
            co[cnt] = [(2 * i - p + 1) / (p - 1), -1, (2 * (j + 1) - p + 1) / (p - 1)]
            cnt += 1
    for i in range(p - 1):
        for j in range(p - 1):
            co[cnt] = [(2 * (i + 1) - p + 1) / (p - 1), (2 * j - p + 1) / (p - 1), -1]
            cnt += 1
    flat = co.reshape(-1)
    flat[cnt * 3:cnt * 3 + (n // 2) * 3] = -flat[:(n // 2) * 3]
    co = flat.reshape(n, 3)
    r = 0.5 * 0.5 ** depth
    b = alpha * r
    return (co + 1.0) * b + np.asarray(c, dtype=np.float64)


def _shifted(c, depth, rad):
    r = 0.5 * 0.5 ** depth
    return np.asarray(c, dtype=np.float64) - r * (rad - 1.0)


def u_check_surf(m, c, depth):
    return surface(m, _shifted(c, depth, RAD1), RAD1, depth)


def u_equiv_surf(m, c, depth):
    return surface(m, _shifted(c, depth, RAD0), RAD0, depth)


def d_check_surf(m, c, depth):
    return surface(m, _shifted(c, depth, RAD0), RAD0, depth)


def d_equiv_surf(m, c, depth):
    return surface(m, _shifted(c, depth, RAD1), RAD1, depth)


def pinv_factors(M: np.ndarray):
    """C2E0 = V^T S^+ and C2E1 = U^T with the cutoff S > 4 eps max(S)
    (fmm_pts.txx:478-537).  check_row @ C2E0 @ C2E1 = equiv_row."""
    U, s, Vh = np.linalg.svd(M, full_matrices=M.shape[0] == M.shape[1])  # thin SVD when not square
    eps = np.finfo(np.float64).eps
    cut = eps * s.max() * 4
    sinv = np.where(s > cut, 1.0 / np.where(s > cut, s, 1.0), 0.0)
    return Vh.T * sinv[None, :], U.T


class Operators:
    """Level-0 translation operators of one kernel and order
    (FMM_Pts::Initialize + Precomp, fmm_pts.txx:223-331, 453-764)."""

    def __init__(self, kernel: Kernel, m: int):
        self.kernel = kernel
        self.m = m
        self.ns = 6 * (m - 1) ** 2 + 2
        ke = kernel.exp
        z = np.zeros(3)
        # UC2UE0/1 (fmm_pts.txx:478-537)
        M_up = ke.matrix(u_equiv_surf(m, z, 0), u_check_surf(m, z, 0))
        self.uc2ue0, self.uc2ue1 = pinv_factors(M_up)
        # DC2DE0/1 (fmm_pts.txx:538-581)
        M_dn = ke.matrix(d_equiv_surf(m, z, 0), d_check_surf(m, z, 0))
        self.dc2de0, self.dc2de1 = pinv_factors(M_dn)
        # U2U per child octant c, parent at level 0 (fmm_pts.txx:582-606)
        self.u2u = []
        for c in range(8):
            cc = np.array([c & 1, (c >> 1) & 1, (c >> 2) & 1]) * 0.5
            Mce2c = ke.matrix(u_equiv_surf(m, cc, 1), u_check_surf(m, z, 0))
            self.u2u.append((Mce2c @ self.uc2ue0) @ self.uc2ue1)
        # D2D per child octant c, parent at level 0 (fmm_pts.txx:607-643)
        self.d2d = []
        for c in range(8):
            cc = np.array([c & 1, (c >> 1) & 1, (c >> 2) & 1]) * 0.5
            Mpe2c = ke.matrix(d_equiv_surf(m, z, 0), d_check_surf(m, cc, 1))
            self.d2d.append(self.dc2de0 @ (self.dc2de1 @ Mpe2c))
        # V operators: kernel on the conv grid, r2c FFT (fmm_pts.txx:671-718)
        n1 = 2 * m
        self.n1 = n1
        self.vhat = {}
        for k in range(-3, 4):
            for j in range(-3, 4):
                for i in range(-3, 4):
                    if max(abs(i), abs(j), abs(k)) <= 1:
                        continue
                    self.vhat[(i, j, k)] = self._v_operator(np.array([i, j, k], dtype=np.float64))
        # FFT maps (fmm_pts.txx:2703-2712, 2790-2797)
        s = surface(m, z, m - 1, 0)
        self.fft_map = np.array([(int(m - 1 - s[i, 0] + 0.5), int(m - 1 - s[i, 1] + 0.5), int(m - 1 - s[i, 2] + 0.5))
                                 for i in range(self.ns)])
        self.ifft_map = np.array([(int(m * 2 - 0.5 - s[i, 0]), int(m * 2 - 0.5 - s[i, 1]), int(m * 2 - 0.5 - s[i, 2]))
                                  for i in range(self.ns)])

    @classmethod
    def from_arrays(cls, kernel: Kernel, m: int, arrays: dict) -> "Operators":
        """Operators given as arrays in the layout of the CUDA library's
        precompute (``PVFMMPrecompOperator``), with din = ns*kin equivalent and
        dout = ns*kout check values and r = min(din, dout): uc2ue0/dc2de0
        (dout x r), uc2ue1/dc2de1 (r x din), u2u (8*din x din, child-major
        rows), d2d (dout x 8*dout, child-major columns) and vop (complex
        [f][26][8][8][kin][kout], divided by n3).  Lets the oracle run on
        exactly the operators the library builds."""
        self = cls.__new__(cls)
        self.kernel, self.m = kernel, m
        self.ns = 6 * (m - 1) ** 2 + 2
        kin, kout = kernel.exp.k0, kernel.exp.k1
        din, dout = self.ns * kin, self.ns * kout
        r = min(din, dout)
        self.uc2ue0 = arrays["uc2ue0"].reshape(dout, r)
        self.uc2ue1 = arrays["uc2ue1"].reshape(r, din)
        self.dc2de0 = arrays["dc2de0"].reshape(dout, r)
        self.dc2de1 = arrays["dc2de1"].reshape(r, din)
        self.u2u = list(arrays["u2u"].reshape(8, din, din))
        d2d = arrays["d2d"].reshape(dout, 8, dout)
        self.d2d = [np.ascontiguousarray(d2d[:, c, :]) for c in range(8)]
        n1 = 2 * m
        self.n1 = n1
        n3 = n1 ** 3
        vop = arrays["vop"].reshape(-1, 2)
        vop = (vop[:, 0] + 1j * vop[:, 1]).reshape(n1, n1, n1 // 2 + 1, 26, 8, 8, kin, kout)
        self.vhat = {}
        for ci in range(27):
            if ci == 13:
                continue
            o = ci if ci < 13 else ci - 1
            po = np.array([ci % 3 - 1, (ci // 3) % 3 - 1, ci // 9 - 1])
            for j1 in range(8):
                b1 = np.array([j1 & 1, (j1 >> 1) & 1, (j1 >> 2) & 1])
                for j2 in range(8):
                    b2 = np.array([j2 & 1, (j2 >> 1) & 1, (j2 >> 2) & 1])
                    rel = tuple(int(v) for v in (2 * po - b1 + b2))
                    if max(abs(r) for r in rel) <= 1 or rel in self.vhat:
                        continue
                    self.vhat[rel] = vop[:, :, :, o, j1, j2] * n3
        z = np.zeros(3)
        s = surface(m, z, m - 1, 0)
        self.fft_map = np.array([(int(m - 1 - s[i, 0] + 0.5), int(m - 1 - s[i, 1] + 0.5), int(m - 1 - s[i, 2] + 0.5))
                                 for i in range(self.ns)])
        self.ifft_map = np.array([(int(m * 2 - 0.5 - s[i, 0]), int(m * 2 - 0.5 - s[i, 1]), int(m * 2 - 0.5 - s[i, 2]))
                                  for i in range(self.ns)])
        return self

    def _v_operator(self, rel):
        m, n1, ke = self.m, self.n1, self.kernel.exp
        a = RAD0
        g = np.arange(n1)
        # grid[(i + n1 j + n2 k)] = ((i-m) a/(m-1) + d) ... (conv_grid, fmm_pts.txx:140-158)
        K_, J_, I_ = np.meshgrid(g, g, g, indexing="ij")
        coords = np.stack([(I_ - m) * a / (m - 1) + rel[0], (J_ - m) * a / (m - 1) + rel[1],
                           (K_ - m) * a / (m - 1) + rel[2]], axis=-1).reshape(-1, 3)
        P = ke.matrix(coords, np.zeros((1, 3)))          # (n3*k0, k1)
        P = P.reshape(n1, n1, n1, ke.k0, ke.k1)           # [z][y][x][i][k]
        return np.fft.rfftn(P, axes=(0, 1, 2))           # [z][y][xh][i][k]


# ----------------------------------------------------------------------------
# FMM evaluation
# ----------------------------------------------------------------------------
class FMM:
    """PtFMM-style evaluation on sorted points (fmm_tree.txx:237-738)."""

    def __init__(self, kernel_id: int, m: int, max_pts: int, ops: Operators | None = None):
        self.kernel = KERNELS[kernel_id]
        self.kernel_id = kernel_id
        self.m = m
        self.max_pts = max_pts
        self.ops = ops if ops is not None else Operators(self.kernel, m)
        self.ns = self.ops.ns

    # ------------------------------------------------------------------
    def setup(self, src_c: np.ndarray, trg_c: np.ndarray, real=np.float64, src_counted=True,
              pt_coord="seed", src_weight=None):
        """Tree for unit-box coordinates (pvfmm-wrapper.cpp:543-775).  The
        tree's point set is the context's seed grid (pt_coord="seed",
        pvfmm-wrapper.cpp:416-432) or the targets (pt_coord="trg", the C++
        interface, pvfmm.txx:238)."""
        self.src_perm, src_keys = sorted_keys(src_c)
        self.trg_perm, trg_keys = sorted_keys(trg_c)
        if pt_coord == "seed":
            _, grid_keys = sorted_keys(seed_grid_coords(self.max_pts, real))
        else:
            grid_keys = trg_keys
        self.tree = Tree(src_keys, trg_keys, grid_keys, self.max_pts, src_counted=src_counted,
                         src_weight=src_weight)
        self.src = np.asarray(src_c, dtype=np.float64)[self.src_perm]
        self.trg = np.asarray(trg_c, dtype=np.float64)[self.trg_perm]
        self.lists = build_lists(self.tree, self.ns)

    def _corner(self, n: Node):
        return np.array([n.X, n.Y, n.Z], dtype=np.float64) / TWO30

    def evaluate(self, den_sorted: np.ndarray | None, surf_sorted: np.ndarray | None = None) -> np.ndarray:
        """RunFMM (fmm_tree.txx:237-264) on sorted single-layer densities
        and/or sorted double-layer values (k0 + 3 per point); returns the
        sorted target values (n_trg, k1).  The double layer enters where the
        sources' points do: S2U, X-list and U-list (EvalListPts calls the
        sub-kernel's dbl_layer_poten on surf_value, fmm_pts.txx:4346-4366)."""
        K = self.kernel
        ke, kt = K.exp, K.s2t
        kd_exp, kd_s2t = K.dbl
        if surf_sorted is not None and (kd_exp is None or kd_s2t is None):
            raise ValueError(f"kernel {K.name} has no double-layer kernel")
        ops, m, ns = self.ops, self.m, self.ns
        tree = self.tree
        N = tree.nodes
        k0, k1e = ke.k0, ke.k1
        # Expansion kernels have src_scal = 0 and trg_scal = deg on every
        # component, so a check->equivalent operator at level l is 2^(-deg l)
        # times the level-0 one (fmm_pts.txx:2447-2465).
        e_exp = ke.deg - EXP_SRC_SCAL
        den = None if den_sorted is None else np.asarray(den_sorted, dtype=np.float64).reshape(-1, K.k0)
        surf = None if surf_sorted is None else np.asarray(surf_sorted, dtype=np.float64).reshape(-1, K.k0 + 3)
        nn = len(N)

        def from_points(kfn, kdbl, lo, hi, T, pts):
            """Potentials at `pts` (relative to T's corner) of the source points
            [lo, hi): single layer plus double layer."""
            r = np.zeros((len(pts), kfn.k1))
            if den is not None:
                r += kfn.eval(self.src[lo:hi] - self._corner(T), den[lo:hi], pts)
            if surf is not None:
                r += kdbl.eval(self.src[lo:hi] - self._corner(T), surf[lo:hi], pts)
            return r

        ue = np.zeros((nn, ns * k0))
        dc = np.zeros((nn, ns * k1e))
        out = np.zeros((len(self.trg), K.k1))

        # All kernel evaluations use coordinates relative to the corner of the
        # node being evaluated, as the reference does through coord_shift and
        # surfaces built at c = 0 (fmm_pts.txx:2489-2496, 4645-4650, 4947-4952,
        # 5262-5340); corner differences are exact dyadic numbers.
        def rel(n, T):
            return np.array([n.X - T.X, n.Y - T.Y, n.Z - T.Z], dtype=np.float64) / TWO30

        def pts_rel(arr, lo, hi, T):
            return arr[lo:hi] - self._corner(T)

        # wall time per stage (ms), named as the library's stage times
        stage = self.stage_ms = {k: 0.0 for k in ("S2U", "U2U", "X-List", "V-List", "D2D", "D2T+W+U")}
        clock = [time.perf_counter()]

        def tick(name):
            now = time.perf_counter()
            stage[name] += 1000 * (now - clock[0])
            clock[0] = now

        # --- S2U (fmm_pts.txx:2275-2637 + EvalListPts 4390-4426) ---------
        # The two pseudo-inverse factors are applied one after the other, as
        # the reference does: multiplying them out first loses the accuracy.
        z3 = np.zeros(3)
        for i, n in enumerate(N):
            if n.leaf and n.n_src > 0:
                chk = from_points(ke, kd_exp, n.src[0], n.src[1], n, u_check_surf(m, z3, n.depth))
                ue[i] = ((chk.reshape(-1) * 2.0 ** (-e_exp * n.depth)) @ ops.uc2ue0) @ ops.uc2ue1
        tick("S2U")
        # --- U2U bottom-up (fmm_pts.txx:2602-2630, EvalList) ------------
        for d in range(tree.depth - 1, -1, -1):
            for i in range(tree.level_start[d], tree.level_start[d + 1]):
                n = N[i]
                if n.leaf or n.n_src == 0:
                    continue
                acc = np.zeros(ns * k0)
                for c in range(8):
                    acc += ue[n.child0 + c] @ ops.u2u[c]
                ue[i] = acc
        tick("U2U")
        p2p, xl, wl, v1 = self.lists
        # --- X-list (fmm_pts.txx:4444-4736) ------------------------------
        for t, srcs in xl.items():
            T = N[t]
            pts = d_check_surf(m, z3, T.depth)
            for s in srcs:
                S = N[s]
                dc[t] += from_points(ke, kd_exp, S.src[0], S.src[1], T, pts).reshape(-1)
        tick("X-List")
        # --- W-list (fmm_pts.txx:4746-5022) ------------------------------
        for t, srcs in wl.items():
            T = N[t]
            tp = pts_rel(self.trg, T.trg[0], T.trg[1], T)
            for s in srcs:
                S = N[s]
                out[T.trg[0]:T.trg[1]] += kt.eval(u_equiv_surf(m, rel(S, T), S.depth), ue[s], tp)
        # --- U-list (fmm_pts.txx:5032-5418) ------------------------------
        for t, srcs in p2p.items():
            T = N[t]
            if not srcs:
                continue
            idx = np.concatenate([np.arange(N[s].src[0], N[s].src[1]) for s in srcs])
            tp = pts_rel(self.trg, T.trg[0], T.trg[1], T)
            if den is not None:
                out[T.trg[0]:T.trg[1]] += kt.eval(self.src[idx] - self._corner(T), den[idx], tp)
            if surf is not None:
                out[T.trg[0]:T.trg[1]] += kd_s2t.eval(self.src[idx] - self._corner(T), surf[idx], tp)
        tick("D2T+W+U")
        # --- V-list via FFT (fmm_pts.txx:3597-3759, 2689-2858) ----------
        self._vlist(ue, dc, v1)
        tick("V-List")
        # --- D2D top-down (fmm_pts.txx:3762-3790) ------------------------
        for d in range(0, tree.depth):
            for i in range(tree.level_start[d], tree.level_start[d + 1]):
                n = N[i]
                if n.leaf or n.n_trg == 0:
                    continue
                for c in range(8):
                    dc[n.child0 + c] += dc[i] @ ops.d2d[c]
        tick("D2D")
        # --- D2T (fmm_pts.txx:5427-5737) ---------------------------------
        for i, n in enumerate(N):
            if n.leaf and n.n_trg > 0:
                de = ((dc[i] * 2.0 ** (-e_exp * n.depth)) @ ops.dc2de0) @ ops.dc2de1
                out[n.trg[0]:n.trg[1]] += kt.eval(d_equiv_surf(m, z3, n.depth), de,
                                                  pts_rel(self.trg, n.trg[0], n.trg[1], n))
        tick("D2T+W+U")
        self.ue, self.dc = ue, dc
        return out

    def _vlist(self, ue, dc, v1):
        ops, m = self.ops, self.m
        ke = self.kernel.exp
        k0, k1 = ke.k0, ke.k1
        N = self.tree.nodes
        n1 = 2 * m
        fm, im = ops.fft_map, ops.ifft_map
        spec = {}

        def spectrum(q):
            if q in spec:
                return spec[q]
            Q = N[q]
            g = np.zeros((8, k0, n1, n1, n1))
            for c in range(8):
                u = ue[Q.child0 + c].reshape(-1, k0) * 2.0 ** (EXP_SRC_SCAL * (Q.depth + 1))
                for i in range(k0):
                    g[c, i, fm[:, 2], fm[:, 1], fm[:, 0]] = u[:, i]
            spec[q] = np.fft.rfftn(g, axes=(2, 3, 4))
            return spec[q]

        for p, lst in v1.items():
            P = N[p]
            acc = np.zeros((8, k1, n1, n1, n1 // 2 + 1), dtype=np.complex128)
            for (q, ci) in lst:
                S = spectrum(q)
                po = np.array([ci % 3 - 1, (ci // 3) % 3 - 1, ci // 9 - 1])
                for j1 in range(8):
                    b1 = np.array([j1 & 1, (j1 >> 1) & 1, (j1 >> 2) & 1])
                    for j2 in range(8):
                        b2 = np.array([j2 & 1, (j2 >> 1) & 1, (j2 >> 2) & 1])
                        rel = tuple(int(v) for v in (2 * po - b1 + b2))
                        if max(abs(r) for r in rel) <= 1:
                            continue
                        V = ops.vhat[rel]            # [z][y][xh][i][k]
                        acc[j1] += np.einsum("zyxik,izyx->kzyx", V, S[j2])
            res = np.fft.irfftn(acc, s=(n1, n1, n1), axes=(2, 3, 4))
            lvl = P.depth + 1
            for c in range(8):
                vals = res[c][:, im[:, 2], im[:, 1], im[:, 0]].T          # (ns, k1)
                dc[P.child0 + c] += vals.reshape(-1) * 2.0 ** (ke.deg * lvl)


# ----------------------------------------------------------------------------
# C-ABI style entry (PVFMMEval, pvfmm-wrapper.cpp:445-811)
# ----------------------------------------------------------------------------
def surf_scal(K: Kernel, scale: float, real=np.float64) -> np.ndarray:
    """Scaling of the double-layer values (pvfmm-wrapper.cpp:521-535): the
    first k0 values by scale * scale^src_scal, the last three by 1 (in the
    interface's precision `real`)."""
    real = np.dtype(real).type
    return np.array([real(scale) * real(scale) ** real(e) for e in K.src_scal] + [1.0, 1.0, 1.0], dtype=real)


def pvfmm_eval(kernel_id: int, m: int, max_pts: int, src_pos, sl_den, trg_pos, ops=None, return_fmm=False,
               dl_den=None, real=np.float64):
    """PVFMMEvalD(src, sl_den, dl_den, n_src, trg, trg_val, n_trg, ctx,
    setup=1).  Either density may be None (NULL); dl_den holds k0 + 3 values
    per source (pvfmm.h:269-272).  real=np.float32 follows PVFMMEvalF up to
    the FMM itself: the bounding box, the mapped coordinates, the seed grid
    and the density and output scales in FP32 (pvfmm-wrapper.cpp:458-599);
    the FMM runs in FP64 on those values."""
    K = KERNELS[kernel_id]
    src_pos = np.asarray(src_pos, dtype=np.float64).reshape(-1, 3)
    trg_pos = np.asarray(trg_pos, dtype=np.float64).reshape(-1, 3)
    if sl_den is not None:
        sl_den = np.asarray(sl_den, dtype=np.float64).reshape(-1, K.k0)
    if dl_den is not None:
        dl_den = np.asarray(dl_den, dtype=np.float64).reshape(-1, K.k0 + 3)
    rt = np.dtype(real).type
    scale, shift = bounding_box_map(src_pos, trg_pos, real)
    src_c = map_points(src_pos, scale, shift, real).astype(np.float64)
    trg_c = map_points(trg_pos, scale, shift, real).astype(np.float64)
    src_scal = np.array([rt(scale) ** rt(e) for e in K.src_scal], dtype=rt).astype(np.float64)
    trg_scal = np.array([rt(scale) ** rt(e) for e in K.trg_scal], dtype=rt).astype(np.float64)
    fmm = FMM(kernel_id, m, max_pts, ops)
    t0 = time.perf_counter()
    fmm.setup(src_c, trg_c, real=real, src_weight=(sl_den is not None) + (dl_den is not None))
    setup_ms = 1000 * (time.perf_counter() - t0)
    fmm.io_scal = (src_scal, trg_scal, surf_scal(K, scale, real).astype(np.float64))
    fmm.io_real = rt
    out = _eval_scaled(fmm, sl_den, dl_den)
    fmm.stage_ms["setup"] = setup_ms
    if return_fmm:
        return out, fmm
    return out


def _eval_scaled(fmm: "FMM", sl_den, dl_den) -> np.ndarray:
    src_scal, trg_scal, sf_scal = fmm.io_scal
    K = fmm.kernel
    if sl_den is None and dl_den is None:           # no source points at all
        fmm.stage_ms = {}
        return np.zeros((len(fmm.trg), K.k1))
    rt = getattr(fmm, "io_real", np.float64)   # densities scaled in the interface's precision
    den = None if sl_den is None else \
        (np.asarray(sl_den, dtype=rt).reshape(-1, K.k0) * src_scal.astype(rt)[None, :]).astype(np.float64)[fmm.src_perm]
    surf = None if dl_den is None else \
        (np.asarray(dl_den, dtype=rt).reshape(-1, K.k0 + 3) * sf_scal.astype(rt)[None, :]).astype(np.float64)[fmm.src_perm]
    out_sorted = fmm.evaluate(den, surf)
    out = np.empty_like(out_sorted)
    out[fmm.trg_perm] = out_sorted
    return out * trg_scal[None, :]


def pvfmm_eval_setup0(fmm: "FMM", sl_den, dl_den=None) -> np.ndarray:
    """PVFMMEvalD with setup=0 (src/pvfmm-wrapper.cpp:637-654): the tree of a
    previous pvfmm_eval(..., return_fmm=True) on the same points, new
    densities (the same ones NULL as before)."""
    return _eval_scaled(fmm, sl_den, dl_den)


def ptfmm_eval(kernel_id: int, m: int, max_pts: int, src_pos, sl_den, trg_pos, ops=None, dl_pos=None, dl_den=None):
    """C++ interface: PtFMM_CreateTree + SetupFMM + PtFMM_Evaluate
    (pvfmm.txx:216-328).  Coordinates in [0,1)^3 are used as given (no
    bounding-box map, so no kernel-exponent scaling) and the tree's point set
    is the targets.  The double layer has its own point set (surf_coord,
    dl_pos with k0 + 3 values per point, unscaled); both sets count in the
    leaf-size rule and pt_cnt[0] (fmm_node.txx:81-92, fmm_pts.txx:1332-1333),
    so they are evaluated as one source set, each point carrying its own
    layer's values and zeros for the other (zero values add exact zeros)."""
    K = KERNELS[kernel_id]
    src_c = np.asarray(src_pos, dtype=np.float64).reshape(-1, 3)
    trg_c = np.asarray(trg_pos, dtype=np.float64).reshape(-1, 3)
    sl_den = np.asarray(sl_den, dtype=np.float64).reshape(-1, K.k0)
    surf = None
    if dl_pos is not None:
        dl_c = np.asarray(dl_pos, dtype=np.float64).reshape(-1, 3)
        dl_v = np.asarray(dl_den, dtype=np.float64).reshape(-1, K.k0 + 3)
        surf = np.concatenate([np.zeros((len(src_c), K.k0 + 3)), dl_v])
        sl_den = np.concatenate([sl_den, np.zeros((len(dl_c), K.k0))])
        src_c = np.concatenate([src_c, dl_c])
    if src_c.min() < 0 or trg_c.min() < 0 or src_c.max() >= 1 or trg_c.max() >= 1:
        raise ValueError("coordinates must lie in [0,1)^3")
    fmm = FMM(kernel_id, m, max_pts, ops)
    fmm.setup(src_c, trg_c, pt_coord="trg")
    out_sorted = fmm.evaluate(sl_den[fmm.src_perm], None if surf is None else surf[fmm.src_perm])
    out = np.empty_like(out_sorted)
    out[fmm.trg_perm] = out_sorted
    return out


def direct_sum(kernel_id: int, src_pos, sl_den, trg_pos, chunk=2048) -> np.ndarray:
    """FP64 direct sum over all sources (the reference's CheckFMMOutput check,
    examples/include/utils.txx:7-109)."""
    K = KERNELS[kernel_id]
    src = np.asarray(src_pos, dtype=np.float64).reshape(-1, 3)
    trg = np.asarray(trg_pos, dtype=np.float64).reshape(-1, 3)
    den = np.asarray(sl_den, dtype=np.float64).reshape(-1)
    out = np.zeros((len(trg), K.k1))
    for a in range(0, len(trg), chunk):
        out[a:a + chunk] = K.s2t.eval(src, den, trg[a:a + chunk])
    return out


def direct_sum_mapped(kernel_id: int, src_pos, sl_den, trg_pos, dl_den=None, chunk=512) -> np.ndarray:
    """FP64 direct sum of what PVFMMEvalD approximates: both layers evaluated
    in the reference's unit-box frame, on the densities scaled as it scales
    them, and the result scaled back (pvfmm-wrapper.cpp:458-541, 800-808).
    For single-layer densities this equals direct_sum; for double-layer
    values it is the quantity the reference's FMM converges to."""
    K = KERNELS[kernel_id]
    src = np.asarray(src_pos, dtype=np.float64).reshape(-1, 3)
    trg = np.asarray(trg_pos, dtype=np.float64).reshape(-1, 3)
    scale, shift = bounding_box_map(src, trg)
    src_c, trg_c = map_points(src, scale, shift), map_points(trg, scale, shift)
    src_scal = np.array([scale ** e for e in K.src_scal])
    trg_scal = np.array([scale ** e for e in K.trg_scal])
    out = np.zeros((len(trg), K.k1))
    for a in range(0, len(trg), chunk):
        if sl_den is not None:
            den = np.asarray(sl_den, dtype=np.float64).reshape(-1, K.k0) * src_scal[None, :]
            out[a:a + chunk] += K.s2t.eval(src_c, den, trg_c[a:a + chunk])
        if dl_den is not None:
            surf = np.asarray(dl_den, dtype=np.float64).reshape(-1, K.k0 + 3) * surf_scal(K, scale)[None, :]
            out[a:a + chunk] += K.dbl[1].eval(src_c, surf, trg_c[a:a + chunk])
    return out * trg_scal[None, :]


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).reshape(-1)
    b = np.asarray(b, dtype=np.float64).reshape(-1)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
