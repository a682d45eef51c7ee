"""ctypes access to the reference PVFMM built from its own sources
(``oracle/ref_fmm/build.sh`` -> ``oracle/_ref/libpvfmm_ref_<isa>.so``).

Test infrastructure: the golden-fixture generator, the tests that pin the
oracle and the CPU-baseline arm of bench.py use it.  It calls the reference's
C interface (``PVFMMCreateContextDWorld`` / ``PVFMMEvalD`` /
``PVFMMDestroyContextD``, src/pvfmm-wrapper.cpp:877-928) and the driver's
read-only tree and list dumps (``ref_driver.cpp``).
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(os.path.dirname(HERE), "_ref")

# reference Mat_Type values of the interaction lists (include/precomp_mat.hpp:21-38)
U0, U1, U2, W, X, V1 = 8, 9, 10, 12, 13, 14

_lib = None


def _isa() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
    except OSError:
        return "avx2"
    return "avx512" if " avx512f" in flags and " avx512dq" in flags and " avx512vl" in flags else "avx2"


def library_path(isa: str | None = None, lattice: bool = False) -> str:
    """The reference library for an instruction set; lattice=True: the build
    without PVFMM_EXTENDED_BC (periodic lattice sum; AVX2 code only)."""
    if lattice:
        return os.path.join(REF_DIR, "libpvfmm_ref_avx2_lattice.so")
    return os.path.join(REF_DIR, f"libpvfmm_ref_{isa or _isa()}.so")


def available(lattice: bool = False) -> bool:
    return os.path.exists(library_path(lattice=lattice))


_libs = {}


def load(lattice: bool = False):
    """Loads the reference library for this host's instruction set (or the
    lattice-sum build).  The reference reads and writes its precompute files
    in $PVFMM_DIR (or the working directory); a private temporary directory is
    used when unset.  The two builds write precompute files of the same name
    with different periodic operators, so the lattice build gets a directory
    of its own."""
    global _lib
    if lattice in _libs:
        return _libs[lattice]
    path = library_path(lattice=lattice)
    if not os.path.exists(path):
        raise RuntimeError(f"reference library not built: {path} (run oracle/ref_fmm/build.sh)")
    if not os.environ.get("PVFMM_DIR"):
        os.environ["PVFMM_DIR"] = tempfile.mkdtemp(prefix="pvfmm_ref_precomp_")
    if lattice:
        # the library reads PVFMM_DIR when a context is created; contexts of
        # the lattice build are created under a directory of their own
        _lattice_dir[0] = tempfile.mkdtemp(prefix="pvfmm_ref_precomp_lattice_")
    lib = ctypes.CDLL(path)
    vp, lg = ctypes.c_void_p, ctypes.c_long
    lib.PVFMMCreateContextDWorld.restype = vp
    lib.PVFMMCreateContextDWorld.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.PVFMMEvalD.restype = None
    lib.PVFMMEvalD.argtypes = [vp, vp, vp, lg, vp, vp, lg, vp, ctypes.c_int]
    lib.PVFMMDestroyContextD.restype = None
    lib.PVFMMDestroyContextD.argtypes = [ctypes.POINTER(vp)]
    lib.ref_tree_nodes.restype = lg
    lib.ref_tree_nodes.argtypes = [vp, vp, lg]
    lib.ref_tree_lists.restype = lg
    lib.ref_tree_lists.argtypes = [vp, vp, lg]
    lib.ref_set_threads.restype = ctypes.c_int
    lib.ref_set_threads.argtypes = [ctypes.c_int]
    lib.ref_profile_enable.restype = None
    lib.ref_profile_enable.argtypes = [ctypes.c_int]
    lib.ref_profile_report.restype = lg
    lib.ref_profile_report.argtypes = [vp, lg]
    lib.ref_ptfmm_eval.restype = ctypes.c_int
    lib.ref_ptfmm_eval.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, lg, vp, vp, lg, vp, vp, lg, vp, vp]
    lib.ref_ptfmm_eval_bc.restype = ctypes.c_int
    lib.ref_ptfmm_eval_bc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, lg, vp, vp, lg, vp,
                                      vp, lg, vp, vp]
    lib.ref_cheb_integ0.restype = ctypes.c_int
    lib.ref_cheb_integ0.argtypes = [ctypes.c_int, vp, ctypes.c_double, vp]
    _libs[lattice] = lib
    if not lattice:
        _lib = lib
    return lib


_lattice_dir = [None]


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


# PVFMMKernel ids of the reference (include/pvfmm.h:21-28) -> (k0, k1)
KDIM = {0: (1, 1), 1: (1, 3), 2: (3, 1), 3: (3, 3), 4: (3, 9), 5: (3, 3)}


class RefContext:
    """A reference PVFMM context: free space (box_size <= 0) or periodic with
    period box_size (the 5x5x5-image boundary operator of the default build,
    or with lattice=True the lattice-sum build), `max_pts` points per leaf,
    multipole order m, kernel id of the C interface."""

    def __init__(self, kernel: int, m: int, max_pts: int, threads: int = 0, box_size: float = -1.0,
                 lattice: bool = False):
        self.lib = load(lattice)
        if threads:
            self.lib.ref_set_threads(threads)
        self.kernel = kernel
        self.k0, self.k1 = KDIM[kernel]
        saved = os.environ.get("PVFMM_DIR")
        if lattice:
            os.environ["PVFMM_DIR"] = _lattice_dir[0]
        try:
            self.ctx = self.lib.PVFMMCreateContextDWorld(box_size, max_pts, m, kernel)
        finally:
            if lattice and saved is not None:
                os.environ["PVFMM_DIR"] = saved
        if not self.ctx:
            raise RuntimeError("reference context creation failed")

    def evaluate(self, src, den, trg, setup=True, dl=None) -> np.ndarray:
        """PVFMMEvalD(src, den, dl, ...): `den` (n, k0) single-layer
        densities or None, `dl` (n, k0+3) double-layer values or None."""
        src = np.ascontiguousarray(src, dtype=np.float64).reshape(-1)
        den = None if den is None else np.ascontiguousarray(den, dtype=np.float64).reshape(-1)
        dl = None if dl is None else np.ascontiguousarray(dl, dtype=np.float64).reshape(-1)
        same = trg is None
        trg = src if same else np.ascontiguousarray(trg, dtype=np.float64).reshape(-1)
        n_src, n_trg = len(src) // 3, len(trg) // 3
        out = np.zeros(n_trg * self.k1)
        self.lib.PVFMMEvalD(_p(src), None if den is None else _p(den), None if dl is None else _p(dl), n_src,
                            _p(trg), _p(out), n_trg, ctypes.c_void_p(self.ctx), 1 if setup else 0)
        return out.reshape(n_trg, self.k1)

    def tree(self):
        """Nodes of the last tree: int64 array (n, 10) with X, Y, Z (units of
        2^-30), depth, leaf, #sources and #targets held, pt_cnt[0], pt_cnt[1]."""
        n = self.lib.ref_tree_nodes(ctypes.c_void_p(self.ctx), None, 0)
        a = np.zeros((n, 10), dtype=np.int64)
        self.lib.ref_tree_nodes(ctypes.c_void_p(self.ctx), _p(a), n)
        return a

    def lists(self):
        """Interaction-list entries of the last tree: int64 array (n, 6) with
        owner node index, list type (U0 8, U1 9, U2 10, W 12, X 13, V1 14),
        slot, member node index."""
        n = self.lib.ref_tree_lists(ctypes.c_void_p(self.ctx), None, 0)
        a = np.zeros((n, 6), dtype=np.int64)
        self.lib.ref_tree_lists(ctypes.c_void_p(self.ctx), _p(a), n)
        return a

    def close(self):
        if self.ctx:
            c = ctypes.c_void_p(self.ctx)
            self.lib.PVFMMDestroyContextD(ctypes.byref(c))
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def profile_enable(on=True):
    """Turns the reference's profiler (pvfmm::Profile) on (with a cleared
    log) or off (keeping the log)."""
    load().ref_profile_enable(1 if on else 0)


def profile_report() -> list:
    """The reference profiler's log since profile_enable: a list of
    (indent, tag, t_avg seconds) in the profiler's print order
    (pvfmm::Profile::print, src/profile.cpp:128-230); the tag names are those
    of fmm_tree.txx / fmm_pts.txx (S2U, U2U, U-List, V-List, D2T, ...)."""
    lib = load()
    n = lib.ref_profile_report(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib.ref_profile_report(buf, n + 1)
    rows = []
    for line in buf.value.decode(errors="replace").splitlines():
        toks = line.split()
        if len(toks) < 13:
            continue
        try:
            nums = [float(v) for v in toks[-12:]]
        except ValueError:
            continue
        name = " ".join(toks[:-12]).replace("|", " ").replace("+-", " ").strip()
        indent = len(line) - len(line.lstrip(" |+-"))
        rows.append((indent, name, nums[1]))
    return rows


def ref_eval(kernel, m, max_pts, src, den, trg=None, threads=0, dl=None, box_size=-1.0, lattice=False):
    ctx = RefContext(kernel, m, max_pts, threads, box_size=box_size, lattice=lattice)
    try:
        out = ctx.evaluate(src, den, trg, dl=dl)
        return out, ctx.tree(), ctx.lists()
    finally:
        ctx.close()


def ref_ptfmm_eval(kernel, m, max_pts, sl_coord, sl_den, dl_coord, dl_den, trg, threads=0, periodic=False,
                   lattice=False, bndry=None):
    """The reference's C++ interface (PtFMM_CreateTree with separate single-
    and double-layer point sets, SetupFMM, PtFMM_Evaluate; coordinates in
    [0,1)^3 as given; BoundaryType Periodic when periodic, or the BoundaryType
    value bndry (0 FreeSpace, 1 PX, 2 PXY, 3 PXYZ); from the lattice build
    when lattice).  Either point set may be empty (shape (0, 3))."""
    lib = load(lattice)
    if threads:
        lib.ref_set_threads(threads)
    k0, k1 = KDIM[kernel]
    sc = np.ascontiguousarray(sl_coord, dtype=np.float64).reshape(-1)
    sv = np.ascontiguousarray(sl_den, dtype=np.float64).reshape(-1)
    dc = np.ascontiguousarray(dl_coord, dtype=np.float64).reshape(-1)
    dv = np.ascontiguousarray(dl_den, dtype=np.float64).reshape(-1)
    tc = np.ascontiguousarray(trg, dtype=np.float64).reshape(-1)
    n_trg = len(tc) // 3
    out = np.zeros(n_trg * k1)
    saved = os.environ.get("PVFMM_DIR")
    if lattice:
        os.environ["PVFMM_DIR"] = _lattice_dir[0]
    try:
        bt = bndry if bndry is not None else (3 if periodic else 0)
        rc = lib.ref_ptfmm_eval_bc(kernel, m, max_pts, bt, len(sc) // 3, _p(sc), _p(sv),
                                   len(dc) // 3, _p(dc), _p(dv), n_trg, _p(tc), _p(out))
    finally:
        if lattice and saved is not None:
            os.environ["PVFMM_DIR"] = saved
    if rc != 0:
        raise ValueError(f"kernel {kernel} is not driven through the C++ interface here")
    return out.reshape(n_trg, k1)
