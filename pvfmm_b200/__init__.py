"""pvfmm_b200 -- B200 particle FMM with the PVFMM interface.

Python surface mirroring the reference bindings (python/src/pvfmm/wrapper.py,
ffi.py): ``FMMKernel``, ``FMMParticleContext(box_size, max_points,
multipole_order, kernel, comm, dtype)`` and ``.evaluate(src_pos, sl_den,
dl_den, trg_pos, setup)``.  Everything runs in libpvfmm_b200.so (CUDA,
sm_100a); there is no CPU fallback: without the library, or without a GPU,
constructing a context raises.

Differences from the reference bindings: ``comm`` is optional (mpi4py is not
needed; one rank per GPU), output arrays have n_trg*k1 entries for every
kernel, and ``precision`` selects the plain FP64 or the mixed form.
"""
from __future__ import annotations

import ctypes
import os
from enum import Enum
from pathlib import Path
from typing import Optional

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libpvfmm_b200.so"


class FMMKernel(Enum):
    """Mirrors PVFMMKernel in pvfmm.h (reference include/pvfmm.h:21-28)."""
    LaplacePotential = 0
    LaplaceGradient = 1
    StokesPressure = 2
    StokesVelocity = 3
    StokesVelocityGrad = 4
    BiotSavartPotential = 5
    LaplacePotGrad = 6          # extension: potential and -grad, 4 outputs


# (k0, k1) per kernel, from the BuildKernel calls in include/kernel.txx.
KERNEL_DIMS = {
    FMMKernel.LaplacePotential: (1, 1),
    FMMKernel.LaplaceGradient: (1, 3),
    FMMKernel.StokesPressure: (3, 1),
    FMMKernel.StokesVelocity: (3, 3),
    FMMKernel.StokesVelocityGrad: (3, 9),
    FMMKernel.BiotSavartPotential: (3, 3),
    FMMKernel.LaplacePotGrad: (1, 4),
}
SUPPORTED = set(FMMKernel)  # every PVFMMKernel value plus the pot+grad extension

PRECISION_PLAIN = 0
PRECISION_MIXED = 1

_lib = None


def load_library(path: Optional[os.PathLike] = None) -> ctypes.CDLL:
    """Loads libpvfmm_b200.so (built by ``python -m pvfmm_b200.build``)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m pvfmm_b200.build`")
    lib = ctypes.CDLL(str(p))
    vp, cl, ci, cd, cf = ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_double, ctypes.c_float
    sig = {
        "PVFMMCreateContextD": (vp, [cd, ci, ci, ci, ci]),
        "PVFMMCreateContextF": (vp, [cf, ci, ci, ci, ci]),
        "PVFMMCreateContextDWorld": (vp, [cd, ci, ci, ci]),
        "PVFMMCreateContextFWorld": (vp, [cf, ci, ci, ci]),
        "PVFMMCreateContextExD": (vp, [cd, ci, ci, ci, ci]),
        "PVFMMEvalD": (None, [vp, vp, vp, cl, vp, vp, cl, vp, ci]),
        "PVFMMEvalF": (None, [vp, vp, vp, cl, vp, vp, cl, vp, ci]),
        "PVFMMEvalDeviceD": (ci, [vp, vp, vp, cl, vp, vp, cl, ci, vp]),
        "PVFMMEvalDeviceF": (ci, [vp, vp, vp, cl, vp, vp, cl, ci, vp]),
        "PVFMMEvalLayersDeviceD": (ci, [vp, vp, vp, vp, cl, vp, vp, cl, ci, vp]),
        "PVFMMEvalLayersDeviceF": (ci, [vp, vp, vp, vp, cl, vp, vp, cl, ci, vp]),
        "PVFMMEvalAdjointDeviceD": (ci, [vp, vp, cl, vp, vp, cl, vp, ci, vp]),
        "PVFMMEvalAdjointDeviceF": (ci, [vp, vp, cl, vp, vp, cl, vp, ci, vp]),
        "PVFMMSetUnitBox": (ci, [vp, ci]),
        "PVFMMSetLayerPoints": (ci, [vp, ci]),
        "PVFMMSetPeriodicBC": (ci, [vp, ci, vp]),
        "PVFMMSetPeriodicAxes": (ci, [vp, ci]),
        "PVFMMKernelEvalD": (ci, [ci, vp, vp, cl, vp, vp, cl]),
        "PVFMMKernelEvalDeviceNoAllocD": (ci, [ci, vp, vp, cl, vp, vp, cl, vp]),
        "PVFMMDestroyContextD": (None, [ctypes.POINTER(vp)]),
        "PVFMMDestroyContextF": (None, [ctypes.POINTER(vp)]),
        "PVFMMGetLastError": (ctypes.c_char_p, []),
        "PVFMMGetStageTimes": (ci, [vp, vp, ci]),
        "PVFMMGetLaunchCount": (cl, [vp]),
        "PVFMMGetTreeData": (cl, [vp, ci, vp, cl]),
        "PVFMMPrecompOperator": (cl, [ci, ci, ci, ci, vp, cl]),
        "PVFMMKernelEvalDeviceD": (ci, [ci, vp, vp, cl, vp, vp, cl, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def last_error() -> str:
    return load_library().PVFMMGetLastError().decode()


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def precomp_operator(kernel: FMMKernel, m: int, precision: int, which: int) -> np.ndarray:
    """Host FP64 operator from the library's precompute (see pvfmm.h)."""
    lib = load_library()
    n = lib.PVFMMPrecompOperator(int(kernel.value), m, precision, which, None, 0)
    if n < 0:
        raise RuntimeError(last_error())
    out = np.empty(n, dtype=np.float64)
    lib.PVFMMPrecompOperator(int(kernel.value), m, precision, which, _ptr(out), n)
    return out


def kernel_eval_device(kernel: FMMKernel, src_ptr: int, den_ptr: int, n_src: int, trg_ptr: int, out_ptr: int,
                       n_trg: int, stream: int = 0) -> None:
    """Direct FP64 kernel sum on device pointers, accumulated into out
    (the GPU form of Kernel<T>::ker_poten)."""
    lib = load_library()
    rc = lib.PVFMMKernelEvalDeviceD(int(kernel.value), ctypes.c_void_p(src_ptr), ctypes.c_void_p(den_ptr), n_src,
                                    ctypes.c_void_p(trg_ptr), ctypes.c_void_p(out_ptr), n_trg,
                                    ctypes.c_void_p(stream) if stream else None)
    if rc != 0:
        raise RuntimeError(f"PVFMMKernelEvalDeviceD failed: {last_error()}")


def kernel_eval(kernel: FMMKernel, src_pos: np.ndarray, den: np.ndarray, trg_pos: np.ndarray,
                out: Optional[np.ndarray] = None) -> np.ndarray:
    """Direct FP64 kernel sum on host arrays (PVFMMKernelEvalD), accumulated
    into ``out`` (zeros when not given); evaluated on the current GPU."""
    k0, k1 = KERNEL_DIMS[kernel]
    src = np.ascontiguousarray(src_pos, dtype=np.float64).reshape(-1)
    trg = np.ascontiguousarray(trg_pos, dtype=np.float64).reshape(-1)
    q = np.ascontiguousarray(den, dtype=np.float64).reshape(-1)
    n_src, n_trg = src.size // 3, trg.size // 3
    if q.size != n_src * k0:
        raise ValueError("density length does not match the source count")
    if out is None:
        out = np.zeros(n_trg * k1)
    elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size != n_trg * k1:
        raise ValueError("out must be a C-contiguous float64 array of n_trg*k1 values")
    rc = load_library().PVFMMKernelEvalD(int(kernel.value), _ptr(src), _ptr(q), n_src, _ptr(trg), _ptr(out), n_trg)
    if rc != 0:
        raise RuntimeError(f"PVFMMKernelEvalD failed: {last_error()}")
    return out


OPERATOR_NAMES = ["uc2ue0", "uc2ue1", "dc2de0", "dc2de1", "u2u", "d2d", "usurf", "vop"]


def precomp_operators(kernel: FMMKernel, m: int, precision: int = PRECISION_PLAIN) -> dict:
    return {name: precomp_operator(kernel, m, precision, i) for i, name in enumerate(OPERATOR_NAMES)}


class FMMParticleContext:
    """Particle FMM context (reference python/src/pvfmm/wrapper.py:90-180).

    ``dtype`` float64 creates a D context (plain FP64 unless ``precision`` is
    given), float32 an F context (mixed form).
    """

    def __init__(self, box_size: float, max_points: int, multipole_order: int, kernel: FMMKernel,
                 comm=None, dtype=np.float64, precision: Optional[int] = None):
        if multipole_order <= 0 or multipole_order % 2 != 0:
            raise ValueError("multipole order must be even and postive")
        if kernel not in SUPPORTED:
            raise NotImplementedError(f"kernel {kernel.name} is not implemented")
        self.kernel = kernel
        self.dtype = np.dtype(dtype)
        self.k0, self.k1 = KERNEL_DIMS[kernel]
        self.multipole_order = multipole_order
        self._lib = load_library()
        if self.dtype == np.float64:
            prec = PRECISION_PLAIN if precision is None else precision
            self._ptr = self._lib.PVFMMCreateContextExD(float(box_size), max_points, multipole_order,
                                                        int(kernel.value), prec)
            self.precision = prec
        elif self.dtype == np.float32:
            if precision not in (None, PRECISION_MIXED):
                raise ValueError("float32 contexts use the mixed form")
            self._ptr = self._lib.PVFMMCreateContextF(float(box_size), max_points, multipole_order,
                                                      int(kernel.value), 0)
            self.precision = PRECISION_MIXED
        else:
            raise ValueError("Invalid dtype, must be either float64 or float32")
        if not self._ptr:
            raise RuntimeError(f"PVFMMCreateContext failed: {last_error()}")

    def close(self):
        if getattr(self, "_ptr", None):
            p = ctypes.c_void_p(self._ptr)
            if self.dtype == np.float64:
                self._lib.PVFMMDestroyContextD(ctypes.byref(p))
            else:
                self._lib.PVFMMDestroyContextF(ctypes.byref(p))
            self._ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, name, a, per_point, n=None):
        if a.dtype != self.dtype:
            raise ValueError(f"{name} had the wrong dtype: {a.dtype}. This object was created with dtype {self.dtype}")
        if not a.flags.c_contiguous:
            raise ValueError(f"{name} must be C-contiguous")
        if a.size % per_point != 0 or (n is not None and a.size != n * per_point):
            raise ValueError(f"{name} has a length that does not match the point count")

    def evaluate(self, src_pos: np.ndarray, sl_den: Optional[np.ndarray], dl_den: Optional[np.ndarray],
                 trg_pos: np.ndarray, setup: bool = True) -> np.ndarray:
        """PVFMMEval on host arrays; returns n_trg*k1 values."""
        self._check("src_pos", src_pos, 3)
        n_src = src_pos.size // 3
        if sl_den is not None:
            self._check("sl_den", sl_den, self.k0, n_src)
        if dl_den is not None:
            # k0 + 3 values per source (the reference's wrapper.py:155 checks
            # for 6, which fits StokesVelocity only)
            self._check("dl_den", dl_den, self.k0 + 3, n_src)
        self._check("trg_pos", trg_pos, 3)
        n_trg = trg_pos.size // 3
        trg_val = np.empty(n_trg * self.k1, dtype=self.dtype)
        f = self._lib.PVFMMEvalD if self.dtype == np.float64 else self._lib.PVFMMEvalF
        same = trg_pos is src_pos
        f(_ptr(src_pos), _ptr(sl_den), _ptr(dl_den), n_src, _ptr(src_pos) if same else _ptr(trg_pos),
          _ptr(trg_val), n_trg, self._ptr, int(setup))
        err = last_error()
        if err:
            raise RuntimeError(f"PVFMMEval failed: {err}")
        return trg_val

    def evaluate_device(self, src_ptr: int, den_ptr: Optional[int], n_src: int, trg_ptr: int, out_ptr: int,
                        n_trg: int, setup: bool = True, stream: int = 0, dl_ptr: Optional[int] = None) -> None:
        """PVFMMEvalDevice* on raw CUDA pointers (e.g. torch ``tensor.data_ptr()``);
        with ``dl_ptr`` (double-layer values) PVFMMEvalLayersDevice*."""
        vp = ctypes.c_void_p
        common = (n_src, vp(trg_ptr), vp(out_ptr), n_trg, int(setup), vp(stream) if stream else None)
        den = vp(den_ptr) if den_ptr else None
        if dl_ptr:
            f = self._lib.PVFMMEvalLayersDeviceD if self.dtype == np.float64 else self._lib.PVFMMEvalLayersDeviceF
            rc = f(self._ptr, vp(src_ptr), den, vp(dl_ptr), *common)
        else:
            f = self._lib.PVFMMEvalDeviceD if self.dtype == np.float64 else self._lib.PVFMMEvalDeviceF
            rc = f(self._ptr, vp(src_ptr), den, *common)
        if rc != 0:
            raise RuntimeError(f"PVFMMEvalDevice failed: {last_error()}")

    def evaluate_adjoint_device(self, src_ptr: int, n_src: int, trg_ptr: int, trg_den_ptr: int, n_trg: int,
                                out_ptr: int, setup: bool = True, stream: int = 0) -> None:
        """PVFMMEvalAdjointDevice*: densities at the targets, values at the
        sources (same kernel).  With src_ptr == trg_ptr the forward tree is
        reused when setup is False."""
        f = self._lib.PVFMMEvalAdjointDeviceD if self.dtype == np.float64 else self._lib.PVFMMEvalAdjointDeviceF
        rc = f(self._ptr, ctypes.c_void_p(src_ptr), n_src, ctypes.c_void_p(trg_ptr), ctypes.c_void_p(trg_den_ptr),
               n_trg, ctypes.c_void_p(out_ptr), int(setup), ctypes.c_void_p(stream) if stream else None)
        if rc != 0:
            raise RuntimeError(f"PVFMMEvalAdjointDevice failed: {last_error()}")

    def set_unit_box(self, on: bool = True) -> None:
        """Tree rule of the reference C++ interface: coordinates used as given
        in [0,1)^3, tree points = targets (PVFMMSetUnitBox)."""
        if self._lib.PVFMMSetUnitBox(self._ptr, int(on)) != 0:
            raise RuntimeError(last_error())

    def set_periodic_bc(self, lattice: bool = False, m2c: Optional[np.ndarray] = None) -> None:
        """Boundary operator of a periodic context (box_size > 0; see
        PVFMMSetPeriodicBC): the 5x5x5-image form of the reference's default
        build plus an optional (ns*k0) x (ns*k1) operator ``m2c`` (FMM_Pts::
        SetM2C), or with ``lattice`` the lattice sum over all images."""
        a = None if m2c is None else np.ascontiguousarray(m2c, dtype=np.float64).reshape(-1)
        if self._lib.PVFMMSetPeriodicBC(self._ptr, int(bool(lattice)), None if a is None else _ptr(a)) != 0:
            raise RuntimeError(last_error())

    def set_periodic_axes(self, axes: int) -> None:
        """Periodic axes of a periodic context (PVFMMSetPeriodicAxes): 1 = x
        (BoundaryType PX), 3 = x and y (PXY), 7 = all (PXYZ, the default)."""
        if self._lib.PVFMMSetPeriodicAxes(self._ptr, int(axes)) != 0:
            raise RuntimeError(last_error())

    def set_layer_points(self, on: bool = True) -> None:
        """Separate single- and double-layer point sets, passed concatenated
        (each point counts once in the tree; PVFMMSetLayerPoints)."""
        if self._lib.PVFMMSetLayerPoints(self._ptr, int(on)) != 0:
            raise RuntimeError(last_error())

    def stage_times(self) -> dict:
        buf = np.zeros(12)
        self._lib.PVFMMGetStageTimes(self._ptr, _ptr(buf), 12)
        names = ["setup", "S2U", "U2U", "V-FFT", "V-Hadamard", "V-IFFT", "X-List", "D2D", "D2T+W+U", "total",
                 "near-field kernel", "D2T GEMMs"]
        return dict(zip(names, buf.tolist()))

    STAT_NAMES = ["n_nodes", "depth", "n_sleaf", "n_tleaf", "n_vsrc", "n_vtrg", "n_xtrg", "p2p_entries",
                  "x_entries", "w_entries", "p2p_pairs", "x_pairs", "w_pairs", "d2t_pairs", "s2u_pairs",
                  "n_leaves", "n_src", "n_trg", "v_pairs"]

    def tree_stats(self) -> dict:
        """Sizes of the tree and lists of the last setup (for roofline bookkeeping)."""
        return dict(zip(self.STAT_NAMES, self.tree_data(11).tolist()))

    def launch_count(self) -> int:
        return int(self._lib.PVFMMGetLaunchCount(self._ptr))

    def tree_data(self, what: int) -> np.ndarray:
        n = self._lib.PVFMMGetTreeData(self._ptr, what, None, 0)
        if n < 0:
            raise RuntimeError(last_error())
        dt = np.float64 if what in (7, 8, 11) else np.int64
        out = np.empty(n, dtype=dt)
        self._lib.PVFMMGetTreeData(self._ptr, what, _ptr(out), n)
        return out
