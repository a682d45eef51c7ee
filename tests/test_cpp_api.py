"""The C++ interface (include/pvfmm.hpp) against the oracle.

tests/cpp/ptfmm_example.cpp is written like the reference's C++ examples
(examples/src/example1.cpp: PtFMM::Initialize, PtFMM_CreateTree, SetupFMM,
PtFMM_Evaluate, ClearFMMData, a second evaluation with new densities) and
dumps its inputs and outputs.  The CPU test checks that the header compiles
and links against the library; the GPU tests run the program and compare with
the oracle's C++-interface path (ptfmm_eval: coordinates used as given, tree
points = targets), ker_poten with a direct sum and BuildMatrix with the
oracle's kernel matrix.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import pvfmm_b200 as P
from oracle import pvfmm_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "ptfmm_example.cpp")


def _compile(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "ptfmm_example")
    lib_dir = os.path.dirname(str(P.LIB_PATH))
    cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", lib_dir, "-lpvfmm_b200", "-Wl,-rpath," + lib_dir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_header_compiles_and_links(tmp_path):
    _compile(tmp_path)


def _read(path):
    a = np.fromfile(path, dtype=np.float64)
    k0, k1 = int(a[0]), int(a[1])
    pos = 2
    parts = []
    for _ in range(11):
        n = int(a[pos])
        parts.append(a[pos + 1: pos + 1 + n])
        pos += 1 + n
    assert pos == len(a)
    return k0, k1, parts


_OPS = {}


def _ops(kid, m):
    if (kid, m) not in _OPS:
        _OPS[(kid, m)] = O.Operators.from_arrays(O.KERNELS[kid], m, P.precomp_operators(P.FMMKernel(kid), m, 0))
    return _OPS[(kid, m)]


@pytest.mark.gpu
@pytest.mark.parametrize("kid,m,mp,ns,nt,real,tol", [
    (0, 6, 100, 3000, 2500, "d", 1e-12),
    (6, 6, 64, 2000, 2000, "d", 1e-12),
    (1, 4, 80, 1500, 1800, "d", 1e-12),
    (3, 4, 100, 1500, 1500, "d", 1e-11),
    (0, 6, 100, 3000, 2500, "f", 5e-5),
])
def test_cpp_interface_matches_oracle(tmp_path, kid, m, mp, ns, nt, real, tol):
    exe = _compile(tmp_path)
    out = str(tmp_path / "out.bin")
    r = subprocess.run([exe, out, str(kid), str(m), str(mp), str(ns), str(nt), "7", real],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    k0, k1, (src, den, den2, trg, val1, val2, kp, mat, _, _, _) = _read(out)
    K = O.KERNELS[kid]
    assert (k0, k1) == (K.k0, K.k1)
    src = src.reshape(-1, 3)
    trg = trg.reshape(-1, 3)
    ops = _ops(kid, m)
    ref1 = O.ptfmm_eval(kid, m, mp, src, den, trg, ops=ops)
    ref2 = O.ptfmm_eval(kid, m, mp, src, den2, trg, ops=ops)
    assert O.rel_l2(val1, ref1) < tol
    assert O.rel_l2(val2, ref2) < tol
    # the FMM itself is accurate (guards against a wrong tree rule on both sides)
    assert O.rel_l2(ref1, O.direct_sum(kid, src, den, trg)) < (5e-3 if m == 4 else 1e-4)
    # ker_poten accumulated twice; BuildMatrix layout
    ds, dt = min(ns, 200), min(nt, 64)
    direct = K.s2t.eval(src[:ds], den.reshape(-1, K.k0)[:ds].reshape(-1), trg[:dt])
    kp_tol = 1e-12 if real == "d" else 1e-5
    assert O.rel_l2(kp, 2 * direct) < kp_tol
    M = K.s2t.matrix(src[:3], trg[:dt])
    assert O.rel_l2(mat, M.reshape(-1)) < kp_tol


@pytest.mark.gpu
def test_unit_box_rejects_points_outside_unit_cube():
    """Unit-box mode (the C++ interface's tree rule) refuses coordinates
    outside [0,1)^3 instead of mapping them."""
    ctx = P.FMMParticleContext(-1, 50, 4, P.FMMKernel.LaplacePotential)
    ctx.set_unit_box(True)
    x = np.random.default_rng(3).random((200, 3))
    ctx.evaluate(x.reshape(-1), np.ones(200), None, x.reshape(-1), True)
    x[5, 1] = 1.25
    with pytest.raises(RuntimeError, match=r"\[0,1\)"):
        ctx.evaluate(x.reshape(-1), np.ones(200), None, x.reshape(-1), True)


@pytest.mark.gpu
def test_host_kernel_eval_matches_direct_sum():
    rng = np.random.default_rng(5)
    for kid in (0, 1, 3, 6):
        K = O.KERNELS[kid]
        s = rng.random((700, 3))
        t = rng.random((300, 3))
        q = rng.uniform(-1, 1, 700 * K.k0)
        out = np.full(300 * K.k1, 0.5)
        P.kernel_eval(P.FMMKernel(kid), s, q, t, out)
        assert O.rel_l2(out - 0.5, O.direct_sum(kid, s, q, t)) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("kid,m,tol", [(0, 6, 1e-12), (3, 4, 1e-11)])
def test_cpp_interface_double_layer_points_match_oracle(tmp_path, kid, m, tol):
    """PtFMM_CreateTree with a separate double-layer point set (surf_coord,
    surf_value) and PtFMM_Evaluate with new values for both layers, against the
    oracle's C++-interface path (both point sets count in the tree; the
    oracle is pinned to the reference's own C++ interface in
    tests/test_reference_pins.py)."""
    exe = _compile(tmp_path)
    out = str(tmp_path / "out.bin")
    r = subprocess.run([exe, out, str(kid), str(m), "60", "1500", "1200", "11", "d", "900"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    k0, k1, (src, den, den2, trg, val1, val2, _, _, dl, dd, dd2) = _read(out)
    src, trg, dl = src.reshape(-1, 3), trg.reshape(-1, 3), dl.reshape(-1, 3)
    ops = _ops(kid, m)
    ref1 = O.ptfmm_eval(kid, m, 60, src, den, trg, ops=ops, dl_pos=dl, dl_den=dd)
    ref2 = O.ptfmm_eval(kid, m, 60, src, den2, trg, ops=ops, dl_pos=dl, dl_den=dd2)
    assert O.rel_l2(val1, ref1) < tol
    assert O.rel_l2(val2, ref2) < tol


@pytest.mark.gpu
@pytest.mark.parametrize("bc,axes", [("periodic", 7), ("px", 1), ("pxy", 3)])
def test_cpp_interface_periodic_tree(tmp_path, bc, axes):
    """PtFMM_CreateTree(..., pvfmm::Periodic / PX / PXY) in the header: a
    periodic context of period 1 in unit-box mode with those periodic axes
    (pinned to the reference's C++ interface in tests/test_gpu_periodic.py)."""
    exe = _compile(tmp_path)
    out = str(tmp_path / "out.bin")
    r = subprocess.run([exe, out, "0", "6", "60", "2500", "1500", "13", "d", "0", bc],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    _, _, (src, den, den2, trg, val1, val2, _, _, _, _, _) = _read(out)
    ctx = P.FMMParticleContext(1.0, 60, 6, P.FMMKernel.LaplacePotential)
    ctx.set_unit_box(True)
    if axes != 7:
        ctx.set_periodic_axes(axes)
    ref1 = ctx.evaluate(src, den, None, trg, True)
    ref2 = ctx.evaluate(src, den2, None, trg, False)
    assert O.rel_l2(val1, ref1) < 1e-14
    assert O.rel_l2(val2, ref2) < 1e-14
    free = P.FMMParticleContext(-1.0, 60, 6, P.FMMKernel.LaplacePotential)
    free.set_unit_box(True)
    assert O.rel_l2(val1, free.evaluate(src, den, None, trg, True)) > 1e-3   # the images matter
    ctx.close()
    free.close()
