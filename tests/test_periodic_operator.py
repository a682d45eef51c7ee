"""The periodic boundary operator (BC_Type of BoundaryType Periodic,
reference include/fmm_pts.txx:790-1232) of the host precompute against the
reference's own, read from the precompute files that the reference builds
wrote (tests/golden/reference_bc_*.npz, tests/golden/make_golden.py): the
5x5x5-image form of its default build (PVFMM_EXTENDED_BC) and the lattice sum
of the build without that option.  CPU only.
"""
import os
import sys

import numpy as np
import pytest

import pvfmm_b200 as P

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_golden import PERIODIC_OPERATORS, periodic_operator_probe  # noqa: E402

# the lattice sum passes the SVDs of order m+2 pseudo-inverses through 45
# levels of products: the two builds' SVDs (LAPACK there, one-sided Jacobi
# here) agree to ~1e-11 relative in the operator
TOL = {False: 1e-14, True: 1e-10}


@pytest.mark.parametrize("name", sorted(PERIODIC_OPERATORS))
def test_periodic_operator_matches_reference(name):
    z = np.load(os.path.join(HERE, "golden", f"reference_bc_{name}.npz"))
    kid, m, lattice = int(z["kernel"]), int(z["m"]), bool(z["lattice"])
    M = P.precomp_operator(P.FMMKernel(kid), m, 0, 10 if lattice else 9)
    n = int(round(np.sqrt(M.size)))
    M = M.reshape(n, n)
    V = periodic_operator_probe(kid, m)
    for ours, ref in ((M @ V, z["MV"]), (M.T @ V, z["MtV"])):
        assert np.linalg.norm(ours - ref) / np.linalg.norm(ref) < TOL[lattice]
    assert abs(np.linalg.norm(M) / float(z["norm"]) - 1) < TOL[lattice]


def test_lattice_form_rejects_kernels_without_it():
    with pytest.raises(RuntimeError):
        P.precomp_operator(P.FMMKernel.StokesPressure, 4, 0, 10)
    # the 5x5x5-image form exists for every kernel (rectangular for 3 -> 1)
    M = P.precomp_operator(P.FMMKernel.StokesPressure, 4, 0, 9)
    ns = 6 * 3 * 3 + 2
    assert M.size == ns * 3 * ns


def test_lattice_operator_file(tmp_path):
    """With PVFMM_DIR the lattice operator is written once and read back
    (the same values); a file of the wrong size is an error."""
    import subprocess
    code = ("import numpy as np, pvfmm_b200 as P, time; "
            "t=time.time(); a=P.precomp_operator(P.FMMKernel.LaplacePotential, 4, 0, 10); "
            "print(len(a), a[:3].tolist())")
    env = dict(os.environ, PVFMM_DIR=str(tmp_path))
    root = os.path.dirname(HERE)
    r1 = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True, text=True, timeout=600)
    assert r1.returncode == 0, r1.stderr
    files = [f for f in os.listdir(tmp_path) if f.endswith("_lattice_bc.data")]
    assert files == ["Precomp_laplace_m4_lattice_bc.data"]
    r2 = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True, text=True, timeout=600)
    assert r2.returncode == 0 and r2.stdout == r1.stdout
    with open(tmp_path / files[0], "r+b") as f:
        f.truncate(100)
    r3 = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True, text=True, timeout=600)
    assert r3.returncode != 0 and "operator file" in r3.stderr
