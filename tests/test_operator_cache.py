"""Operator cache (no GPU): with PVFMM_DIR set, the pseudo-inverse factors are
written to / read from Precomp_<kernel>_m<m>.data in the layout of the
reference's precompute files (include/precomp_mat.txx:213-345 Save2File and
LoadFile; name include/fmm_pts.txx:246-276), and every operator built from
the file equals the one computed without it, bit for bit.
"""
import numpy as np
import pytest

import pvfmm_b200 as P

K = P.FMMKernel
N_WHICH = 9  # UC2UE0, UC2UE1, DC2DE0, DC2DE1, U2U, D2D, surface, V-list operators, projector


def _all(kernel, m, precision):
    # a different (kernel, order) first: the library keeps the last operator set
    P.precomp_operator(K.LaplacePotential, 2, 0, 0)
    return [P.precomp_operator(kernel, m, precision, w) for w in range(N_WHICH)]


def _read_reference_layout(path):
    """Parses a file in the reference's layout: [(n1, n2, data) per entry] per type."""
    b = open(path, "rb").read()
    pos = 0

    def i32():
        nonlocal pos
        v = int(np.frombuffer(b, np.int32, 1, pos)[0])
        pos += 4
        return v

    assert i32() == 8 and i32() == 1  # sizeof(double), scale-invariant
    types = []
    for _ in range(16):
        ents = []
        for _ in range(i32()):
            n1, n2 = i32(), i32()
            ents.append((n1, n2, np.frombuffer(b, np.float64, n1 * n2, pos)))
            pos += 8 * n1 * n2
        types.append(ents)
    assert pos == len(b)
    return types


def _write_reference_layout(path, types):
    with open(path, "wb") as fh:
        fh.write(np.array([8, 1], np.int32).tobytes())
        for ents in types:
            fh.write(np.array([len(ents)], np.int32).tobytes())
            for n1, n2, data in ents:
                fh.write(np.array([n1, n2], np.int32).tobytes())
                fh.write(np.asarray(data, np.float64).tobytes())


@pytest.fixture
def cache_dir(tmp_path, monkeypatch):
    monkeypatch.setenv("PVFMM_DIR", str(tmp_path))
    yield tmp_path
    monkeypatch.delenv("PVFMM_DIR")
    P.precomp_operator(K.LaplacePotential, 2, 0, 0)  # drop the operator set built with the cache


@pytest.mark.parametrize("kernel,m,name,kin,kout", [(K.LaplacePotential, 4, "laplace", 1, 1),
                                                    (K.StokesVelocity, 4, "stokes_vel", 3, 3),
                                                    (K.StokesPressure, 4, "stokes_press", 3, 1),
                                                    (K.StokesVelocityGrad, 4, "stokes_grad", 3, 9)])
def test_cache_is_written_and_reread_bit_identically(monkeypatch, cache_dir, kernel, m, name, kin, kout):
    monkeypatch.delenv("PVFMM_DIR")
    ref = _all(kernel, m, 0)
    monkeypatch.setenv("PVFMM_DIR", str(cache_dir))
    written = _all(kernel, m, 0)                    # computes, writes the file
    path = cache_dir / f"Precomp_{name}_m{m}.data"
    assert path.exists()
    reread = _all(kernel, m, 0)                     # reads the file
    for a, b, c in zip(ref, written, reread):
        assert np.array_equal(a, b) and np.array_equal(a, c)
    types = _read_reference_layout(path)
    ns = 6 * (m - 1) ** 2 + 2
    din, dout = ns * kin, ns * kout
    r = min(din, dout)
    for t in range(4):
        assert len(types[t]) == 1
        n1, n2, data = types[t][0]
        assert (n1, n2) == ((r, din) if t & 1 else (dout, r)) and np.array_equal(data, ref[t])
    assert all(len(types[t]) == 0 for t in range(4, 16))


def test_mixed_cutoffs_come_from_the_fp64_factors(monkeypatch, cache_dir):
    monkeypatch.delenv("PVFMM_DIR")
    ref = _all(K.StokesVelocity, 6, 1)              # FP32 cutoff throughout
    monkeypatch.setenv("PVFMM_DIR", str(cache_dir))
    _all(K.StokesVelocity, 6, 0)                    # file from the FP64-cutoff run
    got = _all(K.StokesVelocity, 6, 1)
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)
    dim = int(np.sqrt(got[0].size))
    assert np.count_nonzero(np.abs(got[0].reshape(dim, dim)).sum(0) == 0) > 0  # the FP32 cutoff drops columns


def test_reads_files_with_other_entries_in_the_reference_layout(monkeypatch, cache_dir):
    """A reference-written file keeps 500 entries per type, mostly empty, and
    other types filled (U2U class matrices, boundary operators): only entry 0
    of types 0-3 is used."""
    monkeypatch.delenv("PVFMM_DIR")
    ref = _all(K.LaplacePotential, 4, 0)
    dim = int(np.sqrt(ref[0].size))
    rng = np.random.default_rng(0)
    types = []
    for t in range(16):
        ents = [(0, 0, np.empty(0))] * 500
        if t < 4:
            ents = [(dim, dim, ref[t])] + ents[1:]
            ents[7] = (3, 5, rng.random(15))
        elif t in (5, 15):
            ents = [(dim, dim, rng.random(dim * dim))] + ents[1:]
        types.append(ents)
    _write_reference_layout(cache_dir / "Precomp_laplace_m4.data", types)
    monkeypatch.setenv("PVFMM_DIR", str(cache_dir))
    got = _all(K.LaplacePotential, 4, 0)
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)


def test_unusable_files_are_errors(cache_dir):
    _all(K.LaplacePotential, 4, 0)
    good = (cache_dir / "Precomp_laplace_m4.data").read_bytes()
    (cache_dir / "Precomp_laplace_m4.data").write_bytes(good[: len(good) // 2])
    with pytest.raises(RuntimeError, match="operator cache .* truncated"):
        _all(K.LaplacePotential, 4, 0)
    (cache_dir / "Precomp_laplace_m6.data").write_bytes(good)   # an m=4 file under the m=6 name
    with pytest.raises(RuntimeError, match="expected"):
        _all(K.LaplacePotential, 6, 0)
    (cache_dir / "Precomp_laplace_m8.data").write_bytes(np.array([4, 1], np.int32).tobytes())
    with pytest.raises(RuntimeError, match="not an FP64"):
        _all(K.LaplacePotential, 8, 0)
    # a declared size whose byte count overflows 64 bits
    (cache_dir / "Precomp_laplace_m10.data").write_bytes(np.array([8, 1, 1, 2**31 - 1, 2**31 - 1], np.int32).tobytes())
    with pytest.raises(RuntimeError, match="truncated"):
        _all(K.LaplacePotential, 10, 0)


def test_unwritable_directory_is_skipped(monkeypatch, tmp_path):
    missing = tmp_path / "missing"
    monkeypatch.setenv("PVFMM_DIR", str(missing))
    got = _all(K.LaplacePotential, 4, 0)
    monkeypatch.delenv("PVFMM_DIR")
    ref = _all(K.LaplacePotential, 4, 0)
    assert not missing.exists()
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)
