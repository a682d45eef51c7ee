"""GPU checks at the sizes of the benchmark configurations.

* Laplace potential, 100,000 uniform points (seeds 1, 2), m=6, 300/leaf,
  plain FP64: GPU vs the oracle FMM on all N, rel-L2 <= 1e-12.
* Stokes velocity, 2,000,000 uniform points (seed 21), forces N(0,1)^3
  (seed 22), m=10, 300/leaf, mixed form: rel-L2 vs an FP64 direct sum on
  1,000 targets (seed 23) <= 1e-6.
* Laplace potential, 30,000,000 points uniform by area on the ellipsoid with
  semi-axes (0.45, 0.3, 0.15) centred at 0.5 (rejection sampling with
  acceptance proportional to the area element, seed 41), q ~ U[-1,1]
  (seed 42), m=8, 128/leaf, mixed form: forward and adjoint (swapped-role)
  evaluations vs FP64 direct sums on 1,000 points, rel-L2 <= 1e-6, and the
  adjoint identity <g, A q> = <A^T g, q> to the same tolerance.
"""
import math

import numpy as np
import pytest
import torch

import pvfmm_b200 as P
from oracle import pvfmm_oracle as O

pytestmark = pytest.mark.gpu


def _direct(kid, x, q, t, chunk=1 << 14):
    """FP64 direct sum on the GPU (torch): values at targets t, r == 0 excluded."""
    X = torch.as_tensor(x, device="cuda", dtype=torch.float64)
    Q = torch.as_tensor(q, device="cuda", dtype=torch.float64).reshape(X.shape[0], -1)
    T = torch.as_tensor(t, device="cuda", dtype=torch.float64)
    k1 = 3 if kid == 3 else (4 if kid == 6 else 1)
    out = torch.zeros((T.shape[0], k1), device="cuda", dtype=torch.float64)
    for a in range(0, X.shape[0], chunk):
        d = T[:, None, :] - X[None, a:a + chunk, :]
        r2 = (d * d).sum(-1)
        rinv = torch.where(r2 > 0, r2.clamp_min(1e-300).rsqrt(), torch.zeros_like(r2))
        qa = Q[a:a + chunk]
        if kid == 0:
            out[:, 0] += rinv @ qa[:, 0]
        elif kid == 3:
            ip = torch.einsum("tsk,sk->ts", d, qa) * rinv * rinv
            out += torch.einsum("ts,sk->tk", rinv, qa) + torch.einsum("ts,tsk->tk", rinv * ip, d)
        else:
            raise ValueError(kid)
    return (out / (8 * math.pi if kid == 3 else 4 * math.pi)).cpu().numpy()


def test_config1_plain_matches_oracle_100k():
    n = 100_000
    x = np.random.default_rng(1).random((n, 3))
    q = np.random.default_rng(2).uniform(-1, 1, n)
    ops = O.Operators.from_arrays(O.KERNELS[0], 6, P.precomp_operators(P.FMMKernel.LaplacePotential, 6, 0))
    ref = O.pvfmm_eval(0, 6, 300, x, q, x, ops=ops)
    ctx = P.FMMParticleContext(-1, 300, 6, P.FMMKernel.LaplacePotential)
    xf = x.reshape(-1)
    got = ctx.evaluate(xf, q, None, xf, True).reshape(n, 1)
    assert O.rel_l2(got, ref) < 1e-12
    idx = np.random.default_rng(3).choice(n, 1000, replace=False)
    assert O.rel_l2(got[idx], _direct(0, x, q, x[idx])) < 1e-5
    ctx.close()


def test_config3_stokes_2m_mixed_accuracy():
    n = 2_000_000
    x = np.random.default_rng(21).random((n, 3))
    f = np.random.default_rng(22).standard_normal((n, 3))
    ctx = P.FMMParticleContext(-1, 300, 10, P.FMMKernel.StokesVelocity, precision=P.PRECISION_MIXED)
    xf = x.reshape(-1)
    got = ctx.evaluate(xf, f.reshape(-1), None, xf, True).reshape(n, 3)
    idx = np.random.default_rng(23).choice(n, 1000, replace=False)
    err = O.rel_l2(got[idx], _direct(3, x, f, x[idx]))
    assert err < 1e-6, err
    ctx.close()


def ellipsoid_surface(n, seed=41, axes=(0.45, 0.3, 0.15), centre=0.5):
    """Points uniform by area on the ellipsoid c + a*u, |u| = 1: uniform
    directions u, accepted with probability |u/a| min(a) (the area element
    abc |u/a| over its maximum abc / min(a))."""
    rng = np.random.default_rng(seed)
    a = np.asarray(axes)
    out = []
    have = 0
    while have < n:
        m = int((n - have) * 2.2) + 1000
        u = rng.standard_normal((m, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        acc = rng.random(m) < np.linalg.norm(u / a, axis=1) * a.min()
        pts = centre + u[acc] * a
        out.append(pts)
        have += len(pts)
    return np.concatenate(out)[:n]


def test_config5_ellipsoid_30m_forward_and_adjoint():
    n = 30_000_000
    x = ellipsoid_surface(n)
    q = np.random.default_rng(42).uniform(-1, 1, n)
    g = np.random.default_rng(43).uniform(-1, 1, n)
    X = torch.as_tensor(x, device="cuda")
    Q = torch.as_tensor(q, device="cuda")
    Gd = torch.as_tensor(g, device="cuda")
    ctx = P.FMMParticleContext(-1, 128, 8, P.FMMKernel.LaplacePotential, precision=P.PRECISION_MIXED)
    phi = torch.empty(n, device="cuda", dtype=torch.float64)
    adj = torch.empty(n, device="cuda", dtype=torch.float64)
    ctx.evaluate_device(X.data_ptr(), Q.data_ptr(), n, X.data_ptr(), phi.data_ptr(), n, True, 0)
    ctx.evaluate_adjoint_device(X.data_ptr(), n, X.data_ptr(), Gd.data_ptr(), n, adj.data_ptr(), False, 0)
    idx = np.random.default_rng(44).choice(n, 1000, replace=False)
    e_fwd = O.rel_l2(phi.cpu().numpy()[idx], _direct(0, x, q, x[idx])[:, 0])
    e_adj = O.rel_l2(adj.cpu().numpy()[idx], _direct(0, x, g, x[idx])[:, 0])
    assert e_fwd < 1e-6, e_fwd
    assert e_adj < 1e-6, e_adj
    lhs = float(torch.dot(Gd, phi))
    rhs = float(torch.dot(adj, Q))
    assert abs(lhs - rhs) <= 1e-6 * math.sqrt(float(torch.dot(Gd, Gd)) * float(torch.dot(phi, phi)))
    ctx.close()
