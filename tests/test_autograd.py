"""Gradients of the differentiable Laplace FMM (pvfmm_b200.autograd).

Workload: N = 1,000,000 points uniform in [0,1)^3 (seed 31), densities
q ~ U[-1,1] (seed 32), weights w ~ U[0,1] (seed 33), loss L = sum_i w_i phi_i^2
with phi the Laplace single-layer potential of the points at themselves,
m = 8, 256 points per leaf, FP32 tensors, mixed form.

* Against an FP64 direct-sum gradient on a 20,000-point subset (seed 35):
  dL/dq and dL/dx, rel-L2 <= 1e-5.
* Against central finite differences of FP64 FMM evaluations at full size on
  20 coordinates chosen with seed 34 (10 densities, 10 position components):
  densities by one central difference with h = 1e-4 (L is quadratic in q, so
  it is exact up to rounding), positions by Richardson extrapolation of the
  central differences at h = 1e-5 and h/2 (truncation O(h^4 / r^4) for a
  neighbour at distance r: at h = 1e-4 a neighbour 1e-3 away would already
  leave ~1e-4).  The FP64 evaluations
  use a unit-box tree (coordinates as given), and a position coordinate whose
  perturbation changes the octree is replaced by the next candidate, so every
  difference is taken on one fixed octree.  Differences of L are summed as
  sum_i w_i (phi+_i - phi-_i)(phi+_i + phi-_i), which avoids cancelling two
  large totals.  Bar: rel-L2 <= 1e-5 for each group.
* Separate sources and targets (companion tree for the swapped roles), FP64:
  gradients of src, den and trg against the direct sum.
"""
import math

import numpy as np
import pytest
import torch

import pvfmm_b200 as P
import pvfmm_b200.autograd as PA

pytestmark = pytest.mark.gpu


def _field(x_trg, x_src, d, chunk=1024):
    """FP64 direct sums at x_trg: phi = sum_j d_j/(4 pi r), F = sum_j d_j (x - y_j)/(4 pi r^3), r == 0 excluded."""
    phi = torch.zeros(x_trg.shape[0], dtype=torch.float64, device=x_trg.device)
    F = torch.zeros(x_trg.shape[0], 3, dtype=torch.float64, device=x_trg.device)
    for a in range(0, x_trg.shape[0], chunk):
        r = x_trg[a:a + chunk, None, :] - x_src[None, :, :]
        r2 = (r * r).sum(-1)
        rinv = torch.where(r2 > 0, r2.clamp_min(1e-300).rsqrt(), torch.zeros_like(r2)) / (4 * math.pi)
        phi[a:a + chunk] = rinv @ d
        rinv3 = rinv * torch.where(r2 > 0, 1.0 / r2.clamp_min(1e-300), torch.zeros_like(r2))
        F[a:a + chunk] = torch.einsum("ij,ijk->ik", rinv3 * d[None, :], r)
    return phi, F


def _rel(a, b):
    a = a.double().reshape(-1)
    b = b.double().reshape(-1)
    return float((a - b).norm() / b.norm())


def _config_points(n, seed_x=31, seed_q=32, seed_w=33):
    x = np.random.default_rng(seed_x).random((n, 3))
    q = np.random.default_rng(seed_q).uniform(-1, 1, n)
    w = np.random.default_rng(seed_w).uniform(0, 1, n)
    return x, q, w


def test_gradients_match_direct_sum_on_subset():
    x, q, w = _config_points(1_000_000)
    idx = np.sort(np.random.default_rng(35).choice(len(x), 20000, replace=False))
    dev = torch.device("cuda:0")
    xs = torch.tensor(x[idx], dtype=torch.float32, device=dev).requires_grad_(True)
    qs = torch.tensor(q[idx], dtype=torch.float32, device=dev).requires_grad_(True)
    ws = torch.tensor(w[idx], dtype=torch.float64, device=dev)
    fmm = PA.LaplaceFMM(256, 8, "mixed")
    phi = fmm(xs, qs)
    L = (ws * phi.double() ** 2).sum()
    L.backward()
    # FP64 direct reference on the same (FP32-rounded) inputs
    X = xs.detach().double()
    Q = qs.detach().double()
    phi_d, F_q = _field(X, X, Q)
    g = 2 * ws * phi_d
    gq_d, F_g = _field(X, X, g)
    gx_d = -g[:, None] * F_q - Q[:, None] * F_g
    assert _rel(phi.detach(), phi_d) < 1e-5
    assert _rel(qs.grad, gq_d) < 1e-5
    assert _rel(xs.grad, gx_d) < 1e-5
    fmm.close()


def test_gradients_plain_fp64_separate_targets():
    rng = np.random.default_rng(8)
    dev = torch.device("cuda:0")
    y = torch.tensor(rng.random((6000, 3)), device=dev).requires_grad_(True)
    x = torch.tensor(rng.random((5000, 3)), device=dev).requires_grad_(True)
    q = torch.tensor(rng.uniform(-1, 1, 6000), device=dev).requires_grad_(True)
    w = torch.tensor(rng.uniform(0, 1, 5000), device=dev)
    fmm = PA.LaplaceFMM(64, 8, "plain")
    phi = fmm(y, q, x)
    (w * phi ** 2).sum().backward()
    Y, X, Q = y.detach(), x.detach(), q.detach()
    phi_d, E = _field(X, Y, Q)
    g = 2 * w * phi_d
    A, F_g = _field(Y, X, g)
    assert _rel(phi.detach(), phi_d) < 1e-6
    assert _rel(q.grad, A) < 1e-6
    assert _rel(x.grad, -g[:, None] * E) < 1e-6
    assert _rel(y.grad, -Q[:, None] * F_g) < 1e-6
    # a second forward + backward gives identical gradients (deterministic)
    gq = q.grad.clone()
    q.grad = None
    x.grad = None
    y.grad = None
    phi2 = fmm(y, q, x)
    (w * phi2 ** 2).sum().backward()
    assert torch.equal(q.grad, gq)
    fmm.close()


def test_gradients_match_finite_differences_full_size():
    n = 1_000_000
    x, q, w = _config_points(n)
    dev = torch.device("cuda:0")
    x32 = torch.tensor(x, dtype=torch.float32, device=dev).requires_grad_(True)
    q32 = torch.tensor(q, dtype=torch.float32, device=dev).requires_grad_(True)
    wt = torch.tensor(w, dtype=torch.float64, device=dev)
    fmm = PA.LaplaceFMM(256, 8, "mixed")
    (wt * fmm(x32, q32).double() ** 2).sum().backward()
    gq = q32.grad.double().cpu().numpy()
    gx = x32.grad.double().cpu().numpy()
    fmm.close()

    # FP64 FMM evaluations on the FP32-rounded inputs, unit-box tree
    X = x32.detach().double().cpu().numpy().copy()
    Q = q32.detach().double().cpu().numpy().copy()
    ctx = P.FMMParticleContext(-1, 256, 8, P.FMMKernel.LaplacePotential, dtype=np.float64)
    ctx.set_unit_box(True)

    def phi(xx, qq, setup):
        return ctx.evaluate(xx.reshape(-1), qq, None, xx.reshape(-1), setup)

    def tree_sig():
        return ctx.tree_data(2).tobytes() + ctx.tree_data(4).tobytes()

    phi(X, Q, True)
    sig0 = tree_sig()
    rng = np.random.default_rng(34)
    h = 1e-4
    fd_q, ag_q = [], []
    for j in rng.choice(n, 10, replace=False):
        qp, qm = Q.copy(), Q.copy()
        qp[j] += h
        qm[j] -= h
        pp, pm = phi(X, qp, False), phi(X, qm, False)
        fd_q.append(np.sum(w * (pp - pm) * (pp + pm)) / (2 * h))
        ag_q.append(gq[j])
    fd_x, ag_x = [], []
    hx = 1e-5
    for j, k in zip(rng.choice(n, 40, replace=False), rng.integers(0, 3, 40)):
        if len(fd_x) == 10:
            break
        if not (hx < X[j, k] < 1 - hx):
            continue
        d = []
        same_tree = True
        for step in (hx, hx / 2):
            xp, xm = X.copy(), X.copy()
            xp[j, k] += step
            xm[j, k] -= step
            pp = phi(xp, Q, True)
            same_tree &= tree_sig() == sig0
            pm = phi(xm, Q, True)
            same_tree &= tree_sig() == sig0
            d.append(np.sum(w * (pp - pm) * (pp + pm)) / (2 * step))
        if not same_tree:
            continue
        fd_x.append((4 * d[1] - d[0]) / 3)
        ag_x.append(gx[j, k])
    ctx.close()
    assert len(fd_x) == 10
    rel_q = np.linalg.norm(np.array(ag_q) - fd_q) / np.linalg.norm(fd_q)
    rel_x = np.linalg.norm(np.array(ag_x) - fd_x) / np.linalg.norm(fd_x)
    per_x = np.abs(np.array(ag_x) - fd_x) / np.abs(fd_x)
    assert rel_q < 1e-5, rel_q
    assert rel_x < 1e-5, (rel_x, per_x)


def test_outputs_keep_the_input_dtype():
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(2)
    x = torch.tensor(rng.random((3000, 3)), device=dev).requires_grad_(True)
    q = torch.tensor(rng.uniform(-1, 1, 3000), device=dev).requires_grad_(True)
    fmm = PA.LaplaceFMM(128, 6, "mixed")
    phi = fmm(x, q)
    assert phi.dtype == torch.float64
    phi.sum().backward()
    assert x.grad.dtype == torch.float64 and q.grad.dtype == torch.float64
    fmm.close()
