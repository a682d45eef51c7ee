"""The oracle's Stokes pressure, Stokes velocity gradient and Biot-Savart
kernels (reference include/kernel.txx:1366-1432, 1492-1511) and its FMM on
them (the kernels expand themselves, kernel.txx:894-901).

Pins, independent of the formulas restated in the oracle:
* the Stokeslet satisfies the Stokes equations away from the source:
  Laplacian(u) = grad(p) (unit viscosity) and div(u) = 0, with u the Stokes
  velocity kernel already pinned against the reference's normalisation;
* the velocity-gradient kernel is the target gradient of the velocity kernel,
  u[3a+b] = d u_b / d x_a (finite differences);
* the Biot-Savart kernel is the curl of the vector potential f / (4 pi r);
* the scale exponents follow the reference's rule (kernel.txx:64-196:
  log2 K(x/2)/K(x) per component pair, least squares with src_scal[0] = 0);
* the FMM converges to the direct sum as the order grows.
"""
import numpy as np
import pytest

from oracle import pvfmm_oracle as O

H = 1e-4


def _val(fn, f, x, y=np.zeros(3)):
    """fn's field at targets x from a point force f at y: (n, k1)."""
    return fn.eval(y[None], f, np.atleast_2d(x))


def _grad(fn, f, x, k):
    """d/dx_a of output component k at x (central differences), a = 0..2."""
    g = np.zeros(3)
    for a in range(3):
        e = np.zeros(3)
        e[a] = H
        g[a] = (_val(fn, f, x + e)[0, k] - _val(fn, f, x - e)[0, k]) / (2 * H)
    return g


def _points(seed, n=6):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, 3))
    return x / np.linalg.norm(x, axis=1, keepdims=True) * rng.uniform(0.5, 2.0, (n, 1))


def test_stokeslet_satisfies_stokes_equations():
    f = np.array([0.3, -1.1, 0.7])
    for x in _points(1):
        grad_p = _grad(O.STOKES_PRESS, f, x, 0)
        lap_u = np.zeros(3)
        for a in range(3):
            e = np.zeros(3)
            e[a] = H
            lap_u += (_val(O.STOKES, f, x + e)[0] - 2 * _val(O.STOKES, f, x)[0] + _val(O.STOKES, f, x - e)[0]) / H ** 2
        np.testing.assert_allclose(lap_u, grad_p, rtol=1e-5, atol=1e-7)
        div_u = sum(_grad(O.STOKES, f, x, b)[b] for b in range(3))
        assert abs(div_u) < 1e-8


def test_velocity_gradient_kernel_is_the_gradient_of_the_velocity():
    f = np.array([-0.4, 0.9, 1.3])
    for x in _points(2):
        G = _val(O.STOKES_GRAD, f, x)[0].reshape(3, 3)      # G[a][b] = d u_b / d x_a
        fd = np.array([_grad(O.STOKES, f, x, b) for b in range(3)]).T
        np.testing.assert_allclose(G, fd, rtol=1e-6, atol=1e-9)
        assert abs(np.trace(G)) < 1e-12 * np.abs(G).max()


def test_biot_savart_is_the_curl_of_the_vector_potential():
    f = np.array([1.0, -0.5, 0.25])
    for x in _points(3):
        B = _val(O.BIOT_SAVART, f, x)[0]
        # A_i = f_i / (4 pi r): curl A from finite differences of the Laplace kernel
        dA = np.array([_grad(O.LAPLACE, np.array([fi]), x, 0) for fi in f])   # dA[i][a] = d A_i / d x_a
        curl = np.array([dA[2][1] - dA[1][2], dA[0][2] - dA[2][0], dA[1][0] - dA[0][1]])
        np.testing.assert_allclose(B, curl, rtol=1e-6, atol=1e-9)


def _reference_scale_exponents(fn):
    """Restates Kernel::Initialize's scale detection (include/kernel.txx:64-196)
    for a homogeneous kernel: s[i0][i1] = log2 |K(x/2)| / |K(x)| per component
    pair, then the least-squares split s = src[i0] + trg[i1] with src[0] = 0."""
    x = np.array([[0.31, -0.27, 0.44], [0.52, 0.11, -0.37], [-0.23, 0.41, 0.19]])
    K1 = np.abs(fn.matrix(np.zeros((1, 3)), x)).reshape(fn.k0, -1, fn.k1).sum(1)
    K2 = np.abs(fn.matrix(np.zeros((1, 3)), x / 2)).reshape(fn.k0, -1, fn.k1).sum(1)
    M = np.zeros((fn.k0 * fn.k1 + 1, fn.k0 + fn.k1))
    b = np.zeros(fn.k0 * fn.k1 + 1)
    M[-1, 0] = 1
    for i0 in range(fn.k0):
        for i1 in range(fn.k1):
            if K1[i0, i1] > 0:
                j = i0 * fn.k1 + i1
                b[j] = np.log2(K2[i0, i1] / K1[i0, i1])
                M[j, i0] = M[j, fn.k0 + i1] = 1
    x = np.linalg.pinv(M) @ b
    return x[:fn.k0], x[fn.k0:]


@pytest.mark.parametrize("kid", [O.STOKES_PRESSURE, O.STOKES_VELOCITY_GRAD, O.BIOT_SAVART_POTENTIAL,
                                 O.LAPLACE_POTENTIAL, O.LAPLACE_GRADIENT, O.STOKES_VELOCITY])
def test_scale_exponents_follow_the_reference_rule(kid):
    K = O.KERNELS[kid]
    src, trg = _reference_scale_exponents(K.s2t)
    np.testing.assert_allclose(src, K.src_scal, atol=1e-9)
    np.testing.assert_allclose(trg, K.trg_scal, atol=1e-9)
    s_e, t_e = _reference_scale_exponents(K.exp)
    np.testing.assert_allclose(s_e, 0.0, atol=1e-9)
    np.testing.assert_allclose(t_e, K.exp.deg, atol=1e-9)


@pytest.mark.parametrize("kid", [O.STOKES_PRESSURE, O.STOKES_VELOCITY_GRAD, O.BIOT_SAVART_POTENTIAL])
def test_fmm_on_self_expanded_kernels_converges(kid):
    K = O.KERNELS[kid]
    rng = np.random.default_rng(40 + kid)
    x = rng.random((1500, 3))
    f = rng.standard_normal((1500, 3))
    ref = O.direct_sum(kid, x, f, x)
    errs = [O.rel_l2(O.pvfmm_eval(kid, m, 60, x, f, x), ref) for m in (4, 6)]
    assert errs[1] < 0.1 * errs[0], errs
    assert errs[1] < 1e-4, errs
