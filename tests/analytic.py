"""Independent numpy evaluation of the analytic solutions, the modal basis and the L2 error.

Test infrastructure for checks that must not share code with the library or the oracle: nothing here
uses function_sets.h, quadrature.h or the library's basis tables.

- Dubiner basis (basis_dubiner_2D.cpp:4-83): phi_{p,q} = P_p^{0,0}(n1) ((1 - n2)/2)^p P_q^{2p+1,0}(n2) with
  n1 = 2 (1 + z1) / (1 - z2) - 1, n2 = z2, modes ordered by total degree n = p + q and then by p
  (dof = n (n + 1)/2 + p); at the singular vertex z2 = 1 the limit is q + 1 for p = 0 and 0 otherwise.
  Jacobi polynomials from scipy; pinned to the reference's own table (tests/golden/dubiner_2d.json).
- Quadrature: a collapsed (Duffy) Gauss-Legendre product rule on the master triangle
  (-1,-1), (1,-1), (-1,1), from numpy's leggauss.
- Manufactured standing wave (the configuration's formula): ze = A sin(kx) cos(ky) cos(wt), k = 2 pi / L.
  The momenta are chosen so that the continuity equation holds with no source:
  ze_t + (qx)_x + (qy)_y = 0 for qx = -B cos(kx) cos(ky) sin(wt), qy = B sin(kx) sin(ky) sin(wt),
  B = A w / (2k); w = k sqrt(2 g H), the frequency of the (k, k) gravity mode on depth H.
- Thacker (1981) oscillating paraboloid in the bowl b(r) = h0 (1 - r^2/a^2):
  A = ((h0 + eta0)^2 - h0^2) / ((h0 + eta0)^2 + h0^2), w = sqrt(8 g h0) / a,
  ze = h0 [sqrt(1 - A^2) / (1 - A cos wt) - 1 - r^2/a^2 ((1 - A^2)/(1 - A cos wt)^2 - 1)],
  (u, v) = w A sin(wt) / (2 (1 - A cos wt)) (x, y); dry (ze = -b, q = 0) where ze + b <= 0.
"""
import math

import numpy as np
from numpy.polynomial.legendre import leggauss
from scipy.special import eval_jacobi


def dof_pq(dof):
    n = int(math.ceil((-3.0 + math.sqrt(1.0 + 8.0 * (dof + 1))) / 2.0))
    p = dof - n * (n + 1) // 2
    return p, n - p


def dubiner_phi(order, z1, z2):
    """phi [ndof][npt] of the Dubiner basis of the given order at master points (z1, z2)."""
    z1 = np.asarray(z1, np.float64)
    z2 = np.asarray(z2, np.float64)
    nd = (order + 1) * (order + 2) // 2
    sing = np.isclose(z2, 1.0, rtol=0, atol=0)
    with np.errstate(divide="ignore", invalid="ignore"):
        n1 = np.where(sing, 0.0, 2.0 * (1.0 + z1) / (1.0 - z2) - 1.0)
    out = np.empty((nd, len(z1)))
    for dof in range(nd):
        p, q = dof_pq(dof)
        v = eval_jacobi(p, 0, 0, n1) * ((1.0 - z2) / 2.0) ** p * eval_jacobi(q, 2 * p + 1, 0, z2)
        out[dof] = np.where(sing, float(q + 1) if p == 0 else 0.0, v)
    return out


def collapsed_rule(n):
    """n x n collapsed Gauss rule on the master triangle: (z1, z2, w), sum(w) = 2 (the triangle's area);
    exact for polynomials of total degree <= 2n - 2."""
    a, wa = leggauss(n)
    b, wb = leggauss(n)
    A, B = np.meshgrid(a, b, indexing="ij")
    WA, WB = np.meshgrid(wa, wb, indexing="ij")
    z1 = (1.0 + A) * (1.0 - B) / 2.0 - 1.0
    z2 = B
    w = WA * WB * (1.0 - B) / 2.0
    return z1.ravel(), z2.ravel(), w.ravel()


def physical_points(node_xyz, elem_nodes, z1, z2):
    """x, y [ne][nq] of the master points in every straight triangle, and |J| [ne] (physical area / 2)."""
    X = node_xyz[elem_nodes, 0]
    Y = node_xyz[elem_nodes, 1]
    s0, s1, s2 = -(z1 + z2) / 2.0, (1.0 + z1) / 2.0, (1.0 + z2) / 2.0
    x = X[:, :1] * s0 + X[:, 1:2] * s1 + X[:, 2:3] * s2
    y = Y[:, :1] * s0 + Y[:, 1:2] * s1 + Y[:, 2:3] * s2
    detJ = ((X[:, 1] - X[:, 0]) * (Y[:, 2] - Y[:, 0]) - (X[:, 2] - X[:, 0]) * (Y[:, 1] - Y[:, 0])) / 4.0
    return x, y, detJ


class Manufactured:
    def __init__(self, L=40000.0, A=0.1, H=2.0, g=9.81):
        self.L, self.A, self.H, self.g = L, A, H, g
        self.k = 2.0 * math.pi / L
        self.w = self.k * math.sqrt(2.0 * g * H)
        self.B = A * self.w / (2.0 * self.k)

    def __call__(self, t, x, y):
        k, w = self.k, self.w
        ze = self.A * np.sin(k * x) * np.cos(k * y) * math.cos(w * t)
        qx = -self.B * np.cos(k * x) * np.cos(k * y) * math.sin(w * t)
        qy = self.B * np.sin(k * x) * np.sin(k * y) * math.sin(w * t)
        return np.stack([ze, qx, qy])

    def bath(self, x, y):
        return np.full_like(np.asarray(x, np.float64), self.H)


class Thacker:
    def __init__(self, h0=10.0, a=3000.0, eta0=2.0, g=9.81):
        self.h0, self.a, self.eta0, self.g = h0, a, eta0, g
        hp = (h0 + eta0) ** 2
        self.Acoef = (hp - h0 * h0) / (hp + h0 * h0)
        self.w = math.sqrt(8.0 * g * h0) / a

    def bath(self, x, y):
        return self.h0 * (1.0 - (np.asarray(x) ** 2 + np.asarray(y) ** 2) / self.a ** 2)

    def __call__(self, t, x, y):
        A, h0, a, w = self.Acoef, self.h0, self.a, self.w
        x = np.asarray(x, np.float64)
        y = np.asarray(y, np.float64)
        den = 1.0 - A * math.cos(w * t)
        r2 = x * x + y * y
        ze = h0 * (math.sqrt(1.0 - A * A) / den - 1.0 - r2 / a ** 2 * ((1.0 - A * A) / den ** 2 - 1.0))
        b = self.bath(x, y)
        h = ze + b
        fac = w * A * math.sin(w * t) / (2.0 * den)
        wet = h > 0.0
        return np.stack([np.where(wet, ze, -b), np.where(wet, h * x * fac, 0.0), np.where(wet, h * y * fac, 0.0)])


def l2_error(state, node_xyz, elem_nodes, order, true, t, n=8):
    """sqrt(sum_e int_e sum_var (q_true - q_h)^2 dA) of a modal state [ne][3][ndof] (ascending element
    order) against true(t, x, y) -> [3][...] (Simulation::ComputeL2Residual's quantity)."""
    z1, z2, w = collapsed_rule(n)
    phi = dubiner_phi(order, z1, z2)
    qh = np.einsum("evk,kq->veq", state, phi)
    x, y, detJ = physical_points(node_xyz, elem_nodes, z1, z2)
    err = true(t, x, y) - qh
    return math.sqrt(float(np.sum((err ** 2).sum(0) * w[None, :] * np.abs(detJ)[:, None])))
