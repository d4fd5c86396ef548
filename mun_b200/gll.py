"""1-D Gauss-Lobatto-Legendre machinery in float64.

Same discrete quantities as MUN's ``Bspline_Coupling/SEM/sem_waveform/utils.py:5-61``:
nodes (roots of P_N' plus +-1), weights 2/(N(N+1)P_N^2), the barycentric
differentiation matrix, and Lagrange polynomials with the reference's ``+1e-12`` added
to every denominator (so the interpolation matrix L is diag(l) with l = 1 - O(1e-11)).
The roots are polished with Newton's method on P_N' (analytic P_N''), so they agree
with the reference's secant-refined roots to about one unit in the last place.
"""
import numpy as np


def legendre(n, x):
    """(P_n(x), P_n'(x)) by the three-term recurrence."""
    x = np.asarray(x, dtype=np.float64)
    p_prev, p = np.ones_like(x), x.copy()
    if n == 0:
        return np.ones_like(x), np.zeros_like(x)
    for k in range(2, n + 1):
        p_prev, p = p, ((2 * k - 1) * x * p - (k - 1) * p_prev) / k
    with np.errstate(divide="ignore", invalid="ignore"):
        dp = n * (x * p - p_prev) / (x * x - 1.0)
    return p, dp


def gll_points(n):
    if n == 0:
        return np.array([0.0])
    if n == 1:
        return np.array([-1.0, 1.0])
    x = np.sort(np.cos(np.pi * np.arange(n + 1) / n))
    for i in range(1, n):
        xi = float(x[i])
        for _ in range(60):
            p, dp = legendre(n, xi)
            d2p = (2.0 * xi * dp - n * (n + 1) * p) / (1.0 - xi * xi)
            step = float(dp / d2p)
            xi -= step
            if abs(step) <= 1e-17:
                break
        x[i] = xi
    x[0], x[-1] = -1.0, 1.0
    return x


def gll_weights(nodes):
    n = len(nodes) - 1
    p, _ = legendre(n, nodes)
    return 2.0 / (n * (n + 1) * p * p)


def lagrange_basis(x, i, nodes):
    """i-th Lagrange polynomial at x with ``+1e-12`` in each denominator."""
    x = np.asarray(x, dtype=np.float64)
    out = np.ones_like(x)
    for j in range(len(nodes)):
        if j != i:
            out = out * ((x - nodes[j]) / (nodes[i] - nodes[j] + 1e-12))
    return out


def diff_matrix(nodes):
    """D[a, b] = l_b'(x_a) from barycentric weights; diagonal = -row sum."""
    n = len(nodes)
    w = np.array([1.0 / np.prod([nodes[j] - nodes[k] for k in range(n) if k != j]) for j in range(n)])
    D = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            if i != j:
                D[i, j] = w[j] / (w[i] * (nodes[i] - nodes[j]))
        D[i, i] = -np.sum(D[i, :])
    return D


def lagrange_diag(nodes):
    """l_a = L[a, a] of the reference's interpolation matrix (exactly diagonal)."""
    return np.array([float(lagrange_basis(nodes[a], a, nodes)) for a in range(len(nodes))])
