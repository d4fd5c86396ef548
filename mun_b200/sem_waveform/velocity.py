"""Velocity model builders of MUN's ``sem_waveform.velocity`` (host, float64).

A closed cubic B-spline interface curve is turned into a nodal velocity through the
signed distance to the curve and a sigmoid blend v = v_out + (v_in - v_out) s(-d/tau):

* canonical/layered packages (``Bspline_Coupling/SEM/sem_waveform/velocity.py:8-202``,
  ``CO2_plume/layered_model/inversion/sem_waveform/velocity.py:9-267``): the first
  control point is repeated 3 times and the knot vector is clamped on [0, 1];
* gridded-background package (``CO2_plume/one_stage/single_cubic/sem_waveform/
  velocity.py:10-332``): periodic closure (first 3 points appended, integer knots).

The closest curve parameter comes from the nearest of ``samples`` curve samples refined
by 7 Newton steps on phi(u) = |C(u) - x|^2 / 2 with clipping to the valid interval; the
sign is an even-odd point-in-polygon test against the sampled curve (the reference uses
matplotlib's Path.contains_points on the same polygon).
"""
from __future__ import annotations

import numpy as np

# ------------------------------------------------------------------ B-spline evaluation


class ClosedBSpline:
    """Cubic B-spline curve with value/first/second derivative evaluation."""

    def __init__(self, knots, ctrl, degree=3):
        self.t = np.asarray(knots, dtype=np.float64)
        self.c = np.asarray(ctrl, dtype=np.float64)
        self.k = int(degree)
        self.n = len(self.c)  # number of coefficients
        self.lo = self.t[self.k]
        self.hi = self.t[self.n]

    def _span(self, u):
        # index i with t[i] <= u < t[i+1], k <= i <= n-1; u == hi uses the last span
        i = np.searchsorted(self.t, u, side="right") - 1
        return np.clip(i, self.k, self.n - 1)

    def eval(self, u, der=0):
        """Value (der=0), first (1) or second (2) derivative at parameters u (any shape)."""
        u = np.asarray(u, dtype=np.float64)
        shape = u.shape
        uf = u.reshape(-1)
        t, k = self.t, self.k
        i = self._span(uf)
        # de Boor basis functions of degree k and their derivatives at uf
        # N[p, j]: basis N_{i-p+j, p}
        M = len(uf)
        N = np.zeros((M, k + 1))
        N[:, 0] = 1.0
        left = np.zeros((M, k + 1))
        right = np.zeros((M, k + 1))
        ndu = [N[:, :1].copy()]
        for j in range(1, k + 1):
            left[:, j] = uf - t[i + 1 - j]
            right[:, j] = t[i + j] - uf
            saved = np.zeros(M)
            newN = np.zeros((M, j + 1))
            for r in range(j):
                denom = right[:, r + 1] + left[:, j - r]
                with np.errstate(divide="ignore", invalid="ignore"):
                    temp = np.where(denom != 0.0, ndu[-1][:, r] / denom, 0.0)
                newN[:, r] = saved + right[:, r + 1] * temp
                saved = left[:, j - r] * temp
            newN[:, j] = saved
            ndu.append(newN)
        # derivative via the lower-degree basis: d/du sum c_j N_{j,k} = sum (k (c_j - c_{j-1})
        # / (t_{j+k} - t_j)) N_{j,k-1}
        coef = self.c
        deg = k
        basis = ndu[k]
        idx = i[:, None] - k + np.arange(k + 1)[None, :]
        if der == 0:
            return np.einsum("mj,mjd->md", basis, coef[idx]).reshape(shape + coef.shape[1:])
        # differentiate coefficients der times
        c = coef
        tt = t
        for d in range(der):
            dc = np.zeros_like(c)
            for j in range(1, len(c)):
                den = tt[j + deg] - tt[j]
                dc[j] = deg * (c[j] - c[j - 1]) / den if den > 0 else 0.0
            c = dc
            deg -= 1
        basis = ndu[deg]
        idx = i[:, None] - deg + np.arange(deg + 1)[None, :]
        return np.einsum("mj,mjd->md", basis, c[idx]).reshape(shape + coef.shape[1:])

    def basis_matrix(self, u):
        """(len(u), n) values of every basis function at u."""
        u = np.asarray(u, dtype=np.float64).reshape(-1)
        out = np.zeros((len(u), self.n))
        for j in range(self.n):
            e = np.zeros(self.n)
            e[j] = 1.0
            out[:, j] = ClosedBSpline(self.t, e[:, None], self.k).eval(u)[:, 0]
        return out


def closed_spline_clamped(ctrl):
    """First point repeated 3 times, clamped knots on [0, 1] (canonical/layered)."""
    P = np.asarray(ctrl, dtype=np.float64).reshape(-1, 2)
    k = 3
    cc = np.vstack([P, np.tile(P[0], (k, 1))])
    n = len(cc) - 1
    knots = np.zeros(n + k + 2)
    knots[-(k + 1):] = 1.0
    knots[k + 1:-(k + 1)] = np.linspace(0.0, 1.0, n - k + 2)[1:-1]
    return ClosedBSpline(knots, cc, k)


def closed_spline_periodic(ctrl):
    """Periodic closure: first 3 points appended, knots 0..len+3 (gridded package)."""
    P = np.asarray(ctrl, dtype=np.float64).reshape(-1, 2)
    k = 3
    if P.shape[0] < k + 1:
        raise ValueError(f"At least {k + 1} control points are required for degree {k}; got {P.shape[0]}")
    cc = np.vstack([P, P[:k]])
    knots = np.arange(0.0, len(cc) + k + 1)
    return ClosedBSpline(knots, cc, k)


def points_in_polygon(pts, poly):
    """Even-odd crossing test."""
    x, y = pts[:, 0], pts[:, 1]
    vx, vy = poly[:, 0], poly[:, 1]
    wx, wy = np.roll(vx, -1), np.roll(vy, -1)
    inside = np.zeros(len(pts), dtype=bool)
    for ax, ay, bx, by in zip(vx, vy, wx, wy):
        if ay == by:
            continue
        cond = (ay > y) != (by > y)
        xc = ax + (y - ay) * (bx - ax) / (by - ay)
        inside ^= cond & (x < xc)
    return inside


def signed_distance_to_spline_newton(coords_xy, ctrl6_xy, samples=800, newton_steps=7, topk=1,
                                     chunk=20000, return_extra=True, periodic=False):
    X_all = np.asarray(coords_xy, dtype=np.float64).reshape(-1, 2)
    sp = closed_spline_periodic(ctrl6_xy) if periodic else closed_spline_clamped(ctrl6_xy)
    lo, hi = sp.lo, sp.hi
    if periodic:
        u0 = np.linspace(lo, hi, int(samples), endpoint=False)
    else:
        u0 = np.linspace(lo, hi, int(samples))
    C0 = sp.eval(u0)
    n = len(X_all)
    sd = np.empty(n)
    u_star = np.empty(n)
    closest = np.empty((n, 2))
    tangent = np.empty((n, 2))
    normal = np.empty((n, 2))
    for s in range(0, n, chunk):
        X = X_all[s:s + chunk]
        d2 = ((X[:, None, :] - C0[None, :, :]) ** 2).sum(-1)
        if topk == 1:
            u = u0[np.argmin(d2, axis=1)][:, None]
        else:
            u = u0[np.argpartition(d2, topk - 1, axis=1)[:, :topk]]
        for _ in range(newton_steps):
            Cu, Cp, Cpp = sp.eval(u), sp.eval(u, 1), sp.eval(u, 2)
            r = Cu - X[:, None, :]
            f1 = (r * Cp).sum(-1)
            f2 = (Cp * Cp).sum(-1) + (r * Cpp).sum(-1)
            f2 = np.where(np.abs(f2) < 1e-14, 1e-14, f2)
            u = np.clip(u - f1 / f2, lo, hi)
        if topk > 1:
            r = sp.eval(u) - X[:, None, :]
            ub = u[np.arange(len(X)), np.argmin((r * r).sum(-1), axis=1)]
        else:
            ub = u[:, 0]
        Cb = sp.eval(ub)
        Tb = sp.eval(ub, 1)
        th = Tb / (np.linalg.norm(Tb, axis=1, keepdims=True) + 1e-15)
        rv = X - Cb
        dist = np.linalg.norm(rv, axis=1)
        sign = np.where(points_in_polygon(X, C0), -1.0, 1.0)
        sd[s:s + chunk] = sign * dist
        u_star[s:s + chunk] = ub
        closest[s:s + chunk] = Cb
        tangent[s:s + chunk] = th
        normal[s:s + chunk] = sign[:, None] * rv / (dist[:, None] + 1e-15)
    if return_extra:
        return sd, u_star, closest, tangent, normal
    return sd


def _sigmoid_blend(sd, tau):
    tau_safe = max(float(tau), 1e-12)
    x = np.clip(sd / tau_safe, -50.0, 50.0)
    return 1.0 / (1.0 + np.exp(x))


def build_velocity_on_sem_nodes(nodes_xy, ctrl6_xy, v_inside, v_outside, tau, samples=800,
                                newton_steps=7, periodic=False):
    nodes_xy = np.asarray(nodes_xy)
    if nodes_xy.ndim == 1:
        if nodes_xy.size % 2:
            raise ValueError(f"'nodes_xy' must be (N,2); got 1D of size {nodes_xy.size}.")
        nodes_xy = nodes_xy.reshape(-1, 2)
    if nodes_xy.ndim != 2 or nodes_xy.shape[1] != 2:
        raise ValueError(f"'nodes_xy' must be (N,2); got shape {nodes_xy.shape}")
    sd, us, cb, th, no = signed_distance_to_spline_newton(nodes_xy, ctrl6_xy, samples, newton_steps,
                                                          periodic=periodic)
    v = v_outside + (v_inside - v_outside) * _sigmoid_blend(sd, tau)
    return v, sd, {"u_star": us, "closest": cb, "tangent": th, "normal_out": no}


def build_layered_background(nodes_xy, interfaces_z, velocities):
    z = np.asarray(nodes_xy, dtype=np.float64)[:, 1]
    iz = np.asarray(interfaces_z, dtype=np.float64).reshape(-1)
    vel = np.asarray(velocities, dtype=np.float64).reshape(-1)
    if iz.size + 1 != vel.size:
        raise ValueError("len(velocities) must be len(interfaces_z)+1 (L layers).")
    return vel[np.searchsorted(iz, z, side="right")]


def build_velocity_layered_with_anomaly(nodes_xy, interfaces_z, layer_velocities, ctrl6_xy=None,
                                        v_inside=None, tau=10.0, samples=800, newton_steps=7,
                                        blend="smooth", periodic=False):
    v_layer = build_layered_background(nodes_xy, interfaces_z, layer_velocities)
    if ctrl6_xy is None:
        return v_layer, None, None
    sd, us, cb, th, no = signed_distance_to_spline_newton(nodes_xy, ctrl6_xy, samples, newton_steps,
                                                          periodic=periodic)
    if blend == "replace":
        v = v_layer.copy()
        v[sd < 0.0] = float(v_inside)
    else:
        v = v_layer + (float(v_inside) - v_layer) * _sigmoid_blend(sd, tau)
    return v, sd, {"u_star": us, "closest": cb, "tangent": th, "normal_out": no}


def build_background_from_grid(nodes_xy, xg, zg, vp_grid, method="linear", clip=True):
    """Bilinear (or nearest) interpolation of a (nz, nx) grid onto the nodes
    (gridded velocity.py:212-274, RegularGridInterpolator on axes (z, x))."""
    P = np.asarray(nodes_xy, dtype=np.float64).reshape(-1, 2)
    xg = np.asarray(xg, dtype=np.float64).reshape(-1)
    zg = np.asarray(zg, dtype=np.float64).reshape(-1)
    V = np.asarray(vp_grid, dtype=np.float64)
    if V.shape != (zg.size, xg.size):
        raise ValueError(f"vp_grid shape {V.shape} must be (len(zg), len(xg)) = {(zg.size, xg.size)}")
    x, z = P[:, 0].copy(), P[:, 1].copy()
    if clip:
        x = np.clip(x, xg[0], xg[-1])
        z = np.clip(z, zg[0], zg[-1])
    ix = np.clip(np.searchsorted(xg, x, side="right") - 1, 0, xg.size - 2)
    iz = np.clip(np.searchsorted(zg, z, side="right") - 1, 0, zg.size - 2)
    if method == "nearest":
        jx = np.where(np.abs(x - xg[ix]) <= np.abs(xg[ix + 1] - x), ix, ix + 1)
        jz = np.where(np.abs(z - zg[iz]) <= np.abs(zg[iz + 1] - z), iz, iz + 1)
        return V[jz, jx]
    fx = (x - xg[ix]) / (xg[ix + 1] - xg[ix])
    fz = (z - zg[iz]) / (zg[iz + 1] - zg[iz])
    return ((1 - fz) * ((1 - fx) * V[iz, ix] + fx * V[iz, ix + 1])
            + fz * ((1 - fx) * V[iz + 1, ix] + fx * V[iz + 1, ix + 1]))


def build_velocity_2d_background_with_anomaly(nodes_xy, v_background, ctrl6_xy=None, v_inside=None,
                                              tau=10.0, samples=800, newton_steps=7, blend="smooth"):
    P = np.asarray(nodes_xy, dtype=np.float64).reshape(-1, 2)
    v_bg = np.asarray(v_background, dtype=np.float64).reshape(-1)
    if v_bg.size != P.shape[0]:
        raise ValueError(f"v_background must have length {P.shape[0]} (npoints); got {v_bg.size}")
    if ctrl6_xy is None:
        return v_bg.copy(), None, None
    sd, us, cb, th, no = signed_distance_to_spline_newton(P, ctrl6_xy, samples, newton_steps,
                                                          periodic=True)
    if blend == "replace":
        v = v_bg.copy()
        v[sd < 0.0] = float(v_inside)
    else:
        v = v_bg + (float(v_inside) - v_bg) * _sigmoid_blend(sd, tau)
    return v, sd, {"u_star": us, "closest": cb, "tangent": th, "normal_out": no}


# ------------------------------------------------------------------ device builder


def build_velocity_device(coords_dev, ctrl, tau, samples, v_inside, v_outside=None, v_background_dev=None,
                          newton_steps=7, periodic=False, blend="smooth", stream=None, sync=True):
    """Same result as the host builders above, computed on the GPU
    (``sem_velocity_from_curve``).  ``coords_dev``: (P,2) float64 CUDA tensor; the
    background is either ``v_outside`` (constant) or ``v_background_dev`` (P,).
    Returns CUDA tensors (velocity, sd, u_star, normal_out).  ``sync=False`` leaves the
    build queued on the current stream (the outputs are stream-ordered tensors)."""
    import ctypes as C

    import torch

    from .. import _lib
    sp = closed_spline_periodic(ctrl) if periodic else closed_spline_clamped(ctrl)
    if periodic:
        u0 = np.linspace(sp.lo, sp.hi, int(samples), endpoint=False)
    else:
        u0 = np.linspace(sp.lo, sp.hi, int(samples))
    C0 = sp.eval(u0)
    dev = coords_dev.device
    u0_d = torch.as_tensor(u0, device=dev)
    s_d = torch.as_tensor(np.ascontiguousarray(C0), device=dev)
    n = coords_dev.shape[0]
    vel = torch.empty(n, dtype=torch.float64, device=dev)
    sd = torch.empty(n, dtype=torch.float64, device=dev)
    us = torch.empty(n, dtype=torch.float64, device=dev)
    nr = torch.empty((n, 2), dtype=torch.float64, device=dev)
    knots = np.ascontiguousarray(sp.t, dtype=np.float64)
    coef = np.ascontiguousarray(sp.c, dtype=np.float64)
    cd = _lib.CurveDesc(len(coef), knots.ctypes.data_as(C.POINTER(C.c_double)),
                        coef.ctypes.data_as(C.POINTER(C.c_double)), float(sp.lo), float(sp.hi),
                        len(u0), u0_d.data_ptr(), s_d.data_ptr(), int(newton_steps), float(tau),
                        float(v_inside), 1 if blend == "replace" else 0)
    lib = _lib.load()
    cs = coords_dev.contiguous()
    strm = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    rc = lib.sem_velocity_from_curve(
        C.byref(cd), int(n), C.c_void_p(cs.data_ptr()),
        C.c_void_p(v_background_dev.data_ptr()) if v_background_dev is not None else None,
        float(v_outside if v_outside is not None else 0.0), C.c_void_p(vel.data_ptr()),
        C.c_void_p(sd.data_ptr()), C.c_void_p(us.data_ptr()), C.c_void_p(nr.data_ptr()), C.c_void_p(strm))
    if rc != 0:
        raise ValueError("sem_velocity_from_curve: " + lib.sem_velocity_last_error().decode())
    if sync and stream is None:
        torch.cuda.current_stream().synchronize()
    del u0_d, s_d, cs
    return vel, sd, us, nr


def project_ctrl_device(ctrl, periodic, dL, sd, us, nrm, v_inside, tau, v_background_dev=None,
                        v_background_const=0.0, floor_one=True):
    """Control-point gradients for a batch on the GPU (``sem_project_from_curve``).
    dL, sd, us: (S, P) float64 CUDA tensors, nrm (S, P, 2); returns (S, 2K) with the K
    x-components first, then the K z-components."""
    import ctypes as C

    import torch

    from .. import _lib
    P = np.asarray(ctrl, dtype=np.float64).reshape(-1, 2)
    K = P.shape[0]
    sp = closed_spline_periodic(P) if periodic else closed_spline_clamped(P)
    knots = np.ascontiguousarray(sp.t, dtype=np.float64)
    S, npts = dL.shape
    out = torch.empty((S, 2 * K), dtype=torch.float64, device=dL.device)
    tens = [t.contiguous() for t in (dL, sd, us, nrm)]
    lib = _lib.load()
    rc = lib.sem_project_from_curve(
        knots.ctypes.data_as(C.c_void_p), int(len(sp.c)), int(K), 1 if periodic else 0, int(S), int(npts),
        C.c_void_p(tens[0].data_ptr()), C.c_void_p(tens[1].data_ptr()), C.c_void_p(tens[2].data_ptr()),
        C.c_void_p(tens[3].data_ptr()),
        C.c_void_p(v_background_dev.data_ptr()) if v_background_dev is not None else None,
        float(v_background_const), float(v_inside), float(tau), 1 if floor_one else 0,
        C.c_void_p(out.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    if rc != 0:
        raise ValueError("sem_project_from_curve: " + lib.sem_velocity_last_error().decode())
    return out
