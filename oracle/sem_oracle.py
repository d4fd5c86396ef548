"""FP64 CPU oracle for the 2-D acoustic SEM forward solver and adjoint gradient.

TEST INFRASTRUCTURE ONLY.  This module is imported by ``tests/``, by
``__graft_entry__.smoke()`` and by ``bench.py`` (its ``cpu_baseline`` leg and the
``--impl reference`` arm) as the *checker*.  The product package ``mun_b200``
never imports it; the CUDA path fails loudly when its extension is missing.

It restates, in NumPy/PyTorch-CPU float64, the discrete algorithm of MUN's
``sem_waveform`` package (paths relative to the MUN project root):

* ``Bspline_Coupling/SEM/sem_waveform/utils.py:5-111``   GLL nodes/weights, Lagrange
  basis (with its ``+1e-12`` denominator quirk), barycentric D, CFL rule.
* ``Bspline_Coupling/SEM/sem_waveform/mesh.py:4-54``      first-seen node numbering,
  nearest-node source snapping.
* ``Bspline_Coupling/SEM/sem_waveform/operators.py:6-84,193-242`` Gx, Gz, S, w2D,
  lumped mass, assembled stiffness.
* ``Bspline_Coupling/SEM/sem_waveform/boundary.py:5-106`` cubic-ramp sponge.
* ``Bspline_Coupling/SEM/sem_waveform/sources.py:3-21``   Ricker + DC removal + gate.
* ``Bspline_Coupling/SEM/sem_waveform/receivers.py:6-108`` and
  ``CO2_plume/layered_model/inversion/sem_waveform/core.py:90-172`` receiver
  interpolation matrix (circle layout or explicit positions).
* ``Bspline_Coupling/SEM/sem_waveform/core.py:49-85``   per-step sensitivity kernel.
* ``Bspline_Coupling/SEM/sem_waveform/core.py:598-659`` forward loop of ``run()``
  (receivers recorded *before* the update).
* ``Bspline_Coupling/SEM/sem_waveform/core.py:1197-1278`` forward loop of
  ``run_forward_and_adjoint()`` (receivers recorded *after* update + sponge), misfit,
  and the adjoint loop (no sponge; gradient pairs ``u_hist[it]`` with lambda *before*
  its update; no ``dt`` factor in the time sum).
* ``Bspline_Coupling/SEM/sem_waveform/core.py:109-128`` observation alignment.

Parity is pinned by the golden vectors under ``tests/golden/`` which were produced by
running the reference package itself (``tests/golden/make_golden.py``).

The time loops use the same library calls as the reference (torch CSR mat-vec,
einsum, scatter_add) so that, timed on the host cores, they stand for the
reference's own CPU cost.  Set-up (mesh, mass, stiffness assembly) is vectorised
here, where the reference loops over elements in Python, so the oracle's set-up is
faster than the reference's; timings quoted from it are therefore conservative.

``mode='exact'`` additionally applies the sponge inside the adjoint loop, which makes
the gradient the exact discrete adjoint of the forward map (the reference's adjoint
omits it; see ``core.py:1252-1275``).

``method.boundary = 'stacey'`` selects an extension boundary mode that the reference
does not have: first-order Stacey absorbing conditions on the sides and the bottom and a
free surface (pressure release, u = 0) on the top, without the sponge.  Forward:
M u'' + C u' + K u = f with C = diag(c_i beta_i), beta_i the boundary quadrature weight
of node i (sum of w_a h/2 over its absorbing element edges), discretised by central
differences:  (1 + a) u+ = 2 u - (1 - a) u- + dt^2 M^-1 (f - K u),  a = dt c beta / (2 M),
then u+ = 0 on the top row.  Its exact discrete adjoint is the same recurrence run
backwards with the residual source, and the gradient adds to the stiffness term a
boundary-impedance term from d a / d c:
d loglik / d c_i += beta_i / (2 dt) * lambda_i * (u_i(t+1) - u_i(t-1)) at every adjoint step.

``device=`` runs the same float64 time loops on another torch device.  The tests at
the full sizes of the benchmark configurations (up to 1.28 M nodes and 5000 steps,
where the float64 forward history alone is 51 GB) use torch's CUDA backend for speed;
the arithmetic is the same float64 code that the golden vectors pin on the CPU.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
import torch

# --------------------------------------------------------------------------------------
# 1-D GLL machinery (utils.py:5-61)
# --------------------------------------------------------------------------------------


def _legendre(n: int, x):
    """Return (P_n(x), P_n'(x)) by the three-term recurrence."""
    x = np.asarray(x, dtype=np.float64)
    p0 = np.ones_like(x)
    if n == 0:
        return p0, np.zeros_like(x)
    p1 = x.copy()
    for k in range(2, n + 1):
        p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
    # derivative from the standard identity (x^2-1) P_n' = n (x P_n - P_{n-1})
    with np.errstate(divide="ignore", invalid="ignore"):
        dp = n * (x * p1 - p0) / (x * x - 1.0)
    return p1, dp


def gll_points(n: int) -> np.ndarray:
    """GLL nodes exactly as utils.py:5-21 computes them: the roots of P_n' found by
    ``scipy.optimize.newton`` (secant, no derivative given) from sorted Chebyshev
    guesses, with the end points set to +-1.  SciPy is the reference's own
    dependency (unpinned upstream; 1.18.1 in this image)."""
    from scipy.optimize import newton
    from scipy.special import legendre
    if n == 0:
        return np.array([0.0])
    if n == 1:
        return np.array([-1.0, 1.0])
    dP = legendre(n).deriv()
    x = np.sort(np.cos(np.pi * np.arange(n + 1) / n))
    for i in range(1, n):
        x[i] = newton(dP, x[i])
    x[0] = -1.0
    x[-1] = 1.0
    return x


def gll_weights(nodes: np.ndarray) -> np.ndarray:
    """w_i = 2 / (n (n+1) P_n(x_i)^2)   (utils.py:23-29, P_n from scipy.special)."""
    from scipy.special import legendre
    n = len(nodes) - 1
    return np.array([2 / (n * (n + 1) * legendre(n)(x) ** 2) for x in nodes])


def lagrange_basis(x, i: int, nodes: np.ndarray):
    """i-th Lagrange polynomial with the reference's ``+1e-12`` in each
    denominator (utils.py:31-37)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.ones_like(x)
    for j in range(len(nodes)):
        if j != i:
            out = out * ((x - nodes[j]) / (nodes[i] - nodes[j] + 1e-12))
    return out


def diff_matrix(nodes: np.ndarray) -> np.ndarray:
    """Barycentric differentiation matrix, diagonal = -row sum (utils.py:39-61)."""
    n = len(nodes)
    w = np.ones(n)
    for j in range(n):
        for k in range(n):
            if k != j:
                w[j] /= nodes[j] - nodes[k]
    D = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            if i != j:
                D[i, j] = w[j] / (w[i] * (nodes[i] - nodes[j]))
        D[i, i] = -np.sum(D[i, :])
    return D


def cfl_dt(velocity: np.ndarray, dt: float, total_time: float, npol: int,
           dx: float, dz: float):
    """utils.py:64-111: dt_max = 0.35 (min(dx,dz)/(p+1)) / (max c (p+1) sqrt 2);
    dt is lowered to dt_max only if it exceeds it; nt = ceil(T/dt)."""
    if not np.all(np.isfinite(velocity)):
        raise ValueError("[CFL] velocity_model contains non-finite values (NaN/Inf).")
    cmax = float(np.max(velocity))
    p = npol
    h_min = min(dx, dz) / (p + 1)
    dt_max = 0.35 * h_min / (cmax * (p + 1) * np.sqrt(2.0))
    if dt > dt_max:
        dt = float(dt_max)
    return dt, int(np.ceil(total_time / dt))


# --------------------------------------------------------------------------------------
# mesh (mesh.py:4-54)
# --------------------------------------------------------------------------------------


def create_global_mesh(xmin, xmax, zmin, zmax, nelx, nelz, npol):
    """Node coordinates in first-seen order and connectivity [ez*nx+ex][j*(N+1)+i].

    Returns (coords (P,2), conn (E,(N+1)^2) int64, grid_of_node (P,2) int64 holding the
    structured (gx, gz) index of every node)."""
    ngll = npol + 1
    xi = gll_points(npol)
    cx = np.linspace(xmin, xmax, nelx + 1)
    cz = np.linspace(zmin, zmax, nelz + 1)
    ez, ex, j, i = np.meshgrid(np.arange(nelz), np.arange(nelx), np.arange(ngll),
                               np.arange(ngll), indexing="ij")
    gx = (ex * npol + i).reshape(-1)
    gz = (ez * npol + j).reshape(-1)
    nxg = nelx * npol + 1
    lin = gz * nxg + gx
    uniq, first = np.unique(lin, return_index=True)
    order = np.argsort(first, kind="stable")
    node_lin = uniq[order]                       # node id -> structured linear index
    first_occ = first[order]
    ids = np.empty(lin.max() + 1, dtype=np.int64)
    ids[node_lin] = np.arange(len(node_lin))
    conn = ids[lin].reshape(nelz * nelx, ngll * ngll)
    # coordinates exactly as the reference computes them at first sight
    exf = ex.reshape(-1)[first_occ]
    ezf = ez.reshape(-1)[first_occ]
    xif = xi[i.reshape(-1)[first_occ]]
    etf = xi[j.reshape(-1)[first_occ]]
    x0, x1 = cx[exf], cx[exf + 1]
    z0, z1 = cz[ezf], cz[ezf + 1]
    x = 0.5 * ((1 - xif) * x0 + (1 + xif) * x1)
    z = 0.5 * ((1 - etf) * z0 + (1 + etf) * z1)
    coords = np.stack([x, z], axis=1)
    grid = np.stack([node_lin % nxg, node_lin // nxg], axis=1)
    return coords, conn, grid


def find_closest_node(x, z, coords):
    d = np.sqrt((coords[:, 0] - x) ** 2 + (coords[:, 1] - z) ** 2)
    return int(np.argmin(d))


# --------------------------------------------------------------------------------------
# element operators, mass and stiffness (operators.py:6-84,193-242)
# --------------------------------------------------------------------------------------


def sem_operators(dx, dz, npol):
    nodes = gll_points(npol)
    w = gll_weights(nodes)
    D = diff_matrix(nodes)
    ng = npol + 1
    L = np.zeros((ng, ng))
    for j in range(ng):
        for n in range(ng):
            L[j, n] = lagrange_basis(nodes[j], n, nodes)
    J = (dx * dz) * 0.25
    Gx = (2.0 / dx) * np.kron(L, D)
    Gz = (2.0 / dz) * np.kron(D, L)
    S = np.kron(L, L)
    w2D = ((w[:, None] * w[None, :]) * J).reshape(-1)
    return Gx, Gz, S, w2D


def lumped_mass(conn, dx, dz, npol, npoints):
    w = gll_weights(gll_points(npol))
    J = (dx / 2.0) * (dz / 2.0)
    wl = (w[None, :] * w[:, None]).reshape(-1) * J   # local index j*(N+1)+i -> w_i w_j J
    M = np.zeros(npoints)
    np.add.at(M, conn.reshape(-1), np.tile(wl, conn.shape[0]))
    return M


def stiffness_csr(c, conn, Gx, Gz, S, w2D, npoints):
    """Assembled K = sum_e Gx^T diag(w2D S c^2) Gx + Gz^T diag(...) Gz  as torch CSR."""
    c2 = c[conn] ** 2                                # (E, ng)
    wc = w2D[None, :] * (c2 @ S.T)                   # (E, ng)
    Ke = np.einsum("qa,eq,qb->eab", Gx, wc, Gx) + np.einsum("qa,eq,qb->eab", Gz, wc, Gz)
    ng = conn.shape[1]
    rows = np.repeat(conn, ng, axis=1).reshape(-1)
    cols = np.tile(conn, (1, ng)).reshape(-1)
    K = sp.coo_matrix((Ke.reshape(-1), (rows, cols)), shape=(npoints, npoints)).tocsr()
    K.sum_duplicates()
    return torch.sparse_csr_tensor(torch.from_numpy(K.indptr.astype(np.int64)),
                                   torch.from_numpy(K.indices.astype(np.int64)),
                                   torch.from_numpy(K.data), size=K.shape,
                                   dtype=torch.float64)


# --------------------------------------------------------------------------------------
# sponge, wavelet, receivers
# --------------------------------------------------------------------------------------


def sponge_decay(xmin, xmax, zmin, zmax, thickness, coords, dt, c_max, R=1e-8):
    """boundary.py:5-58: sigma = d0 ((delta-dist)/delta)^3 per side, summed x+z,
    d0 = -(m+1) c_max ln R / (2 delta), decay = exp(-sigma dt)."""
    m = 3
    d = float(thickness)
    d0 = -(m + 1) * float(c_max) * np.log(R) / (2.0 * d)
    x, z = coords[:, 0], coords[:, 1]
    sx = np.zeros(len(coords))
    sz = np.zeros(len(coords))
    left, right = x < xmin + d, x > xmax - d
    bot, top = z < zmin + d, z > zmax - d
    sx[left] = d0 * ((xmin + d - x[left]) / d) ** m
    sx[right] = d0 * ((x[right] - (xmax - d)) / d) ** m
    sz[bot] = d0 * ((zmin + d - z[bot]) / d) ** m
    sz[top] = d0 * ((z[top] - (zmax - d)) / d) ** m
    sig = sx + sz
    return np.exp(-sig * dt), sig > 0.0


def ricker_source(nt, dt, f0, amp, t0=0.1, gate=0.3):
    """sources.py:3-21: Ricker, minus its trapezoid mean, zero for t >= gate."""
    t = np.arange(nt) * dt
    a = (np.pi * f0 * (t - t0)) ** 2
    s = (1.0 - 2.0 * a) * np.exp(-a) * amp
    if nt > 1:
        s = s - np.trapezoid(s, t) / (t[-1] - t[0])
    s[~(t < gate)] = 0.0
    return s


def receiver_matrix(positions, xmin, zmin, dx, dz, nelx, nelz, conn, npol, npoints):
    """Lagrange interpolation rows (receivers.py:6-80 / layered core.py:90-172):
    element = clamp(int((x-xmin)/dx)), weights l_i(xi) l_j(eta)."""
    nodes = gll_points(npol)
    ng = npol + 1
    rows, cols, vals = [], [], []
    for r, (rx, rz) in enumerate(positions):
        ex = min(max(int((rx - xmin) / dx), 0), nelx - 1)
        ez = min(max(int((rz - zmin) / dz), 0), nelz - 1)
        e = ez * nelx + ex
        xi = 2.0 * (rx - (xmin + ex * dx)) / dx - 1.0
        eta = 2.0 * (rz - (zmin + ez * dz)) / dz - 1.0
        for j in range(ng):
            lz = lagrange_basis(eta, j, nodes)
            for i in range(ng):
                rows.append(r)
                cols.append(int(conn[e][j * ng + i]))
                vals.append(float(lagrange_basis(xi, i, nodes) * lz))
    R = sp.csr_matrix((vals, (rows, cols)), shape=(len(positions), npoints))
    R.sum_duplicates()
    R.eliminate_zeros()
    return R


def circle_receivers(src_x, src_z, radius, n):
    ang = np.linspace(0, 2 * np.pi, n, endpoint=False)
    return np.stack([src_x + radius * np.cos(ang), src_z + radius * np.sin(ang)], axis=1)


def align_observation(y, src_dt, src_nt, dst_dt, dst_nt):
    """core.py:109-128: linear resampling onto the simulation grid, zero outside."""
    y = np.asarray(y, dtype=np.float64)
    src_t = np.arange(src_nt, dtype=np.float64) * float(src_dt)
    dst_t = np.arange(dst_nt, dtype=np.float64) * float(dst_dt)
    if y.shape[0] > src_nt:
        y = y[:src_nt]
    if y.shape[0] == dst_nt and np.allclose(src_t[:dst_nt], dst_t, atol=1e-12, rtol=0.0):
        return y
    out = np.zeros((dst_nt, y.shape[1]))
    for r in range(y.shape[1]):
        out[:, r] = np.interp(dst_t, src_t, y[:, r], left=0.0, right=0.0)
        # interp1d(bounds_error=False, fill_value=0) is exact at the end points too
        out[(dst_t < src_t[0]) | (dst_t > src_t[-1]), r] = 0.0
    return out


# --------------------------------------------------------------------------------------
# simulation object
# --------------------------------------------------------------------------------------


@dataclass
class OracleSim:
    """Everything the time loops need, built from a reference-style config dict and
    a nodal velocity (reference node order)."""

    xmin: float
    xmax: float
    zmin: float
    zmax: float
    nelx: int
    nelz: int
    npol: int
    coords: np.ndarray
    conn: np.ndarray
    grid: np.ndarray
    dx: float
    dz: float
    dt: float
    nt: int
    src_node: int
    src: np.ndarray
    R: sp.csr_matrix
    M: np.ndarray
    decay: np.ndarray
    pml_mask: np.ndarray
    ops: tuple
    velocity: np.ndarray
    extra: dict = field(default_factory=dict)

    @property
    def npoints(self):
        return len(self.coords)


def build_sim(config: dict, velocity: np.ndarray | None = None, dt_cfl_velocity=None,
              dt: float | None = None) -> OracleSim:
    """Set up a simulation from a reference-style config dict.  ``dt`` pins the step
    (the reference keeps lowering ``sim.dt`` across calls, ``core.py:375-378``)."""
    d = config["domain"]
    xmin, xmax = float(d["xmin"]), float(d["xmax"])
    zmin, zmax = float(d["zmin"]), float(d["zmax"])
    nelx, nelz = int(d["nelem_x"]), int(d["nelem_z"])
    npol = int(config["method"]["polynomial_order"])
    coords, conn, grid = create_global_mesh(xmin, xmax, zmin, zmax, nelx, nelz, npol)
    dx = (xmax - xmin) / nelx
    dz = (zmax - zmin) / nelz
    vmax_cfg = config["velocity"].get("outside_velocity", config["velocity"].get("vmax", 3000.0))
    if velocity is None:
        velocity = np.full(len(coords), float(vmax_cfg))
    velocity = np.asarray(velocity, dtype=np.float64)
    T = float(config["time"]["total_time"])
    dt0 = float(config["time"]["dt"]) if dt is None else float(dt)
    dt, nt = cfl_dt(velocity if dt_cfl_velocity is None else dt_cfl_velocity, dt0, T, npol, dx, dz)
    if "nt_override" in config["time"]:
        nt = int(config["time"]["nt_override"])
    s = config["source"]
    src_x, src_z = [float(v) for v in s["position"]]
    src = ricker_source(nt, dt, float(s["frequency"]), float(s["amplitude"]))
    src_node = find_closest_node(src_x, src_z, coords)
    rc = config["receivers"]
    if "positions" in rc:
        pos = np.asarray(rc["positions"], dtype=np.float64)
    else:
        pos = circle_receivers(src_x, src_z, float(rc["radius"]), int(rc["num_receivers"]))
    R = receiver_matrix(pos, xmin, zmin, dx, dz, nelx, nelz, conn, npol, len(coords))
    M = lumped_mass(conn, dx, dz, npol, len(coords))
    mode = config["method"].get("boundary", "sponge")
    extra = {"boundary": mode}
    if mode == "sponge":
        decay, mask = sponge_decay(xmin, xmax, zmin, zmax, float(config["method"]["pml_thickness"]),
                                   coords, dt, float(vmax_cfg))
    elif mode == "stacey":
        decay, mask = np.ones(len(coords)), np.zeros(len(coords), dtype=bool)
        beta, top = stacey_weights(grid, nelx, nelz, npol, dx, dz)
        extra.update(beta=beta, top=top)
    else:
        raise ValueError(f"unknown boundary mode {mode!r}")
    ops = sem_operators(dx, dz, npol)
    return OracleSim(xmin, xmax, zmin, zmax, nelx, nelz, npol, coords, conn, grid, dx, dz, dt, nt,
                     src_node, src, R, M, decay, mask, ops, velocity, extra)


def stacey_weights(grid, nelx, nelz, npol, dx, dz):
    """Boundary quadrature weight of every node on the absorbing edges (x = xmin, x = xmax,
    z = zmax): the sum over its element edges of the 1-D GLL weight times the edge
    half-length; and the top-row (z = zmin, free surface) mask.  Reference node order."""
    w = gll_weights(gll_points(npol))
    N = npol
    nxg, nzg = nelx * N + 1, nelz * N + 1
    gx, gz = grid[:, 0], grid[:, 1]
    bx = np.zeros(nxg)   # along the bottom edge, by column
    bz = np.zeros(nzg)   # along the side edges, by row
    for e in range(nelx):
        bx[e * N:(e + 1) * N + 1] += w * (dx / 2.0)
    for e in range(nelz):
        bz[e * N:(e + 1) * N + 1] += w * (dz / 2.0)
    beta = np.zeros(len(grid))
    side = (gx == 0) | (gx == nxg - 1)
    beta[side] += bz[gz[side]]
    bot = gz == nzg - 1
    beta[bot] += bx[gx[bot]]
    return beta, gz == 0


def _torch_csr(R: sp.csr_matrix, device="cpu"):
    return torch.sparse_csr_tensor(torch.from_numpy(R.indptr.astype(np.int64)),
                                   torch.from_numpy(R.indices.astype(np.int64)),
                                   torch.from_numpy(R.data.astype(np.float64)), size=R.shape,
                                   dtype=torch.float64).to(device)


def _stacey_terms(sim: OracleSim, c, device):
    """(a, top mask, beta) of the Stacey / free-surface mode, or None for the sponge."""
    if sim.extra.get("boundary", "sponge") != "stacey":
        return None
    beta = sim.extra["beta"]
    a = 0.5 * sim.dt * np.asarray(c, dtype=np.float64) * beta / sim.M
    return (torch.from_numpy(a).to(device), torch.from_numpy(sim.extra["top"]).to(device),
            torch.from_numpy(beta).to(device))


def _stacey_step(st, u, u_prev, f):
    """(1 + a) u+ = 2 u - (1 - a) u- + f, then u+ = 0 on the free surface."""
    a, top, _ = st
    u_next = (2.0 * u - (1.0 - a) * u_prev + f) / (1.0 + a)
    u_next[top] = 0.0
    return u_next


def forward(sim: OracleSim, velocity=None, convention: str = "run", keep_history: bool = False,
            device="cpu"):
    """Forward time loop.

    convention='run'     : rec[it] = R u_curr recorded before the update (core.py:632-639)
    convention='fwdadj'  : rec[it] = R u_curr after update and sponge (core.py:1197-1219)
    Returns rec (nt, nrec) and optionally the post-update history (nt, P)."""
    c = sim.velocity if velocity is None else np.asarray(velocity, dtype=np.float64)
    Gx, Gz, S, w2D = sim.ops
    K = stiffness_csr(c, sim.conn, Gx, Gz, S, w2D, sim.npoints).to(device)
    R = _torch_csr(sim.R, device)
    P = sim.npoints
    Minv = torch.from_numpy(1.0 / sim.M).to(device)
    Msrc = float(sim.M[sim.src_node])
    dt2 = sim.dt * sim.dt
    idx = torch.from_numpy(np.nonzero(sim.pml_mask)[0]).to(device)
    dec = torch.from_numpy(sim.decay).to(device)[idx]
    src = torch.from_numpy(sim.src).to(device)
    u_prev = torch.zeros(P, dtype=torch.float64, device=device)
    u_curr = torch.zeros(P, dtype=torch.float64, device=device)
    rec = torch.zeros((sim.nt, R.shape[0]), dtype=torch.float64, device=device)
    hist = torch.zeros((sim.nt, P), dtype=torch.float64, device=device) if keep_history else None
    sn = sim.src_node
    st = _stacey_terms(sim, c, device)
    for it in range(sim.nt):
        rhs = -torch.matmul(K, u_curr)
        rhs[sn] += src[it] * Msrc
        if st is None:
            u_next = 2.0 * u_curr - u_prev + dt2 * (Minv * rhs)
        else:
            u_next = _stacey_step(st, u_curr, u_prev, dt2 * (Minv * rhs))
        if convention == "run":
            rec[it] = torch.matmul(R, u_curr)
        if len(idx):
            u_curr[idx] *= dec
            u_next[idx] *= dec
        u_prev, u_curr = u_curr, u_next
        if convention == "fwdadj":
            rec[it] = torch.matmul(R, u_curr)
        if keep_history:
            hist[it] = u_curr
    return rec.cpu().numpy(), (hist if keep_history else None)


def sensitivity_step(u, lam, conn_t, Gx_t, Gz_t, S_t, w2D_t, npoints):
    """core.py:49-85 without the final 2c factor (applied once after the time sum):
    returns S^T (w2D (Gx u . Gx lam + Gz u . Gz lam)) scattered to the nodes."""
    E, ng = conn_t.shape
    gi = conn_t.reshape(-1)
    ul = u.index_select(0, gi).reshape(E, ng)
    ll = lam.index_select(0, gi).reshape(E, ng)
    ux = ul @ Gx_t.T
    uz = ul @ Gz_t.T
    lx = ll @ Gx_t.T
    lz = ll @ Gz_t.T
    gq = w2D_t * (ux * lx + uz * lz)
    loc = gq @ S_t
    out = torch.zeros(npoints, dtype=torch.float64, device=u.device)
    out.scatter_add_(0, gi, loc.reshape(-1))
    return out


def forward_adjoint(sim: OracleSim, y_obs_aligned: np.ndarray, sigma: float,
                    velocity=None, mode: str = "reference", window=None, device="cpu"):
    """run_forward_and_adjoint (core.py:1067-1278) on a given nodal velocity.

    Returns dict(loglik, clean (nt,nrec), dJ_dv (P,) = reference's ``dJ_dv``,
    dL_dv = -dJ_dv).  ``mode='exact'`` applies the sponge in the adjoint too.
    ``window=(it0, it1, decim)`` restates the CO2 misfit window
    (CO2_plume/one_stage/single_cubic/sem_waveform/core.py:1441-1552)."""
    c = sim.velocity if velocity is None else np.asarray(velocity, dtype=np.float64)
    Gx, Gz, S, w2D = sim.ops
    K = stiffness_csr(c, sim.conn, Gx, Gz, S, w2D, sim.npoints).to(device)
    R = _torch_csr(sim.R, device)
    RT = _torch_csr(sim.R.T.tocsr(), device)
    P = sim.npoints
    nt = sim.nt
    Minv = torch.from_numpy(1.0 / (sim.M + 1e-30)).to(device)
    Msrc = float(sim.M[sim.src_node])
    dt2 = sim.dt * sim.dt
    idx = torch.from_numpy(np.nonzero(sim.pml_mask)[0]).to(device)
    dec = torch.from_numpy(sim.decay).to(device)[idx]
    src = torch.from_numpy(sim.src).to(device)
    it0, it1, decim = (0, nt, 1) if window is None else window
    nt_eff = it1 - it0
    u_prev = torch.zeros(P, dtype=torch.float64, device=device)
    u_curr = torch.zeros(P, dtype=torch.float64, device=device)
    hist = torch.zeros((nt_eff, P), dtype=torch.float64, device=device)
    sn = sim.src_node
    st = _stacey_terms(sim, c, device)
    if st is not None and (it0, it1, decim) != (0, nt, 1):
        raise ValueError("the Stacey boundary mode supports the full misfit window only")
    for it in range(nt):
        rhs = -torch.matmul(K, u_curr)
        rhs[sn] += src[it] * Msrc
        if st is None:
            u_next = 2.0 * u_curr - u_prev + dt2 * (Minv * rhs)
        else:
            u_next = _stacey_step(st, u_curr, u_prev, dt2 * (Minv * rhs))
        if len(idx):
            u_curr[idx] *= dec
            u_next[idx] *= dec
        u_prev, u_curr = u_curr, u_next
        if it0 <= it < it1:
            hist[it - it0] = u_curr
    d_syn = torch.stack([torch.matmul(R, hist[i]) for i in range(nt_eff)]).cpu().numpy() \
        if device != "cpu" else torch.matmul(R, hist.T).T.numpy()
    d_dec = d_syn[::decim]
    y = np.asarray(y_obs_aligned, dtype=np.float64)
    resid_dec = d_dec - y
    resid = np.zeros_like(d_syn)
    resid[::decim] = resid_dec
    sigma2 = float(sigma) ** 2 + 1e-24
    loglik = -0.5 * float(np.sum(resid_dec * resid_dec)) / sigma2
    rs = (torch.from_numpy(resid.T.copy()) * (1.0 / sigma2)).to(device)
    conn_t = torch.from_numpy(sim.conn).to(device)
    Gx_t, Gz_t, S_t, w2D_t = (torch.from_numpy(a).to(device) for a in (Gx, Gz, S, w2D))
    lam_n = torch.zeros(P, dtype=torch.float64, device=device)
    lam_c = torch.zeros(P, dtype=torch.float64, device=device)
    acc = torch.zeros(P, dtype=torch.float64, device=device)
    if st is not None:
        # boundary-impedance term per c^2: beta / (4 dt c) lambda (u(t+1) - u(t-1))
        bfac = st[2] / (4.0 * sim.dt * torch.from_numpy(np.asarray(c, dtype=np.float64)).to(device))
    for it in range(nt_eff - 1, -1, -1):
        rhs = torch.matmul(RT, rs[:, it]) - torch.matmul(K, lam_c)
        if st is None:
            lam_p = 2.0 * lam_c - lam_n + dt2 * (Minv * rhs)
        else:
            lam_p = _stacey_step(st, lam_c, lam_n, dt2 * (Minv * rhs))
        acc += sensitivity_step(hist[it], lam_c, conn_t, Gx_t, Gz_t, S_t, w2D_t, P)
        if st is not None and it + 1 < nt_eff:
            u_lo = hist[it - 1] if it >= 1 else torch.zeros_like(lam_c)
            acc += bfac * lam_c * (hist[it + 1] - u_lo)
        if mode == "exact" and len(idx):
            lam_c[idx] *= dec
            lam_p[idx] *= dec
        lam_n, lam_c = lam_c, lam_p
    dJ = (2.0 * torch.from_numpy(c) * acc.cpu()).numpy()
    return {"loglik": loglik, "clean": d_syn, "dJ_dv": dJ, "dL_dv": -dJ, "resid": resid}


def misfit_loglik(sim: OracleSim, velocity, y_obs_aligned, sigma, convention="fwdadj", device="cpu"):
    """-0.5 |d(c) - y|^2 / sigma^2 with d from the chosen receiver convention."""
    rec, _ = forward(sim, velocity, convention=convention, device=device)
    r = rec - y_obs_aligned
    return -0.5 * float(np.sum(r * r)) / (float(sigma) ** 2 + 1e-24)
