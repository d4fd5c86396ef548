"""Float64 NumPy model of the arithmetic the CUDA tick kernel performs, built only from
the plan tables (``mun_b200.plan.build_plan_arrays``).  Tests compare it with the
oracle's assembled CSR operators; this checks the 1-D operator split on the CPU."""
import numpy as np


def grids(a):
    N = a["npol"]
    return a["nelx"] * N + 1, a["nelz"] * N + 1


def to_grid(a, v):
    nxg, nzg = grids(a)
    g = np.zeros(nxg * nzg)
    g[a["node_grid"]] = v
    return g.reshape(nzg, nxg)


def from_grid(a, g):
    return g.reshape(-1)[a["node_grid"]]


def _lines(u, c2, N, D, beta, axis):
    """sum over elements on each grid line of D^T (beta c2 (D u_e)); optionally with a
    second field for the sensitivity beta (D u)(D w)."""
    if axis == 0:
        u, c2 = u.T, c2.T
    nl, nn = u.shape
    nel = (nn - 1) // N
    out = np.zeros_like(u)
    for e in range(nel):
        sl = slice(e * N, e * N + N + 1)
        du = u[:, sl] @ D.T
        out[:, sl] += (beta[None, :] * c2[:, sl] * du) @ D
    return out.T if axis == 0 else out


def _sens(u, w, N, D, beta, axis):
    if axis == 0:
        u, w = u.T, w.T
    nn = u.shape[1]
    nel = (nn - 1) // N
    out = np.zeros_like(u)
    for e in range(nel):
        sl = slice(e * N, e * N + N + 1)
        out[:, sl] += beta[None, :] * (u[:, sl] @ D.T) * (w[:, sl] @ D.T)
    return out.T if axis == 0 else out


def tables(a):
    nxg, nzg = grids(a)
    tx, tz = a["tab_x"], a["tab_z"]
    return (tx[:nxg], tx[nxg:2 * nxg], tx[2 * nxg:], tz[:nzg], tz[nzg:2 * nzg], tz[2 * nzg:])


def K_apply(a, c, ug):
    """K u on the grid (c in reference order)."""
    N, D, beta = a["npol"], a["gll_D"], a["gll_beta"]
    ix, Rx, dx, iz, Rz, dz = tables(a)
    c2 = to_grid(a, c) ** 2
    X = _lines(ug, c2, N, D, beta, 1)
    Z = _lines(ug, c2, N, D, beta, 0)
    return Rz[:, None] * X + Rx[None, :] * Z


def mass_inv_dt2(a):
    ix, Rx, dx, iz, Rz, dz = tables(a)
    return iz[:, None] * ix[None, :]


def sens_apply(a, ug, wg):
    N, D, beta = a["npol"], a["gll_D"], a["gll_beta"]
    ix, Rx, dx, iz, Rz, dz = tables(a)
    return Rz[:, None] * _sens(ug, wg, N, D, beta, 1) + Rx[None, :] * _sens(ug, wg, N, D, beta, 0)


def stacey_weights(a, c):
    """Per-node (e1, e2) of the Stacey mode's update w = e1 v + e2 F on the grid: a = c alpha
    on the absorbing edges' slots, e1 = (1 - a) / (1 + a), e2 = 1 / (1 + a); 1 elsewhere."""
    nxg, nzg = grids(a)
    e1, e2 = np.ones((nzg, nxg)), np.ones((nzg, nxg))
    from mun_b200.plan import boundary_slots
    _, gx, gz, _ = boundary_slots(a["nelx"], a["nelz"], a["npol"])
    ref = a["bnd_ref"]
    k = np.nonzero(ref >= 0)[0]
    av = np.asarray(c, dtype=np.float64)[ref[k]] * a["bnd_alpha"][k]
    e1[gz[k], gx[k]] = (1.0 - av) / (1.0 + av)
    e2[gz[k], gx[k]] = 1.0 / (1.0 + av)
    return e1, e2


def forward(a, c, shift=False):
    """(b, v) forward recurrence exactly as the kernel runs it (float64).  Sponge mode:
    v, b <- d w, d (b + w) with w = v + F; Stacey mode: w = e1 v + e2 F, v, b <- w, b + w,
    and both zero on the free surface (top grid row)."""
    ix, Rx, dx, iz, Rz, dz = tables(a)
    d = (1.0 - dz)[:, None] * (1.0 - dx)[None, :]   # the tables carry the decay defects
    P = mass_inv_dt2(a)
    nxg, nzg = grids(a)
    stacey = a.get("boundary") == "stacey"
    if stacey:
        e1, e2 = stacey_weights(a, c)
    v = np.zeros((nzg, nxg))
    cur = np.zeros((nzg, nxg))
    N = a["npol"]
    nrec = a["nrec"]
    rec = np.zeros((a["nt"], nrec))
    ng = N + 1

    def read(g):
        out = np.zeros(nrec)
        for r in range(nrec):
            bx, bz = a["rec_base"][r]
            out[r] = np.sum(a["rec_w"][r].reshape(ng, ng) * g[bz:bz + ng, bx:bx + ng])
        return out

    hist = []
    for t in range(a["nt"]):
        if not shift:
            rec[t] = read(cur)
        F = -P * K_apply(a, c, cur)
        F[a["src_gz"], a["src_gx"]] += a["src_term"][t]
        if stacey:
            w = e1 * v + e2 * F
            v, cur = w, cur + w
            v[0], cur[0] = 0.0, 0.0
        else:
            w = v + F
            v, cur = d * w, d * (cur + w)
        hist.append(cur)
        if shift:
            rec[t] = read(cur)
    return rec, hist
