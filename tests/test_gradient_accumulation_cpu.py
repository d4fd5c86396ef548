"""The kernels sum the sensitivity over the adjoint ticks in float64: each tick's node
increment (float32, as the kernels form it) is added to a float32 partial sum, which is
folded into a float64 accumulator on the ticks with (t - it0) % 16 == 0; a partial
starts from zero after each fold and on the first gradient tick.  This checks the
numerical argument on the CPU with the float64 oracle's increments: the folded sum stays
within a few 1e-8 of float64 accumulation of the same increments (relative L2), and
within a few 1e-6 node by node on the nodes that carry the gradient (the parity tolerance is 1e-4, the float32 wavefield's
own error about 1e-5).  A plain float32 running sum is shown beside it for scale."""
import numpy as np
import pytest
import torch

from oracle import sem_oracle as so
from oracle.sem_oracle import _torch_csr, sensitivity_step, stiffness_csr
from tests.goldens import load
from tests.gpu_cases import aligned_obs


def _accumulations(name):
    g = load(name)
    sim = so.build_sim(g["config"], g["velocity"], dt=float(g["dt"]))
    sim.nt = int(g["nt"])
    y = aligned_obs(g)
    c = sim.velocity
    Gx, Gz, S, w2D = sim.ops
    K = stiffness_csr(c, sim.conn, Gx, Gz, S, w2D, sim.npoints)
    R = _torch_csr(sim.R)
    RT = _torch_csr(sim.R.T.tocsr())
    P, nt = sim.npoints, sim.nt
    Minv = torch.from_numpy(1.0 / (sim.M + 1e-30))
    Msrc = float(sim.M[sim.src_node])
    dt2 = sim.dt ** 2
    idx = torch.from_numpy(np.nonzero(sim.pml_mask)[0])
    dec = torch.from_numpy(sim.decay)[idx]
    src = torch.from_numpy(sim.src)
    u_prev = torch.zeros(P, dtype=torch.float64)
    u_curr = torch.zeros(P, dtype=torch.float64)
    hist = torch.zeros((nt, P), dtype=torch.float64)
    for it in range(nt):
        rhs = -torch.matmul(K, u_curr)
        rhs[sim.src_node] += src[it] * Msrc
        u_next = 2.0 * u_curr - u_prev + dt2 * (Minv * rhs)
        if len(idx):
            u_curr[idx] *= dec
            u_next[idx] *= dec
        u_prev, u_curr = u_curr, u_next
        hist[it] = u_curr
    resid = torch.matmul(R, hist.T).T.numpy() - y
    sigma2 = float(g["sigma"]) ** 2 + 1e-24
    rs = torch.from_numpy(resid.T.copy()) * (1.0 / sigma2)
    # the kernels' power-of-two adjoint scale, so float32 increments stay in range
    m = float(np.abs(resid).max()) / sigma2
    scale = 2.0 ** (-np.floor(np.log2(m))) if m > 0 else 1.0
    conn_t = torch.from_numpy(sim.conn)
    Gx_t, Gz_t, S_t, w2D_t = (torch.from_numpy(a) for a in (Gx, Gz, S, w2D))
    lam_n = torch.zeros(P, dtype=torch.float64)
    lam_c = torch.zeros(P, dtype=torch.float64)
    acc64 = torch.zeros(P, dtype=torch.float64)
    acc32 = torch.zeros(P, dtype=torch.float32)
    fold64 = torch.zeros(P, dtype=torch.float64)
    part32 = torch.zeros(P, dtype=torch.float32)
    it0, it1 = 0, nt
    for it in range(nt - 1, -1, -1):
        rhs = torch.matmul(RT, rs[:, it]) - torch.matmul(K, lam_c)
        lam_p = 2.0 * lam_c - lam_n + dt2 * (Minv * rhs)
        inc32 = (sensitivity_step(hist[it], lam_c, conn_t, Gx_t, Gz_t, S_t, w2D_t, P) * scale).float()
        acc64 += inc32.double()
        acc32 += inc32
        if it == it1 - 1 or (it - it0) % FOLD == FOLD - 1:
            part32 = inc32.clone()
        else:
            part32 = part32 + inc32
        if (it - it0) % FOLD == 0:
            fold64 += part32.double()
            part32 = torch.zeros(P, dtype=torch.float32)
        lam_n, lam_c = lam_c, lam_p
    return acc64.numpy(), fold64.numpy(), acc32.double().numpy()


FOLD = 16


def _errors(ref, got):
    rel_l2 = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    # node by node, on the nodes carrying at least 1e-3 of the largest |gradient|
    big = np.abs(ref) >= 1e-3 * np.abs(ref).max()
    rel_node = float((np.abs(got - ref)[big] / np.abs(ref)[big]).max())
    return rel_l2, rel_node


@pytest.mark.parametrize("name", ["inject_n1", "inject_n3", "layered_cfg0"])
def test_folded_float64_accumulation_error_is_negligible(name):
    a64, fold, a32 = _accumulations(name)
    l2, node = _errors(a64, fold)
    l2_32, node_32 = _errors(a64, a32)
    print(f"{name}: folded float64 vs float64 accumulation rel. L2 {l2:.2e}, max per node {node:.2e} "
          f"(plain float32 running sum: {l2_32:.2e}, {node_32:.2e})")
    # per node the error is set by cancellation in a node's time-sum (increments of both
    # signs), which the plain float32 sum shows 2-8 times larger
    assert l2 < 1e-7 and node < 2e-5
    assert l2 < l2_32
