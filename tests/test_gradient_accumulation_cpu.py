"""The kernels accumulate the sensitivity in float32 (one __fadd_rn per node and adjoint
tick).  This checks the numerical argument on the CPU: the float64 oracle's per-tick
node increments, rounded to float32 as the kernels form them and summed in float32, stay
within a few 1e-7 of float64 accumulation of the same increments (the parity tolerance
is 1e-4, the float32 wavefield's own error about 1e-5)."""
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
    for it in range(nt - 1, -1, -1):
        rhs = torch.matmul(RT, rs[:, it]) - torch.matmul(K, lam_c)
        lam_p = 2.0 * lam_c - lam_n + dt2 * (Minv * rhs)
        inc32 = (sensitivity_step(hist[it], lam_c, conn_t, Gx_t, Gz_t, S_t, w2D_t, P) * scale).float()
        acc64 += inc32.double()
        acc32 += inc32
        lam_n, lam_c = lam_c, lam_p
    return acc64.numpy(), acc32.double().numpy()


@pytest.mark.parametrize("name", ["inject_n1", "inject_n3"])
def test_float32_accumulation_error_is_negligible(name):
    a64, a32 = _accumulations(name)
    rel = float(np.linalg.norm(a32 - a64) / np.linalg.norm(a64))
    print(f"{name}: float32 vs float64 accumulation of the same increments {rel:.2e}")
    assert rel < 2e-6
