"""Dense receiver lines: more receivers in one element row of one strip than the strip
kernel reads out in one pass (128 threads) or stages at once for the adjoint source (61 at
order 4, 35 at order 7, 203 at order 1), on a surface line and on a line at depth.  The
strip kernel must equal the tile kernel bitwise (seismograms, gradient, log-likelihood)
and both must match the float64 oracle within 1e-4."""
import numpy as np
import pytest
import torch

from mun_b200 import Batch, SEMPlan, SolveSpec
from oracle import sem_oracle as so

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("N,nelx,nsurf,ndeep", [(4, 30, 150, 80), (7, 16, 100, 60), (1, 60, 230, 40)])
def test_dense_receiver_lines_strip_equals_tile_and_oracle(N, nelx, nsurf, ndeep):
    nelz, xmax, zmax = 8, 600.0, 160.0
    h = zmax / nelz
    # a surface line inside element row 0 and a line inside element row 3, both dense
    rec = np.concatenate([np.stack([np.linspace(3.0, xmax - 3.0, nsurf), np.full(nsurf, 0.4 * h)], 1),
                          np.stack([np.linspace(7.0, xmax - 7.0, ndeep), np.full(ndeep, 3.6 * h)], 1)])
    cfg = {"domain": {"xmin": 0.0, "xmax": xmax, "zmin": 0.0, "zmax": zmax, "nelem_x": nelx, "nelem_z": nelz},
           "time": {"total_time": 1.0, "dt": 1.0},
           "source": {"position": (0.5 * xmax, 0.5 * zmax), "frequency": 25.0, "amplitude": 1.0},
           "receivers": {"positions": rec},
           "method": {"polynomial_order": N, "pml_thickness": 60.0},
           "velocity": {"outside_velocity": 2600.0}}
    sim0 = so.build_sim(cfg)
    x, z = sim0.coords[:, 0], sim0.coords[:, 1]
    v = 2000.0 + 250.0 * np.sin(x / 70.0) * np.cos(z / 40.0)
    v_obs = v + 80.0 * np.exp(-((x - 0.4 * xmax) ** 2 + (z - 0.6 * zmax) ** 2) / 2e3)
    sim = so.build_sim(cfg, v, dt_cfl_velocity=np.full(len(v), 2600.0))
    nt = 300
    sim.nt = nt
    sim.src = so.ricker_source(nt, sim.dt, 25.0, 1.0)
    y, _ = so.forward(sim, v_obs, convention="fwdadj")
    sigma = 1e-4
    ref = so.forward_adjoint(sim, y, sigma)

    plan = SEMPlan(xmin=0.0, xmax=xmax, zmin=0.0, zmax=zmax, nelx=nelx, nelz=nelz, npol=N, dt=sim.dt, nt=nt,
                   src_xz=(0.5 * xmax, 0.5 * zmax), f0=25.0, amp=1.0, receivers=rec, pml_thickness=60.0,
                   sponge_cmax=2600.0)
    dv = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device="cuda")  # noqa: E731
    out = {}
    for kernel in (1, 2):
        s = SolveSpec(plan, dv(v), adjoint=True, y_obs=dv(y), inv_sigma2=1.0 / (sigma ** 2 + 1e-24))
        b = Batch(kernel=kernel)
        b.run([s])
        torch.cuda.synchronize()
        assert b.last_kernel == {1: "tile", 2: "strip"}[kernel]
        assert int(s.status.item()) == 0
        out[kernel] = s
    t, st = out[1], out[2]
    assert torch.equal(st.rec, t.rec) and torch.equal(st.grad, t.grad) and torch.equal(st.loglik, t.loglik)
    e_c = _rel(st.rec.cpu().numpy().astype(np.float64), ref["clean"])
    e_g = _rel(-st.grad.cpu().numpy(), ref["dL_dv"])
    e_l = abs(float(st.loglik.item()) - ref["loglik"]) / abs(ref["loglik"])
    print(f"N={N}: {len(rec)} receivers, seismogram {e_c:.2e}, gradient {e_g:.2e}, loglik {e_l:.2e}")
    assert e_c <= TOL and e_g <= TOL and e_l <= TOL
