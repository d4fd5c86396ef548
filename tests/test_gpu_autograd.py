"""Gradients through torch.autograd for a batch of tensor B-spline node vectors,
checked against central finite differences of the float64 oracle along 5 random
node directions (exact discrete adjoint) and against the oracle's adjoint gradient."""
import numpy as np
import pytest
import torch

from mun_b200 import SEMPlan
from mun_b200.autograd import GridLikelihood, GridModel
from mun_b200.bspline import grid_basis, layered_velocity
from mun_b200.mesh import create_global_mesh
from oracle import sem_oracle as so

pytestmark = pytest.mark.gpu


def _setup():
    xmin, xmax, zmin, zmax, nelx, nelz, N = 0.0, 1500.0, 0.0, 800.0, 30, 16, 4
    coords, _, node_grid = create_global_mesh(xmin, xmax, zmin, zmax, nelx, nelz, N)
    base = layered_velocity(coords[:, 1], [300.0, 550.0], [1500.0, 2200.0, 3000.0])
    rec = np.stack([np.linspace(250.0, 1250.0, 21), np.full(21, 230.0)], 1)
    nt = 500
    dt = 0.35 * (50.0 / 5) / (3400.0 * 5 * np.sqrt(2.0))
    kw = dict(xmin=xmin, xmax=xmax, zmin=zmin, zmax=zmax, nelx=nelx, nelz=nelz, npol=N, dt=dt, nt=nt,
              src_xz=(750.0, 260.0), f0=15.0, amp=1.0, receivers=rec, pml_thickness=150.0,
              sponge_cmax=3000.0)
    cfg = {"domain": {"xmin": xmin, "xmax": xmax, "zmin": zmin, "zmax": zmax, "nelem_x": nelx,
                      "nelem_z": nelz},
           "time": {"total_time": (nt - 0.5) * dt, "dt": dt},
           "source": {"position": (750.0, 260.0), "frequency": 15.0, "amplitude": 1.0},
           "receivers": {"positions": rec}, "method": {"polynomial_order": N, "pml_thickness": 150.0},
           "velocity": {"outside_velocity": 3000.0}}
    return kw, cfg, coords, base


def test_grid_likelihood_gradients_vs_finite_differences():
    kw, cfg, coords, base = _setup()
    plan = SEMPlan(**kw)
    model = GridModel(plan, coords, base, ((0.0, 1500.0), (0.0, 800.0)), 10, 6)
    Bm = grid_basis(coords, (0.0, 1500.0), (0.0, 800.0), 10, 6)
    rng = np.random.default_rng(5)
    theta_true = rng.normal(0, 100.0, 60)
    thetas = np.stack([rng.normal(0, 100.0, 60) for _ in range(3)])
    sigma = 1e-3
    sim = so.build_sim(cfg, base + Bm @ theta_true, dt=kw["dt"])
    assert sim.nt == kw["nt"]
    y, _ = so.forward(sim, base + Bm @ theta_true, convention="fwdadj")
    th = torch.tensor(thetas, device="cuda", requires_grad=True)
    ll = GridLikelihood.apply(th, model, torch.as_tensor(y, device="cuda"), sigma, True)
    ll.sum().backward()
    g = th.grad.cpu().numpy()
    for b in range(len(thetas)):
        v = base + Bm @ thetas[b]
        ref = so.forward_adjoint(sim, y, sigma, velocity=v, mode="exact")
        # oracle gradient in theta space: B^T (d loglik / d v) = -B^T dL_dv
        g_ref = -(Bm.T @ ref["dL_dv"])
        e = np.linalg.norm(g[b] - g_ref) / np.linalg.norm(g_ref)
        e_ll = abs(float(ll[b]) - ref["loglik"]) / abs(ref["loglik"])
        print(f"sample {b}: theta-gradient vs fp64 exact adjoint {e:.2e}, loglik {e_ll:.2e}")
        assert e <= 1e-4 and e_ll <= 1e-4
    # central differences of the float64 oracle along 5 random unit directions
    drng = np.random.default_rng(0)
    eps = 0.5
    for k in range(5):
        d = drng.standard_normal(60)
        d /= np.linalg.norm(d)
        lp = so.misfit_loglik(sim, base + Bm @ (thetas[0] + eps * d), y, sigma)
        lm = so.misfit_loglik(sim, base + Bm @ (thetas[0] - eps * d), y, sigma)
        fd = (lp - lm) / (2 * eps)
        ad = float(g[0] @ d)
        print(f"direction {k}: adjoint {ad:.6e} FD {fd:.6e} rel {abs(ad - fd) / abs(fd):.2e}")
        assert abs(ad - fd) <= 1e-3 * abs(fd)
