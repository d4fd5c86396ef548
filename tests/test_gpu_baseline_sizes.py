"""GPU parity at the full sizes of the benchmark workloads, against the float64 oracle.

The goldens pin the CUDA path on meshes of at most 48x28 elements and 2000 steps; these
tests run the benchmark's own workloads (``bench.workload``, ``bench.single_model``,
``bench.uneven_specs``) at their stated sizes:

* the batched ELBO step's mesh (100x50 elements, order 4, 3000 steps) with four of its
  tensor-spline models through the strip kernel, automatic checkpointing, against the
  oracle, and bitwise against the tile kernel and against explicit k = nt runs;
* the same mesh's 10x6 B-spline grid gradient through ``torch.autograd`` checked by
  central differences of the oracle's log-likelihood along 5 random directions;
* the single large solve (400x200 elements, 1.28 M nodes, 5000 steps, k = 250);
* a mixed batch of orders 3, 4 and 5 from the uneven workload's range.

The oracle is the float64 restatement of the reference path; at these sizes its time
loops run on torch's CUDA backend in float64 (the float64 forward history of the large
solve alone is 51 GB).  Tolerance: relative L2 <= 1e-4 (log-likelihood: relative).
"""
import numpy as np
import pytest
import torch

import bench
from mun_b200 import Batch, SEMPlan, SolveSpec
from oracle import sem_oracle as so
from tests.goldens import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _config(kw, nt, dt):
    """Reference-style config dict of a plan's keyword arguments (oracle input)."""
    return {"domain": {"xmin": kw["xmin"], "xmax": kw["xmax"], "zmin": kw["zmin"], "zmax": kw["zmax"],
                       "nelem_x": kw["nelx"], "nelem_z": kw["nelz"]},
            "time": {"total_time": (nt - 0.5) * dt, "dt": dt},
            "source": {"position": kw["src_xz"], "frequency": kw["f0"], "amplitude": kw["amp"]},
            "receivers": {"positions": kw["receivers"]},
            "method": {"polynomial_order": kw["npol"], "pml_thickness": kw["pml_thickness"]},
            "velocity": {"outside_velocity": kw["sponge_cmax"]}}


def _oracle_sim(kw, v, dt, nt, cfl_velocity=None):
    """Oracle simulation with the plan's dt and nt (the CFL rule sees ``cfl_velocity``,
    the model the benchmark took dt from, default ``v``)."""
    sim = so.build_sim(_config(kw, nt, dt), v, dt=dt, dt_cfl_velocity=cfl_velocity)
    assert sim.nt == nt and sim.dt == dt
    return sim


def _errors(s, ref):
    return (rel_l2(s.rec.cpu().numpy(), ref["clean"]), rel_l2(s.grad.cpu().numpy(), ref["dJ_dv"]),
            abs(float(s.loglik.item()) - ref["loglik"]) / abs(ref["loglik"]))


def test_elbo_mesh_batch_matches_fp64_oracle():
    W = bench.workload(nmodels=4)
    kw = W["plan_kw"]
    plan = SEMPlan(**kw)
    dt, nt, sigma = W["dt"], W["nt"], W["sigma"]
    sim = _oracle_sim(kw, W["v_true"], dt, nt)
    y, _ = so.forward(sim, W["v_true"], convention="fwdadj", device="cuda")
    yd = torch.as_tensor(y, device="cuda")
    inv_s2 = 1.0 / (sigma ** 2 + 1e-24)
    vd = torch.as_tensor(W["vels"], device="cuda")

    def specs(k):
        return [SolveSpec(plan, vd[i], adjoint=True, y_obs=yd, inv_sigma2=inv_s2, ckpt_k=k) for i in range(4)]
    auto = specs(0)
    b = Batch(kernel=2)
    b.run(auto)
    torch.cuda.synchronize()
    assert b.last_kernel == "strip"
    assert all(int(s.status.item()) == 0 for s in auto)
    # the whole forward kept (k = nt), two groups of two solves
    full = specs(nt)
    for half in (full[:2], full[2:]):
        Batch(kernel=2).run(half)
    tile = specs(0)
    Batch(kernel=1).run(tile)
    torch.cuda.synchronize()
    for a, f, t in zip(auto, full, tile):
        for o in ("rec", "grad", "loglik"):
            assert torch.equal(getattr(a, o), getattr(f, o)) and torch.equal(getattr(a, o), getattr(t, o))
    for i, s in enumerate(auto):
        ref = so.forward_adjoint(sim, y, sigma, velocity=W["vels"][i], device="cuda")
        e = _errors(s, ref)
        print(f"model {i}: seismogram {e[0]:.2e} gradient {e[1]:.2e} loglik {e[2]:.2e} "
              f"(vs fp64 oracle, 100x50 el, 3000 steps)")
        assert max(e) <= TOL, e


def test_elbo_mesh_grid_gradient_vs_finite_differences():
    from mun_b200.autograd import GridLikelihood, GridModel
    from mun_b200.bspline import grid_basis, layered_velocity
    W = bench.workload(nmodels=2)
    kw = W["plan_kw"]
    plan = SEMPlan(**kw)
    dt, nt, sigma = W["dt"], W["nt"], W["sigma"]
    coords = W["coords"]
    base = layered_velocity(coords[:, 1], [300.0, 650.0], [1500.0, 2200.0, 3000.0])
    model = GridModel(plan, coords, base, ((0.0, 2000.0), (0.0, 1000.0)), 10, 6)
    Bm = grid_basis(coords, (0.0, 2000.0), (0.0, 1000.0), 10, 6)
    sim = _oracle_sim(kw, W["v_true"], dt, nt)
    y, _ = so.forward(sim, W["v_true"], convention="fwdadj", device="cuda")
    th = torch.tensor(W["thetas"], device="cuda", requires_grad=True)
    ll = GridLikelihood.apply(th, model, torch.as_tensor(y, device="cuda"), sigma, True)
    ll.sum().backward()
    g = th.grad.cpu().numpy()
    # the exact discrete adjoint of the oracle, in theta space: B^T (d loglik / d v)
    v0 = base + Bm @ W["thetas"][0]
    ref = so.forward_adjoint(sim, y, sigma, velocity=v0, mode="exact", device="cuda")
    g_ref = -(Bm.T @ ref["dL_dv"])
    e = rel_l2(g[0], g_ref)
    e_ll = abs(float(ll[0].detach()) - ref["loglik"]) / abs(ref["loglik"])
    print(f"theta-gradient vs fp64 exact adjoint {e:.2e}, loglik {e_ll:.2e}")
    assert e <= TOL and e_ll <= TOL
    # central differences of the float64 oracle along 5 random unit directions
    drng = np.random.default_rng(0)
    eps = 0.5  # m/s on node values of N(0, 100^2)
    for k in range(5):
        d = drng.standard_normal(60)
        d /= np.linalg.norm(d)
        lp = so.misfit_loglik(sim, base + Bm @ (W["thetas"][0] + eps * d), y, sigma, device="cuda")
        lm = so.misfit_loglik(sim, base + Bm @ (W["thetas"][0] - eps * d), y, sigma, device="cuda")
        fd = (lp - lm) / (2 * eps)
        ad = float(g[0] @ d)
        print(f"direction {k}: adjoint {ad:.6e} FD {fd:.6e} rel {abs(ad - fd) / abs(fd):.2e}")
        assert abs(ad - fd) <= 1e-3 * abs(fd)


def test_single_large_solve_matches_fp64_oracle():
    nelx, nelz, N = 400, 200, 4
    coords, ng, v, dt = bench.single_model(nelx, nelz, N)
    nt = 5000
    rec = np.stack([np.linspace(0.0, 8000.0, 400), np.full(400, 1e-3)], 1)
    kw = dict(xmin=0.0, xmax=8000.0, zmin=0.0, zmax=4000.0, nelx=nelx, nelz=nelz, npol=N, dt=dt, nt=nt,
              src_xz=(4000.0, 1e-3), f0=15.0, amp=1.0, receivers=rec, pml_thickness=400.0,
              sponge_cmax=4000.0)
    plan = SEMPlan(coords=coords, node_grid=ng, **kw)
    sigma = 1e-3
    sim = _oracle_sim(kw, v, dt, nt)
    y, _ = so.forward(sim, v * 1.01, convention="fwdadj", device="cuda")
    s = SolveSpec(plan, torch.as_tensor(v, device="cuda"), adjoint=True, y_obs=torch.as_tensor(y, device="cuda"),
                  inv_sigma2=1.0 / (sigma ** 2 + 1e-24), ckpt_k=250)
    b = Batch()
    b.run([s])
    torch.cuda.synchronize()
    assert int(s.status.item()) == 0 and b.last_kernel == "strip"
    ref = so.forward_adjoint(sim, y, sigma, velocity=v, device="cuda")
    e = _errors(s, ref)
    print(f"400x200 el, 5000 steps, k=250: seismogram {e[0]:.2e} gradient {e[1]:.2e} loglik {e[2]:.2e} "
          "(vs fp64 oracle)")
    assert max(e) <= TOL, e


def test_mixed_orders_3_4_5_match_fp64_oracle():
    cases = bench.uneven_specs(64)
    pick = {}
    for c in cases:  # the largest mesh of each order in the uneven workload
        N = c["plan"]["npol"]
        if N not in pick or c["plan"]["nelx"] > pick[N]["plan"]["nelx"]:
            pick[N] = c
    assert sorted(pick) == [3, 4, 5]
    plans, specs, refs = [], [], []
    sigma = 1e-3
    for N in (3, 4, 5):
        c = pick[N]
        kw = {k: c["plan"][k] for k in c["plan"] if k not in ("coords", "node_grid")}
        p = SEMPlan(**c["plan"])
        sim = _oracle_sim(kw, c["v"], kw["dt"], kw["nt"])
        y, _ = so.forward(sim, c["v"] * 0.98, convention="fwdadj", device="cuda")
        plans.append(p)
        specs.append(SolveSpec(p, torch.as_tensor(c["v"], device="cuda"), adjoint=True,
                               y_obs=torch.as_tensor(y, device="cuda"),
                               inv_sigma2=1.0 / (sigma ** 2 + 1e-24), ckpt_k=0))
        refs.append((sim, y, c["v"]))
    b = Batch()
    b.run(specs)  # one launch sequence, one kernel launch per order and tick
    torch.cuda.synchronize()
    for N, s, (sim, y, v) in zip((3, 4, 5), specs, refs):
        assert int(s.status.item()) == 0
        ref = so.forward_adjoint(sim, y, sigma, velocity=v, device="cuda")
        e = _errors(s, ref)
        print(f"order {N}, {s.plan.nelx}x{s.plan.nelz} el, {s.plan.nt} steps: seismogram {e[0]:.2e} "
              f"gradient {e[1]:.2e} loglik {e[2]:.2e} (vs fp64 oracle)")
        assert max(e) <= TOL, e
