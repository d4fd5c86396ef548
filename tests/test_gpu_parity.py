"""GPU parity through the C ABI: float32 CUDA path vs the reference's own outputs
(golden vectors) and vs the float64 oracle.  Tolerance: relative L2 <= 1e-4."""
import numpy as np
import pytest
import torch

from mun_b200 import Batch, SolveSpec, forward, forward_adjoint
from oracle import sem_oracle as so
from tests.goldens import INJECT, load, rel_l2
from tests.gpu_cases import aligned_obs, dev, plan_for

pytestmark = pytest.mark.gpu
TOL = 1e-4
CASES = INJECT + ["circle_n5", "layered_cfg0"]


def _vel(g, run=False):
    return g["velocity_run"] if (run and "velocity_run" in g) else g["velocity"]


@pytest.mark.parametrize("name", CASES)
def test_forward_matches_reference(name):
    g = load(name)
    plan = plan_for(g["config"], g["dt_run"], g["nt_run"])
    rec = forward(plan, dev(_vel(g, run=True))).cpu().numpy()
    err_ref = rel_l2(rec, g["rec_run"])
    sim = so.build_sim(g["config"], _vel(g, run=True), dt=float(g["dt_run"]))
    rec64, _ = so.forward(sim, convention="run")
    err_fp64 = rel_l2(rec, rec64)
    print(f"{name}: forward rel L2 vs reference {err_ref:.2e}, vs fp64 oracle {err_fp64:.2e}")
    assert err_ref <= TOL and err_fp64 <= TOL


@pytest.mark.parametrize("name", CASES)
def test_forward_adjoint_matches_reference(name):
    g = load(name)
    plan = plan_for(g["config"], g["dt"], g["nt"])
    y = aligned_obs(g)
    out = forward_adjoint(plan, dev(g["velocity"]), dev(y), float(g["sigma"]))
    torch.cuda.synchronize()
    assert int(out["status"].item()) == 0
    clean = out["clean"].cpu().numpy()
    dL = -out["grad"].cpu().numpy()
    ll = float(out["loglik"].item())
    e_clean = rel_l2(clean, g["clean"])
    e_grad = rel_l2(dL, g["dL_dv"])
    e_ll = abs(ll - float(g["loglik"])) / abs(float(g["loglik"]))
    print(f"{name}: clean {e_clean:.2e} loglik {e_ll:.2e} dL/dv {e_grad:.2e}")
    assert e_clean <= TOL and e_ll <= TOL and e_grad <= TOL


@pytest.mark.parametrize("name", ["inject_n3", "circle_n5"])
def test_exact_adjoint_matches_fp64_oracle(name):
    g = load(name)
    plan = plan_for(g["config"], g["dt"], g["nt"])
    y = aligned_obs(g)
    out = forward_adjoint(plan, dev(g["velocity"]), dev(y), float(g["sigma"]), exact=True)
    sim = so.build_sim(g["config"], g["velocity"], dt=float(g["dt"]))
    ref = so.forward_adjoint(sim, y, float(g["sigma"]), mode="exact")
    e = rel_l2(-out["grad"].cpu().numpy(), ref["dL_dv"])
    print(f"{name}: exact-mode dL/dv vs fp64 oracle {e:.2e}")
    assert e <= TOL


def test_checkpoint_interval_does_not_change_results():
    g = load("inject_n2")
    plan = plan_for(g["config"], g["dt"], g["nt"])
    y = dev(aligned_obs(g))
    v = dev(g["velocity"])
    outs = [forward_adjoint(plan, v, y, float(g["sigma"]), ckpt_k=k) for k in (2, 7, 64, plan.nt)]
    for o in outs[1:]:
        assert torch.equal(o["grad"], outs[0]["grad"])
        assert torch.equal(o["clean"], outs[0]["clean"])
        assert torch.equal(o["loglik"], outs[0]["loglik"])


def test_batch_invariance_and_graphs():
    """A solve alone and inside a mixed batch (other meshes and orders) is bitwise equal,
    with and without CUDA-graph replay of the tick sequence."""
    names = ["inject_n1", "inject_n2", "inject_n3", "inject_n6"]
    gs = [load(n) for n in names]
    plans = [plan_for(g["config"], g["dt"], g["nt"]) for g in gs]
    alone = []
    for g, p in zip(gs, plans):
        s = SolveSpec(p, dev(g["velocity"]), adjoint=True, y_obs=dev(aligned_obs(g)),
                      inv_sigma2=1.0 / float(g["sigma"]) ** 2, ckpt_k=5)
        Batch().run([s])
        alone.append(s)
    for chunk in (0, 16):
        specs = [SolveSpec(p, dev(g["velocity"]), adjoint=True, y_obs=dev(aligned_obs(g)),
                           inv_sigma2=1.0 / float(g["sigma"]) ** 2, ckpt_k=5)
                 for g, p in zip(gs, plans)]
        Batch(graph_chunk=chunk).run(specs)
        for a, b in zip(alone, specs):
            assert torch.equal(a.grad, b.grad) and torch.equal(a.rec, b.rec)
            assert torch.equal(a.loglik, b.loglik)


@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("adjoint", [False, True])
def test_nonfinite_velocity_sets_status(kernel, adjoint):
    g = load("inject_n2")
    plan = plan_for(g["config"], g["dt"], g["nt"])
    v = np.array(g["velocity"])
    v[len(v) // 2] = np.inf
    kw = dict(adjoint=True, y_obs=dev(aligned_obs(g)), inv_sigma2=1.0) if adjoint else {}
    s = SolveSpec(plan, dev(v), **kw)
    Batch(kernel=kernel).run([s])
    assert int(s.status.item()) != 0


def test_misfit_window_matches_oracle():
    """CO2 misfit window with decimation (single_cubic core.py:1441-1552) vs the oracle."""
    g = load("inject_n3")
    plan = plan_for(g["config"], g["dt"], g["nt"])
    y = aligned_obs(g)
    nt = int(g["nt"])
    win = (nt // 5, 4 * nt // 5, 2)
    yw = y[win[0]:win[1]][::win[2]]
    s = SolveSpec(plan, dev(g["velocity"]), adjoint=True, y_obs=dev(yw), window=win,
                  inv_sigma2=1.0 / float(g["sigma"]) ** 2)
    Batch().run([s])
    sim = so.build_sim(g["config"], g["velocity"], dt=float(g["dt"]))
    ref = so.forward_adjoint(sim, yw, float(g["sigma"]), window=win)
    e_g = rel_l2(-s.grad.cpu().numpy(), ref["dL_dv"])
    e_l = abs(float(s.loglik.item()) - ref["loglik"]) / abs(ref["loglik"])
    print(f"window: dL/dv {e_g:.2e} loglik {e_l:.2e}")
    assert e_g <= TOL and e_l <= TOL
