"""Strip kernel (TMA-staged element-row bands) against the reference goldens and
against the tile kernel; mixed-order batches; graph replay."""
import numpy as np
import pytest
import torch

from mun_b200 import Batch, SolveSpec
from tests.goldens import INJECT, load, rel_l2
from tests.gpu_cases import aligned_obs, dev, plan_for

pytestmark = pytest.mark.gpu
TOL = 1e-4
CASES = INJECT + ["circle_n5", "layered_cfg0"]


def _fwdadj(g, kernel, exact=False, k=0):
    plan = plan_for(g["config"], g["dt"], g["nt"])
    s = SolveSpec(plan, dev(g["velocity"]), adjoint=True, exact=exact, y_obs=dev(aligned_obs(g)),
                  inv_sigma2=1.0 / (float(g["sigma"]) ** 2 + 1e-24), ckpt_k=k)
    b = Batch(kernel=kernel)
    b.run([s])
    assert b.last_kernel == {1: "tile", 2: "strip"}[kernel]
    return s


@pytest.mark.parametrize("name", CASES)
def test_strip_forward_adjoint_matches_reference(name):
    g = load(name)
    s = _fwdadj(g, 2)
    t = _fwdadj(g, 1)
    assert int(s.status.item()) == 0
    e_clean = rel_l2(s.rec.cpu().numpy(), g["clean"])
    e_grad = rel_l2(-s.grad.cpu().numpy(), g["dL_dv"])
    e_ll = abs(float(s.loglik.item()) - float(g["loglik"])) / abs(float(g["loglik"]))
    d_tile = rel_l2(s.grad.cpu().numpy(), t.grad.cpu().numpy())
    print(f"{name} strip: clean {e_clean:.2e} loglik {e_ll:.2e} dL/dv {e_grad:.2e} "
          f"(vs tile kernel {d_tile:.1e}, bitwise={torch.equal(s.grad, t.grad)})")
    assert max(e_clean, e_grad, e_ll) <= TOL
    # same arithmetic in both kernels (explicit rounding where a compiler could fuse)
    assert torch.equal(s.grad, t.grad) and torch.equal(s.rec, t.rec), d_tile
    assert torch.equal(s.loglik, t.loglik)


@pytest.mark.parametrize("name", ["inject_n3", "layered_cfg0"])
def test_strip_forward_run_convention(name):
    g = load(name)
    plan = plan_for(g["config"], g["dt_run"], g["nt_run"])
    v = g["velocity_run"] if "velocity_run" in g else g["velocity"]
    s = SolveSpec(plan, dev(v))
    Batch(kernel=2).run([s])
    e = rel_l2(s.rec.cpu().numpy(), g["rec_run"])
    print(f"{name} strip forward: {e:.2e}")
    assert e <= TOL


def test_strip_checkpoint_and_batch_invariance():
    names = ["inject_n1", "inject_n2", "inject_n3", "inject_n6", "circle_n5"]
    gs = [load(n) for n in names]
    plans = [plan_for(g["config"], g["dt"], g["nt"]) for g in gs]

    def specs(k):
        return [SolveSpec(p, dev(g["velocity"]), adjoint=True, y_obs=dev(aligned_obs(g)),
                          inv_sigma2=1.0 / float(g["sigma"]) ** 2, ckpt_k=k) for g, p in zip(gs, plans)]
    alone = []
    for sp in specs(5):
        Batch(kernel=2).run([sp])
        alone.append(sp)
    for k, chunk in ((5, 0), (11, 32), (1000000, 7)):
        mixed = specs(k)
        Batch(kernel=2, graph_chunk=chunk).run(mixed)
        for a, b in zip(alone, mixed):
            assert torch.equal(a.grad, b.grad) and torch.equal(a.rec, b.rec)
            assert torch.equal(a.loglik, b.loglik)


def test_strip_exact_mode_and_window():
    g = load("inject_n2")
    s = _fwdadj(g, 2, exact=True)
    t = _fwdadj(g, 1, exact=True)
    assert rel_l2(s.grad.cpu().numpy(), t.grad.cpu().numpy()) <= 1e-6
    plan = plan_for(g["config"], g["dt"], g["nt"])
    y = aligned_obs(g)
    nt = int(g["nt"])
    win = (nt // 4, 3 * nt // 4, 3)
    yw = y[win[0]:win[1]][::win[2]]
    outs = []
    for kernel in (1, 2):
        sp = SolveSpec(plan, dev(g["velocity"]), adjoint=True, y_obs=dev(yw), window=win,
                       inv_sigma2=1.0 / float(g["sigma"]) ** 2)
        Batch(kernel=kernel).run([sp])
        outs.append(sp)
    assert rel_l2(outs[0].grad.cpu().numpy(), outs[1].grad.cpu().numpy()) <= 1e-6
    assert abs(float(outs[0].loglik.item()) - float(outs[1].loglik.item())) <= 1e-6 * abs(float(outs[0].loglik.item()))


@pytest.mark.parametrize("name", ["inject_n1", "inject_n3", "inject_n6", "circle_n5", "layered_cfg0"])
def test_strip_z_chunks_bitwise(name):
    # strips split into chunks of 1..3 element rows (each recomputing the z-line segments
    # of the row above) give bitwise the results of full-height strips
    g = load(name)
    plan = plan_for(g["config"], g["dt"], g["nt"])
    nelz = g["config"]["domain"]["nelem_z"]

    def run(bands, **kw):
        s = SolveSpec(plan, dev(g["velocity"]), **kw)
        Batch(kernel=2, strip_bands=bands).run([s])
        return s
    y = dev(aligned_obs(g))
    inv = 1.0 / (float(g["sigma"]) ** 2 + 1e-24)
    it1 = max(2, plan.nt // 2)
    for kw in (dict(), dict(shift=True), dict(adjoint=True, y_obs=y, inv_sigma2=inv),
               dict(adjoint=True, exact=True, y_obs=y[: -(-(it1 - 1) // 3)], inv_sigma2=inv,
                    window=(1, it1, 3))):
        full = run(nelz, **kw)
        for bands in (1, 2, 3):
            part = run(bands, **kw)
            assert int(part.status.item()) == 0
            assert torch.equal(full.rec, part.rec), (name, bands, kw.keys())
            if full.grad is not None:
                assert torch.equal(full.grad, part.grad), (name, bands)
                assert torch.equal(full.loglik, part.loglik)
