"""Automatic checkpoint schedule (ckpt_k = 0): a batch that sem_run splits into
consecutive groups under a memory budget, each group with its own checkpoint interval,
gives bitwise the same traces, log-likelihoods and gradients as one group with an
explicit interval (replay regenerates the forward exactly, and a solve's arithmetic
does not depend on its neighbours).  Also the tick-loop accounting."""
import math

import pytest
import torch

from mun_b200 import Batch, SolveSpec, _lib
from tests.goldens import load
from tests.gpu_cases import aligned_obs, dev, plan_for

pytestmark = pytest.mark.gpu
FLAGS = _lib.SEM_F_ADJOINT | _lib.SEM_F_SHIFT


def _specs(g, plan, n, k):
    y = dev(aligned_obs(g))
    v = dev(g["velocity"])
    return [SolveSpec(plan, v * (1.0 - 0.01 * i), adjoint=True, y_obs=y,
                      inv_sigma2=1.0 / (float(g["sigma"]) ** 2 + 1e-24), ckpt_k=k) for i in range(n)]


def _same(ref, got):
    for a, b in zip(ref, got):
        assert int(b.status.item()) == 0
        assert torch.equal(a.rec, b.rec)
        assert torch.equal(a.loglik, b.loglik)
        assert torch.equal(a.grad, b.grad)


@pytest.mark.parametrize("kernel", [1, 2])
def test_auto_schedule_groups_match_single_group(kernel):
    g = load("inject_n3")
    plan = plan_for(g["config"], g["dt"], g["nt"])
    nt, n = plan.nt, 6
    ref = _specs(g, plan, n, nt)
    b = Batch(kernel=kernel)
    b.run(ref)
    assert b.last_groups == 1
    assert b.last_ticks == 2 * nt + 2          # forward, read-out, scale, adjoint
    assert b.last_tick_ms() > 0.0

    # room for two solves at the smallest interval: at least three groups
    k_floor = max(2, min(nt, int(math.sqrt(2.0 * nt))))
    budget = int(2.5 * plan.workspace_bytes(FLAGS, k_floor))
    got = _specs(g, plan, n, 0)
    b.run(got, memory_budget=budget)
    print(f"kernel {kernel}: budget {budget} B -> {b.last_groups} groups, {b.last_ticks} ticks")
    assert b.last_groups >= 3
    _same(ref, got)

    # room for two whole forward histories: the model picks the split; same results
    budget = 2 * plan.workspace_bytes(FLAGS, nt) + 1
    got = _specs(g, plan, n, 0)
    b.run(got, memory_budget=budget)
    print(f"kernel {kernel}: budget {budget} B -> {b.last_groups} groups, {b.last_ticks} ticks")
    assert 1 <= b.last_groups <= n
    _same(ref, got)


def test_auto_schedule_mixed_explicit_and_forward_solves():
    # explicit intervals and forward-only solves keep their settings inside a split batch
    g = load("inject_n2")
    plan = plan_for(g["config"], g["dt"], g["nt"])
    nt = plan.nt
    ref = _specs(g, plan, 4, nt) + [SolveSpec(plan, dev(g["velocity"]))]
    Batch().run(ref)
    got = _specs(g, plan, 4, 0)
    got[1].ckpt_k = 7
    got.append(SolveSpec(plan, dev(g["velocity"])))
    # 60% of what the batch needs at the smallest intervals: it must be split
    k_floor = max(2, min(nt, int(math.sqrt(2.0 * nt))))
    need = (3 * plan.workspace_bytes(FLAGS, k_floor) + plan.workspace_bytes(FLAGS, 7)
            + plan.workspace_bytes(0, 2))
    b = Batch()
    b.run(got, memory_budget=int(0.6 * need))
    assert b.last_groups >= 2
    _same(ref[:4], got[:4])
    assert torch.equal(ref[4].rec, got[4].rec)
