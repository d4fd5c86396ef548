"""The autotuner picks a configuration and the tuned run gives bitwise the default result."""
import numpy as np
import pytest
import torch

from mun_b200 import Batch, SolveSpec
from mun_b200.autotune import tune, tuned_batch
from tests.goldens import load
from tests.gpu_cases import aligned_obs, dev, plan_for

pytestmark = pytest.mark.gpu


def test_tuned_configuration_gives_the_same_numbers():
    g = load("inject_n3")
    plan = plan_for(g["config"], g["dt"], g["nt"])
    y = dev(aligned_obs(g))
    inv = 1.0 / float(g["sigma"]) ** 2

    def specs():
        return [SolveSpec(plan, dev(np.asarray(g["velocity"]) * (1 + 0.01 * i)), adjoint=True, y_obs=y,
                          inv_sigma2=inv, ckpt_k=9) for i in range(6)]
    cfg = tune(specs(), nt_proxy=24, repeats=1)
    assert cfg["kernel"] in (1, 2, 3, 4) and cfg["graph_chunk"] in (0, 32)
    ref = specs()
    Batch().run(ref)
    sp = specs()
    b, _ = tuned_batch(sp)
    b.run(sp)
    for a, c in zip(ref, sp):
        assert torch.equal(a.grad, c.grad) and torch.equal(a.rec, c.rec)


def test_batch_autotune_option_gives_the_same_numbers():
    g = load("inject_n2")
    plan = plan_for(g["config"], g["dt"], g["nt"])
    y = dev(aligned_obs(g))

    def specs():
        return [SolveSpec(plan, dev(np.asarray(g["velocity"]) * (1 - 0.01 * i)), adjoint=True, y_obs=y,
                          inv_sigma2=1e6, ckpt_k=0) for i in range(5)]
    ref = specs()
    Batch().run(ref)
    b = Batch(autotune=True)
    sp = specs()
    b.run(sp)
    assert b.last_tuned is not None and b.last_tuned["strip_bands"] in (0, 4, 8)
    for a, c in zip(ref, sp):
        assert torch.equal(a.grad, c.grad) and torch.equal(a.rec, c.rec) and torch.equal(a.loglik, c.loglik)
