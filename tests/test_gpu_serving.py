"""Serving engine (continuous batching): results bitwise equal alone and in a mix,
admission under a memory cap, and a Poisson request stream through the request loop."""
import numpy as np
import pytest
import torch

from mun_b200 import Batch, SolveSpec
from mun_b200.serving import Engine, Request, serve
from tests.goldens import INJECT, load
from tests.gpu_cases import aligned_obs, dev, plan_for

pytestmark = pytest.mark.gpu


def _specs():
    out = []
    for name in INJECT + ["circle_n5"]:
        g = load(name)
        plan = plan_for(g["config"], g["dt"], g["nt"])
        y = dev(aligned_obs(g))
        inv = 1.0 / float(g["sigma"]) ** 2
        v = np.asarray(g["velocity"])
        out.append(lambda p=plan, v=v, y=y, inv=inv: SolveSpec(p, dev(v), adjoint=True, y_obs=y,
                                                                inv_sigma2=inv, ckpt_k=7))
        out.append(lambda p=plan, v=v, y=y, inv=inv: SolveSpec(p, dev(v * 1.01), misfit=True, y_obs=y,
                                                                inv_sigma2=inv, shift=True))
        out.append(lambda p=plan, v=v: SolveSpec(p, dev(v * 0.98)))
    return out


@pytest.mark.parametrize("kernel", [0, 1, 2])
def test_engine_mix_is_bitwise_equal_to_alone(kernel):
    makers = _specs()
    alone = []
    for mk in makers:
        s = mk()
        Batch(kernel=kernel).run([s])
        alone.append(s)
    eng = Engine(max_solves=6, memory_cap_bytes=2 << 30, ticks_per_step=13, kernel=kernel)
    tickets = []
    for i, mk in enumerate(makers):  # staggered: a new request every few steps
        tickets.append(eng.submit(mk()))
        for _ in range(i % 3):
            eng.step()
    eng.run_until_done(tickets)
    torch.cuda.synchronize()
    for t, a in zip(tickets, alone):
        b = eng.release(t)
        assert torch.equal(a.rec, b.rec)
        if a.loglik is not None:
            assert torch.equal(a.loglik, b.loglik)
        if a.grad is not None:
            assert torch.equal(a.grad, b.grad)
        assert int(b.status.item()) == 0


def test_engine_memory_cap_queues_and_completes():
    makers = _specs()
    specs = [makers[12]() for _ in range(6)]  # six equal-size forward+adjoint solves (order 5)
    one = specs[0].plan.workspace_bytes(specs[0].flags, 7)
    assert one > (4 << 20)
    eng = Engine(max_solves=64, memory_cap_bytes=int(2.5 * one), ticks_per_step=32)
    tickets = [eng.submit(s) for s in specs]
    eng.step()
    st = eng.stats()
    assert st["running"] <= 2 and st["queued"] >= len(specs) - 2
    eng.run_until_done(tickets)
    for t in tickets:
        assert int(eng.release(t).status.item()) == 0
    assert eng.stats()["bytes_in_use"] == 0


def test_request_loop_poisson_stream():
    makers = _specs()
    rng = np.random.default_rng(0)
    arrivals = np.cumsum(rng.exponential(1.0 / 200.0, size=24))
    reqs = [Request(float(a), makers[i % len(makers)](), "mix") for i, a in enumerate(arrivals)]
    eng = Engine(max_solves=16, memory_cap_bytes=2 << 30, ticks_per_step=16)
    done, lat, wall = serve(eng, reqs)
    assert len(done) == len(reqs)
    assert np.all(lat > 0)
    print(f"served {len(done)} requests in {wall:.3f} s, p50 {1e3 * np.percentile(lat, 50):.1f} ms, "
          f"p99 {1e3 * np.percentile(lat, 99):.1f} ms")
