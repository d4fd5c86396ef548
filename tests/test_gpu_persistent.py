"""Persistent tile kernel (kernel 3): the tile kernel's tick body run for the whole tick
program in one cooperative launch, with a grid barrier between ticks.  Same arithmetic,
so results are bitwise those of the per-tick tile kernel; groups whose tiles cannot all
be resident fall back to per-tick launches."""
import pytest
import torch

from mun_b200 import Batch, SolveSpec
from tests.goldens import load
from tests.gpu_cases import aligned_obs, dev, plan_for

pytestmark = pytest.mark.gpu


def _specs(g, plan, n, adjoint=True, ckpt_k=5, window=None):
    y = dev(aligned_obs(g))
    v = dev(g["velocity"])
    out = []
    for i in range(n):
        kw = {}
        if adjoint:
            kw = dict(adjoint=True, y_obs=y, inv_sigma2=1.0 / (float(g["sigma"]) ** 2 + 1e-24),
                      ckpt_k=ckpt_k)
        out.append(SolveSpec(plan, v * (1.0 - 0.02 * i), **kw))
    return out


def _same(a, b, adjoint=True):
    for x, y in zip(a, b):
        assert int(x.status.item()) == 0 and int(y.status.item()) == 0
        assert torch.equal(x.rec, y.rec)
        if adjoint:
            assert torch.equal(x.grad, y.grad)
            assert torch.equal(x.loglik, y.loglik)


@pytest.mark.parametrize("name", ["inject_n1", "inject_n3", "inject_n6", "circle_n5"])
@pytest.mark.parametrize("ckpt_k", [5, 0])
def test_persistent_equals_tile_kernel(name, ckpt_k):
    g = load(name)
    plan = plan_for(g["config"], g["dt"], g["nt"])
    ref = _specs(g, plan, 2, ckpt_k=ckpt_k)
    got = _specs(g, plan, 2, ckpt_k=ckpt_k)
    # 4x4 tiles: few enough CTAs to be resident at every order
    Batch(kernel=1, tile=(4, 4)).run(ref)
    b = Batch(kernel=3, tile=(4, 4))
    b.run(got)
    assert b.last_kernel == "persistent" and b.last_launches <= 4
    _same(ref, got)


def test_persistent_forward_only():
    g = load("layered_cfg0")
    plan = plan_for(g["config"], g["dt"], g["nt"])
    ref = _specs(g, plan, 1, adjoint=False)
    got = _specs(g, plan, 1, adjoint=False)
    Batch(kernel=1).run(ref)
    b = Batch(kernel=3)
    b.run(got)
    assert b.last_kernel == "persistent"
    _same(ref, got, adjoint=False)


def test_persistent_falls_back_when_tiles_are_not_resident():
    # 2x1 tiles of a 16x10 mesh: 80 CTAs per solve; 12 solves exceed every SM's slots
    g = load("inject_n2")
    plan = plan_for(g["config"], g["dt"], g["nt"])
    ref = _specs(g, plan, 12)
    got = _specs(g, plan, 12)
    Batch(kernel=1, tile=(2, 1)).run(ref)
    b = Batch(kernel=3, tile=(2, 1))
    b.run(got)
    assert b.last_kernel == "tile"
    _same(ref, got)


@pytest.mark.parametrize("name", ["inject_n1", "inject_n3", "inject_n6", "circle_n5", "layered_cfg0"])
@pytest.mark.parametrize("bands", [0, 2])
def test_persistent_strip_equals_strip_kernel(name, bands):
    """Persistent strip kernel (kernel 4): the strip kernel's tick body for the whole tick
    program in one cooperative launch, CTAs synchronised with their four neighbours only;
    bitwise the per-tick strip kernel, with full-height strips and with 2-row chunks (the
    chunks above and below are neighbours too), replay (k = 5) and several solves."""
    g = load(name)
    plan = plan_for(g["config"], g["dt"], g["nt"])
    a = _specs(g, plan, 3)
    Batch(kernel=2, strip_bands=bands).run(a)
    b = _specs(g, plan, 3)
    bb = Batch(kernel=4, strip_bands=bands)
    bb.run(b)
    torch.cuda.synchronize()
    assert bb.last_kernel == "persistent strip"
    _same(a, b)


def test_persistent_strip_stacey_and_forward_only():
    from mun_b200 import SEMPlan
    import numpy as np
    g = load("layered_cfg0")
    cfg = g["config"]
    d = cfg["domain"]
    from tests.gpu_cases import receivers_of, sponge_cmax
    plan = SEMPlan(xmin=d["xmin"], xmax=d["xmax"], zmin=d["zmin"], zmax=d["zmax"], nelx=d["nelem_x"],
                   nelz=d["nelem_z"], npol=cfg["method"]["polynomial_order"], dt=float(g["dt"]), nt=int(g["nt"]),
                   src_xz=cfg["source"]["position"], f0=cfg["source"]["frequency"],
                   amp=cfg["source"]["amplitude"], receivers=receivers_of(cfg),
                   pml_thickness=cfg["method"]["pml_thickness"], sponge_cmax=sponge_cmax(cfg), boundary="stacey")
    for adjoint in (True, False):
        a = _specs(g, plan, 2, adjoint=adjoint, ckpt_k=0)
        Batch(kernel=2, strip_bands=3).run(a)
        b = _specs(g, plan, 2, adjoint=adjoint, ckpt_k=0)
        bb = Batch(kernel=4, strip_bands=3)
        bb.run(b)
        torch.cuda.synchronize()
        assert bb.last_kernel == "persistent strip"
        _same(a, b, adjoint)
        assert np.isfinite(b[0].rec.cpu().numpy()).all()
