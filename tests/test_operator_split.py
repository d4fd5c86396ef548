"""CPU checks of the operator split the kernels use (no GPU needed)."""
import numpy as np
import pytest

from mun_b200 import build_plan_arrays
from mun_b200.mesh import create_global_mesh
from oracle import sem_oracle as so
from tests import kernel_model as km
from tests.goldens import INJECT, load, rel_l2


def _arrays_for(g, dt=None):
    cfg = g["config"]
    d = cfg["domain"]
    sim = so.build_sim(cfg, g["velocity"], dt=float(g["dt"] if dt is None else dt))
    rc = cfg["receivers"]
    pos = np.asarray(rc["positions"]) if "positions" in rc else so.circle_receivers(
        *cfg["source"]["position"], rc["radius"], rc["num_receivers"])
    vcfg = cfg["velocity"]
    vmax = vcfg.get("outside_velocity", vcfg.get("vmax", 3000.0))
    a = build_plan_arrays(d["xmin"], d["xmax"], d["zmin"], d["zmax"], d["nelem_x"], d["nelem_z"],
                          cfg["method"]["polynomial_order"], sim.dt, sim.nt,
                          cfg["source"]["position"], cfg["source"]["frequency"],
                          cfg["source"]["amplitude"], pos, cfg["method"]["pml_thickness"], vmax)
    return sim, a


@pytest.mark.parametrize("name", INJECT + ["circle_n5"])
def test_node_numbering_and_coords(name):
    g = load(name)
    d = g["config"]["domain"]
    coords, conn, node_grid = create_global_mesh(d["xmin"], d["xmax"], d["zmin"], d["zmax"],
                                                 d["nelem_x"], d["nelem_z"],
                                                 g["config"]["method"]["polynomial_order"])
    np.testing.assert_allclose(coords, g["coords"], rtol=0, atol=1e-9)


@pytest.mark.parametrize("name", INJECT + ["circle_n5"])
def test_stiffness_split_matches_assembled_csr(name):
    g = load(name)
    sim, a = _arrays_for(g)
    Gx, Gz, S, w2D = sim.ops
    K = so.stiffness_csr(sim.velocity, sim.conn, Gx, Gz, S, w2D, sim.npoints)
    rng = np.random.default_rng(0)
    u = rng.standard_normal(sim.npoints)
    ref = (K @ __import__("torch").from_numpy(u)).numpy()
    mine = km.from_grid(a, km.K_apply(a, sim.velocity, km.to_grid(a, u)))
    assert rel_l2(mine, ref) < 1e-12
    # mass: dt^2 M^-1 separable
    Pm = km.from_grid(a, km.mass_inv_dt2(a))
    np.testing.assert_allclose(Pm, sim.dt ** 2 / sim.M, rtol=1e-12)
    # sponge separable
    dx = a["tab_x"][2 * (a["nelx"] * a["npol"] + 1):]
    dz = a["tab_z"][2 * (a["nelz"] * a["npol"] + 1):]
    # the tables carry the defects 1 - d of the separable sponge decay d = dx dz
    dd = km.from_grid(a, (1.0 - dz)[:, None] * (1.0 - dx)[None, :])
    np.testing.assert_allclose(dd, sim.decay, rtol=1e-12)
    # source node and receivers
    assert a["src_node"] == sim.src_node
    R = sim.R.toarray()
    N = a["npol"]
    for r in range(a["nrec"]):
        bx, bz = a["rec_base"][r]
        row = np.zeros((a["nelz"] * N + 1, a["nelx"] * N + 1))
        row[bz:bz + N + 1, bx:bx + N + 1] = a["rec_w"][r].reshape(N + 1, N + 1)
        np.testing.assert_allclose(km.from_grid(a, row), R[r], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("name", INJECT)
def test_sensitivity_split_matches_reference_kernel(name):
    import torch
    g = load(name)
    sim, a = _arrays_for(g)
    Gx, Gz, S, w2D = sim.ops
    rng = np.random.default_rng(1)
    u = rng.standard_normal(sim.npoints)
    w = rng.standard_normal(sim.npoints)
    ref = so.sensitivity_step(torch.from_numpy(u), torch.from_numpy(w), torch.from_numpy(sim.conn),
                              *(torch.from_numpy(x) for x in (Gx, Gz, S, w2D)), sim.npoints).numpy()
    mine = km.from_grid(a, km.sens_apply(a, km.to_grid(a, u), km.to_grid(a, w)))
    assert rel_l2(mine, ref) < 1e-12


@pytest.mark.parametrize("name", INJECT)
def test_two_field_recurrence_matches_reference(name):
    g = load(name)
    sim, a = _arrays_for(g, dt=g["dt_run"])
    sim = so.build_sim(g["config"], g["velocity"], dt=float(g["dt_run"]))
    rec, _ = km.forward(a, g["velocity"], shift=False)
    assert rel_l2(rec, g["rec_run"]) < 1e-11
