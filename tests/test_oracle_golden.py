"""Pin the FP64 oracle against golden vectors produced by MUN's own sem_waveform."""
import numpy as np
import pytest

from oracle import sem_oracle as so
from tests.goldens import INJECT, load, rel_l2


@pytest.mark.parametrize("name", INJECT + ["circle_n5"])
def test_mesh_numbering_matches_reference(name):
    g = load(name)
    d = g["config"]["domain"]
    coords, conn, grid = so.create_global_mesh(d["xmin"], d["xmax"], d["zmin"], d["zmax"],
                                               d["nelem_x"], d["nelem_z"],
                                               g["config"]["method"]["polynomial_order"])
    assert coords.shape == g["coords"].shape
    np.testing.assert_array_equal(coords, g["coords"])


@pytest.mark.parametrize("name", INJECT)
def test_run_seismogram_matches_reference(name):
    g = load(name)
    sim = so.build_sim(g["config"], g["velocity"], dt=float(g["dt_run"]))
    assert sim.nt == int(g["nt_run"]) and sim.dt == float(g["dt_run"])
    assert sim.src_node == int(g["src_node"])
    rec, _ = so.forward(sim, convention="run")
    assert rel_l2(rec, g["rec_run"]) < 1e-10


@pytest.mark.parametrize("name", INJECT)
def test_forward_adjoint_matches_reference(name):
    g = load(name)
    sim = so.build_sim(g["config"], g["velocity"], dt=float(g["dt"]))
    assert sim.nt == int(g["nt"])
    y = so.align_observation(g["y_obs"], float(g["obs_dt"]), int(g["obs_nt"]), sim.dt, sim.nt)
    out = so.forward_adjoint(sim, y, float(g["sigma"]))
    assert rel_l2(out["clean"], g["clean"]) < 1e-10
    assert abs(out["loglik"] - float(g["loglik"])) <= 1e-9 * abs(float(g["loglik"]))
    assert rel_l2(out["dL_dv"], g["dL_dv"]) < 1e-9


@pytest.mark.parametrize("name", INJECT)
def test_reference_dot_test_reproduced(name):
    """The reference's node-space FD dot test (core.py:1494-1551), restated."""
    g = load(name)
    sim = so.build_sim(g["config"], g["velocity"], dt=float(g["dt"]))
    y = so.align_observation(g["y_obs"], float(g["obs_dt"]), int(g["obs_nt"]), sim.dt, sim.nt)
    rng = np.random.RandomState(int(g["dot_seed"]))
    delta = rng.randn(sim.npoints)
    delta /= np.linalg.norm(delta) + 1e-24
    lhs = float(np.dot(-g["dL_dv"], delta))
    eps = float(g["dot_eps"])
    s2 = float(g["sigma"]) ** 2 + 1e-24
    Jp = -so.misfit_loglik(sim, g["velocity"] + eps * delta, y, float(g["sigma"]), "run")
    Jm = -so.misfit_loglik(sim, g["velocity"] - eps * delta, y, float(g["sigma"]), "run")
    rhs = (Jp - Jm) / (2 * eps)
    assert abs(lhs - float(g["dot_lhs"])) <= 1e-9 * abs(float(g["dot_lhs"]))
    assert abs(rhs - float(g["dot_rhs"])) <= 1e-6 * abs(float(g["dot_rhs"])) + 1e-6 * abs(lhs)
    del s2


def test_circle_n5_solver_matches_reference():
    g = load("circle_n5")
    sim = so.build_sim(g["config"], g["velocity_run"], dt=float(g["dt_run"]))
    rec, _ = so.forward(sim, convention="run")
    assert rel_l2(rec, g["rec_run"]) < 1e-10
    sim2 = so.build_sim(g["config"], g["velocity"], dt=float(g["dt"]))
    out = so.forward_adjoint(sim2, g["y_obs"], float(g["sigma"]))
    assert rel_l2(out["clean"], g["clean"]) < 1e-10
    assert rel_l2(out["dL_dv"], g["dL_dv"]) < 1e-9


def test_layered_cfg0_oracle_matches_reference():
    g = load("layered_cfg0")
    sim = so.build_sim(g["config"], g["velocity"], dt=float(g["dt"]))
    assert sim.nt == int(g["nt"]) and sim.src_node == int(g["src_node"])
    rec, _ = so.forward(sim, convention="run")
    assert rel_l2(rec, g["rec_run"]) < 1e-10
    out = so.forward_adjoint(sim, g["y_obs"], float(g["sigma"]))
    assert rel_l2(out["clean"], g["clean"]) < 1e-10
    assert abs(out["loglik"] - float(g["loglik"])) <= 1e-9 * abs(float(g["loglik"]))
    assert rel_l2(out["dL_dv"], g["dL_dv"]) < 1e-8
