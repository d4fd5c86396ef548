"""Host-side parts of the drop-in SEMSimulation against the reference's own outputs:
config validation, mesh, velocity builders, CFL/dt, control-point projection."""
import numpy as np
import pytest

from mun_b200.sem_waveform import SEMSimulation
from mun_b200.sem_waveform import velocity as V
from mun_b200.sem_waveform.utils import adjust_time_step_for_stability
from tests.goldens import load, rel_l2


def test_missing_key_raises_value_error():
    with pytest.raises(ValueError, match="Missing required config key"):
        SEMSimulation({"domain": {}}, device="cpu")


@pytest.mark.parametrize("name", ["layered_cfg0", "circle_n5"])
def test_init_matches_reference(name):
    g = load(name)
    sim = SEMSimulation(g["config"], device="cpu")
    assert sim.npoints == len(g["velocity"])
    assert sim.src_node == int(g["src_node"])
    assert sim.dt == pytest.approx(float(g["dt_run"]), rel=1e-15)
    assert sim.nt == int(g["nt_run"])


def test_layered_velocity_builder_matches_reference():
    g = load("layered_cfg0")
    sim = SEMSimulation(g["config"], device="cpu")
    v, sd, ex = sim._build_velocity(np.asarray(g["ctrl"]))
    assert np.max(np.abs(v - g["velocity"])) < 1e-8
    assert np.max(np.abs(sd - g["signed_dist"])) < 1e-8
    vt, _, _ = sim._build_velocity(np.asarray(g["ctrl_true"]))
    assert np.max(np.abs(vt - g["velocity_true"])) < 1e-8


def test_canonical_velocity_builder_matches_reference():
    g = load("circle_n5")
    sim = SEMSimulation(g["config"], device="cpu")
    v, sd, _ = sim._build_velocity(np.asarray(g["ctrl"]))
    assert np.max(np.abs(v - g["velocity"])) < 1e-8
    assert np.max(np.abs(sd - g["signed_dist"])) < 1e-8


@pytest.mark.parametrize("name", ["layered_cfg0", "circle_n5"])
def test_control_point_projection_matches_reference(name):
    """Reference's node-space dL/dv through our projection reproduces its 12-D gradient."""
    g = load(name)
    sim = SEMSimulation(g["config"], device="cpu")
    ctrl = np.asarray(g["ctrl"])
    _, sd, ex = sim._build_velocity(ctrl)
    proj = sim._analytical_gradient_projection_improved(g["dL_dv"], ctrl, g["config"]["velocity"]["tau"],
                                                        sd, ex)
    ours = np.empty(12)
    ours[0::2], ours[1::2] = proj["grad_ctrl_x"], proj["grad_ctrl_z"]
    assert rel_l2(ours, g["grad_ctrl"]) < 1e-8


def test_periodic_curve_basis_partition_of_unity():
    ctrl = np.array([[0, 0], [1, 0], [2, 1], [1, 2], [0, 2], [-1, 1]], dtype=float)
    sp = V.closed_spline_periodic(ctrl)
    u = np.linspace(sp.lo, sp.hi, 50, endpoint=False)
    np.testing.assert_allclose(sp.basis_matrix(u).sum(1), 1.0, atol=1e-13)
    sp = V.closed_spline_clamped(ctrl)
    u = np.linspace(sp.lo, sp.hi, 50)
    np.testing.assert_allclose(sp.basis_matrix(u).sum(1), 1.0, atol=1e-13)


def test_cfl_rule():
    dt, nt = adjust_time_step_for_stability(np.array([1500.0, 3000.0]), 1.0, 0.33, 4, 50.0, 50.0, 3000.0)
    assert dt == pytest.approx(0.35 * 10.0 / (3000.0 * 5 * np.sqrt(2.0)))
    assert nt == int(np.ceil(0.33 / dt))
    dt2, _ = adjust_time_step_for_stability(np.array([1500.0]), 1e-5, 0.33, 4, 50.0, 50.0, 3000.0)
    assert dt2 == 1e-5
    with pytest.raises(ValueError):
        adjust_time_step_for_stability(np.array([np.nan]), 1e-5, 0.33, 4, 50.0, 50.0, 3000.0)


def test_grid_background_bilinear():
    xg = np.array([0.0, 1.0, 2.0])
    zg = np.array([0.0, 2.0])
    grid = np.array([[1.0, 2.0, 3.0], [3.0, 4.0, 5.0]])
    pts = np.array([[0.5, 1.0], [2.0, 2.0], [-1.0, 0.0], [1.5, 0.5]])
    v = V.build_background_from_grid(pts, xg, zg, grid)
    np.testing.assert_allclose(v, [2.5, 5.0, 1.0, 3.0])
