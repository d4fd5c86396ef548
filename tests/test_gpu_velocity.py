"""Device velocity builder (sem_velocity_from_curve) against the reference's velocity
models (goldens) and against the host builders, for both curve closures."""
import numpy as np
import pytest
import torch

from mun_b200.sem_waveform import velocity as V
from mun_b200.sem_waveform.mesh import create_global_mesh
from tests.goldens import load

pytestmark = pytest.mark.gpu


def _coords(cfg):
    d = cfg["domain"]
    c, _, _ = create_global_mesh(d["xmin"], d["xmax"], d["zmin"], d["zmax"], d["nelem_x"], d["nelem_z"],
                                 cfg["method"]["polynomial_order"])
    return c


def test_layered_anomaly_matches_reference():
    g = load("layered_cfg0")
    v = g["config"]["velocity"]
    coords = _coords(g["config"])
    bg = V.build_layered_background(coords, v["layers"]["interfaces_z"], v["layers"]["velocities"])
    vel, sd, us, nr = V.build_velocity_device(torch.as_tensor(coords, device="cuda"), np.asarray(g["ctrl"]),
                                              v["tau"], v["spline_samples"], v["anomaly"]["v_inside"],
                                              v_background_dev=torch.as_tensor(bg, device="cuda"))
    assert np.max(np.abs(vel.cpu().numpy() - g["velocity"])) < 1e-8
    assert np.max(np.abs(sd.cpu().numpy() - g["signed_dist"])) < 1e-8


def test_canonical_matches_reference_and_host_extras():
    g = load("circle_n5")
    v = g["config"]["velocity"]
    coords = _coords(g["config"])
    ctrl = np.asarray(g["ctrl"])
    vel, sd, us, nr = V.build_velocity_device(torch.as_tensor(coords, device="cuda"), ctrl, v["tau"],
                                              v["spline_samples"], v["inside_velocity"],
                                              v_outside=v["outside_velocity"])
    assert np.max(np.abs(vel.cpu().numpy() - g["velocity"])) < 1e-8
    _, sdh, ex = V.build_velocity_on_sem_nodes(coords, ctrl, v["inside_velocity"], v["outside_velocity"],
                                               v["tau"], v["spline_samples"])
    assert np.max(np.abs(us.cpu().numpy() - ex["u_star"])) < 1e-9
    assert np.max(np.abs(nr.cpu().numpy() - ex["normal_out"])) < 1e-9


def test_periodic_closure_matches_host():
    rng = np.random.default_rng(1)
    coords = np.stack(np.meshgrid(np.linspace(0, 2000, 161), np.linspace(0, 1000, 81)), -1).reshape(-1, 2)
    ctrl = np.array([[800, 300], [1000, 250], [1250, 320], [1300, 500], [1050, 600], [820, 520], [760, 400]],
                    dtype=float) + rng.normal(0, 5, (7, 2))
    bg = 2000.0 + coords[:, 1]
    for blend in ("smooth", "replace"):
        vd, sdd, _, _ = V.build_velocity_device(torch.as_tensor(coords, device="cuda"), ctrl, 12.0, 600, 2600.0,
                                                v_background_dev=torch.as_tensor(bg, device="cuda"),
                                                periodic=True, blend=blend)
        vh, sdh, _ = V.build_velocity_2d_background_with_anomaly(coords, bg, ctrl, 2600.0, 12.0, 600, 7, blend)
        assert np.max(np.abs(vd.cpu().numpy() - vh)) < 1e-8
        assert np.max(np.abs(sdd.cpu().numpy() - sdh)) < 1e-8
