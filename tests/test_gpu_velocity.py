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


def _host_projection(ctrl, periodic, dL, sd, us, nrm, v_in, bg, tau, floor_one):
    """The host projection's formula (_analytical_gradient_projection_improved)."""
    ts = max(tau, 1e-12)
    sig = 1.0 / (1.0 + np.exp(np.clip(sd / ts, -50.0, 50.0)))
    delta = v_in - bg
    dv = delta * sig * (1.0 - sig) * (-1.0 / ts)
    mask = np.abs(dv) > 1e-8 * (np.maximum(1.0, np.abs(delta)) if floor_one else np.abs(delta))
    K = len(ctrl)
    if periodic:
        sp = V.closed_spline_periodic(ctrl)
        t = np.clip(sp.lo + np.mod(us[mask], 1.0) * (sp.hi - sp.lo), sp.lo, np.nextafter(sp.hi, sp.lo))
        Bc = sp.basis_matrix(t)
        B = Bc[:, :K].copy()
        for j in range(Bc.shape[1] - K):
            B[:, j] += Bc[:, K + j]
    else:
        sp = V.closed_spline_clamped(ctrl)
        Bc = sp.basis_matrix(us[mask])
        B = Bc[:, :K].copy()
        B[:, 0] += Bc[:, K:].sum(axis=1)
    w = (dL[mask] * dv[mask])[:, None]
    return np.concatenate([np.sum(w * B * nrm[mask, 0:1], 0), np.sum(w * B * nrm[mask, 1:2], 0)])


@pytest.mark.parametrize("case", ["layered", "canonical", "periodic"])
def test_device_projection_matches_host_formula(case):
    rng = np.random.default_rng(2)
    if case == "periodic":
        coords = np.stack(np.meshgrid(np.linspace(0, 2000, 161), np.linspace(0, 1000, 81)), -1).reshape(-1, 2)
        ctrl = np.array([[800, 300], [1000, 250], [1250, 320], [1300, 500], [1050, 600], [820, 520],
                         [760, 400]], dtype=float)
        bg, tau, v_in, floor_one, const = 2000.0 + coords[:, 1], 12.0, 2600.0, True, 0.0
        samples = 600
    elif case == "layered":
        g = load("layered_cfg0")
        v = g["config"]["velocity"]
        coords = _coords(g["config"])
        ctrl = np.asarray(g["ctrl"], dtype=float)
        bg = V.build_layered_background(coords, v["layers"]["interfaces_z"], v["layers"]["velocities"])
        tau, v_in, floor_one, const, samples = v["tau"], v["anomaly"]["v_inside"], True, 0.0, v["spline_samples"]
    else:
        g = load("circle_n5")
        v = g["config"]["velocity"]
        coords = _coords(g["config"])
        ctrl = np.asarray(g["ctrl"], dtype=float)
        bg, tau, v_in, floor_one, const = None, v["tau"], v["inside_velocity"], False, v["outside_velocity"]
        samples = v["spline_samples"]
    S = 3
    builds, dLs = [], []
    for s in range(S):
        c = ctrl + rng.normal(0, 4, ctrl.shape)
        bgd = None if bg is None else torch.as_tensor(bg, device="cuda")
        builds.append((c,) + V.build_velocity_device(torch.as_tensor(coords, device="cuda"), c, tau, samples,
                                                     v_in, v_outside=const, v_background_dev=bgd,
                                                     periodic=(case == "periodic")))
        dLs.append(rng.normal(size=len(coords)))
    dL = torch.as_tensor(np.stack(dLs), device="cuda")
    for s, (c, vel, sd, us, nr) in enumerate(builds):
        got = V.project_ctrl_device(c, case == "periodic", dL[s:s + 1], sd[None], us[None], nr[None], v_in, tau,
                                    v_background_dev=None if bg is None else torch.as_tensor(bg, device="cuda"),
                                    v_background_const=const, floor_one=floor_one).cpu().numpy()[0]
        want = _host_projection(c, case == "periodic", dLs[s], sd.cpu().numpy(), us.cpu().numpy(),
                                nr.cpu().numpy(), v_in, const if bg is None else bg, tau, floor_one)
        err = np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-300)
        print(f"{case} sample {s}: rel {err:.2e}")
        assert np.linalg.norm(want) > 0 and err < 1e-10
    # batched call (S rows) gives the same rows
    allg = V.project_ctrl_device(builds[0][0], case == "periodic", dL, torch.stack([b[2] for b in builds]),
                                 torch.stack([b[3] for b in builds]), torch.stack([b[4] for b in builds]), v_in, tau,
                                 v_background_dev=None if bg is None else torch.as_tensor(bg, device="cuda"),
                                 v_background_const=const, floor_one=floor_one)
    one = V.project_ctrl_device(builds[1][0], case == "periodic", dL[1:2], builds[1][2][None], builds[1][3][None],
                                builds[1][4][None], v_in, tau,
                                v_background_dev=None if bg is None else torch.as_tensor(bg, device="cuda"),
                                v_background_const=const, floor_one=floor_one)
    assert torch.equal(allg[1], one[0])
