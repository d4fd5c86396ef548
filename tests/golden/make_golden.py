"""Generate golden fixtures by running MUN's own ``sem_waveform`` package.

Run where the MUN sources are, with their root in ``MUN_REFERENCE``; the fixtures it
writes are committed so that nothing else needs the reference at run time:

    MUN_REFERENCE=/path/to/MUN python tests/golden/make_golden.py [case ...]

``matplotlib`` and ``imageio`` are not installed here.  The reference imports them at
module level (``core.py:7,10``) but its solver never calls them; the only arithmetic
use is ``matplotlib.path.Path.contains_points`` for the inside/outside sign of the
signed distance (``velocity.py``).  Stub modules are injected into ``sys.modules``;
the ``Path`` stub restates ``contains_points`` as an even-odd ray cast, which agrees
with matplotlib for every point farther than ``radius`` (1e-12) from the polygon.

Cases (each one ``.npz``):

* ``layered_cfg0``   layered-model package (``CO2_plume/layered_model/inversion``):
  the 2000x1000 m, 50 m-element, order-4 model of the plain CPU-runnable workload,
  padded by the 200 m sponge on every side as MUN's CO2 drivers pad their models
  (48x28 elements over [-200,2200]x[-200,1200]) so that the source (1000,20) and the
  50 receivers at z=10 lie outside the sponge; 2000 steps at the CFL limit, 3-layer
  1500/2200/3000 m/s background (interfaces 300/650 m) with a closed-spline 2400 m/s
  anomaly at 110-250 m depth (shallow enough to be seen within 0.33 s).
  ``run()`` and ``run_forward_and_adjoint()`` outputs, node-space dL/dv (captured
  from the projection hook), control-point gradient.
* ``circle_n5``      canonical package (``Bspline_Coupling/SEM``): order 5, circle
  receivers, inside/outside spline velocity, 400 steps.
* ``inject_n{1,2,3,6}`` layered package with a nodal velocity injected in place of
  the model builder (seeded smooth random field), tiny meshes, 150-250 steps, with
  observations on a different time grid (exercises the alignment path) and one
  node-space FD dot test (``dot_test_nodes_fd``).
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys
import types
from pathlib import Path as _P

import numpy as np

OUT = _P(__file__).resolve().parent


# ---------------------------------------------------------------- stub modules
def _install_stubs():
    class Path:  # even-odd crossing test standing in for matplotlib.path.Path
        def __init__(self, vertices, closed=False):
            self.v = np.asarray(vertices, dtype=np.float64)

        def contains_points(self, pts, radius=0.0):
            pts = np.asarray(pts, dtype=np.float64)
            x, y = pts[:, 0], pts[:, 1]
            vx, vy = self.v[:, 0], self.v[:, 1]
            wx, wy = np.roll(vx, -1), np.roll(vy, -1)
            inside = np.zeros(len(pts), dtype=bool)
            for ax, ay, bx, by in zip(vx, vy, wx, wy):
                cond = (ay > y) != (by > y)
                with np.errstate(divide="ignore", invalid="ignore"):
                    xc = ax + (y - ay) * (bx - ax) / (by - ay)
                inside ^= cond & (x < xc)
            return inside

    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    mpath = types.ModuleType("matplotlib.path")
    mpath.Path = Path
    mpl.pyplot = plt
    mpl.path = mpath
    mpl.use = lambda *a, **k: None
    for name in ("figure", "subplots", "close", "show", "pause", "savefig", "plot", "colorbar",
                 "tight_layout", "title", "xlabel", "ylabel", "legend", "imshow", "scatter",
                 "ion", "ioff", "draw", "clf", "gca", "gcf"):
        setattr(plt, name, lambda *a, **k: None)
    imageio = types.ModuleType("imageio")
    imageio.mimsave = lambda *a, **k: None
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)
    sys.modules.setdefault("matplotlib.path", mpath)
    sys.modules.setdefault("imageio", imageio)


def _load(pkg_dir: _P, name: str):
    spec = importlib.util.spec_from_file_location(name, pkg_dir / "__init__.py",
                                                  submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def _cfl_dt(npol, dx, dz, cmax):
    return 0.35 * (min(dx, dz) / (npol + 1)) / (cmax * (npol + 1) * np.sqrt(2.0))


def _capture_projection(core_mod):
    """Wrap SEMSimulation._analytical_gradient_projection_improved to record dL/dv."""
    cap = {}
    orig = core_mod.SEMSimulation._analytical_gradient_projection_improved

    def hook(self, dL_dv_np, *a, **k):
        cap["dL_dv"] = np.array(dL_dv_np, dtype=np.float64)
        cap["velocity"] = np.array(self.velocity_model, dtype=np.float64)
        return orig(self, dL_dv_np, *a, **k)

    core_mod.SEMSimulation._analytical_gradient_projection_improved = hook
    return cap


# ---------------------------------------------------------------- cases
def layered_cfg0(L):
    core = sys.modules[L.__name__ + ".core"]
    cap = _capture_projection(core)
    npol, nelx, nelz = 4, 48, 28
    dx, dz = 2400.0 / nelx, 1400.0 / nelz
    dt = _cfl_dt(npol, dx, dz, 3000.0)
    nt = 2000
    rec = np.stack([np.linspace(0.0, 2000.0, 50), np.full(50, 10.0)], axis=1)
    # a shallow anomaly: its reflections reach the receivers within 2000 steps (0.33 s)
    ctrl = np.array([[880.0, 140.0], [1000.0, 110.0], [1120.0, 140.0],
                     [1140.0, 210.0], [1000.0, 250.0], [860.0, 210.0]])
    cfg = {
        "domain": {"xmin": -200.0, "xmax": 2200.0, "zmin": -200.0, "zmax": 1200.0,
                   "nelem_x": nelx, "nelem_z": nelz},
        "time": {"total_time": (nt - 0.5) * dt, "dt": 1.0},
        "source": {"position": (1000.0, 20.0), "frequency": 10.0, "amplitude": 1.0},
        "receivers": {"positions": rec.tolist()},
        "method": {"polynomial_order": npol, "pml_thickness": 200.0},
        "velocity": {"vmin": 1500.0, "vmax": 3000.0, "control_points": ctrl.tolist(),
                     "tau": 10.0, "spline_samples": 400,
                     "layers": {"interfaces_z": [300.0, 650.0],
                                "velocities": [1500.0, 2200.0, 3000.0]},
                     "anomaly": {"v_inside": 2400.0, "blend": "smooth"}},
        "output": {"visualize": False, "save_wavefield": False},
    }
    sim = L.SEMSimulation(cfg)
    run = sim.run(ctrl_offsets_flat=np.zeros(12))
    dt_run, nt_run = sim.dt, sim.nt
    assert sim.nt == nt, sim.nt
    true_ctrl = ctrl + np.array([[20.0, -15.0], [0.0, -25.0], [-10.0, 10.0],
                                 [15.0, 0.0], [0.0, 20.0], [-20.0, 5.0]])
    obs = sim.run_forward_and_adjoint({"bspline_ctrl": true_ctrl.reshape(-1), "y_obs":
                                       np.zeros((nt, 50)), "obs_dt": sim.dt, "obs_nt": nt,
                                       "noise_std": 1e-9, "verbose": False})
    y = obs["clean_data"]
    vel_true = cap["velocity"].copy()
    res = sim.run_forward_and_adjoint({"bspline_ctrl": ctrl.reshape(-1), "y_obs": y,
                                       "obs_dt": sim.dt, "obs_nt": nt, "noise_std": 1e-9,
                                       "verbose": False})
    return cfg, dict(
        velocity=cap["velocity"], velocity_true=vel_true,
        dt=sim.dt, nt=sim.nt, dt_run=dt_run, nt_run=nt_run, rec_run=run["receiver_data"], y_obs=y,
        clean=res["clean_data"], loglik=res["loglik"], dL_dv=cap["dL_dv"],
        grad_ctrl=res["grad_wrt_ctrl"], sigma=1e-9, ctrl=ctrl, ctrl_true=true_ctrl,
        signed_dist=sim.signed_dist, src_node=sim.src_node)


def circle_n5(B):
    core = sys.modules[B.__name__ + ".core"]
    cap = _capture_projection(core)
    npol, nelx, nelz = 5, 24, 24
    nt = 400
    cfg = {
        "domain": {"xmin": -600.0, "xmax": 600.0, "zmin": -600.0, "zmax": 600.0,
                   "nelem_x": nelx, "nelem_z": nelz},
        "time": {"total_time": nt * 1.0e-4 - 1e-9, "dt": 1.0e-4},
        "source": {"position": (0.0, 0.0), "frequency": 20.0, "amplitude": 1.0},
        "receivers": {"num_receivers": 24, "radius": 350.0},
        "method": {"polynomial_order": npol, "pml_thickness": 150.0},
        "velocity": {"inside_velocity": 2000.0, "outside_velocity": 3000.0,
                     "control_points": [[-100, -100], [100, -100], [150, -50],
                                        [200, 0], [0, 200], [-200, 100]],
                     "perturbations": np.zeros((6, 2)).tolist(),
                     "tau": 10.0, "spline_samples": 400},
        "output": {"visualize": False, "save_wavefield": False},
    }
    sim = B.SEMSimulation(cfg)
    run = sim.run()
    dt_run, nt_run = sim.dt, sim.nt
    vel_run = np.array(sim.velocity_model, dtype=np.float64)
    ctrl0 = np.asarray(cfg["velocity"]["control_points"], dtype=np.float64)
    y = sim.run_forward_and_adjoint({"bspline_ctrl": (ctrl0 + 25.0).reshape(-1),
                                     "y_obs": np.zeros((sim.nt, 24)), "obs_dt": sim.dt,
                                     "obs_nt": sim.nt, "noise_std": 0.0,
                                     "verbose": False})["clean_data"]
    res = sim.run_forward_and_adjoint({"bspline_ctrl": ctrl0.reshape(-1), "y_obs": y,
                                       "obs_dt": sim.dt, "obs_nt": sim.nt,
                                       "noise_std": 1e-8, "verbose": False})
    return cfg, dict(coords=sim.global_coords, velocity=cap["velocity"], dt=sim.dt, nt=sim.nt,
                     dt_run=dt_run, nt_run=nt_run, velocity_run=vel_run,
                     rec_run=run["receiver_data"], y_obs=y, clean=res["clean_data"],
                     loglik=res["loglik"], dL_dv=cap["dL_dv"], grad_ctrl=res["grad_wrt_ctrl"],
                     sigma=1e-8, ctrl=ctrl0, signed_dist=sim.signed_dist, src_node=sim.src_node)


def _smooth_field(coords, seed, mean, amp):
    rng = np.random.default_rng(seed)
    x, z = coords[:, 0], coords[:, 1]
    f = np.zeros(len(coords))
    for _ in range(6):
        kx, kz = rng.uniform(0.002, 0.01, 2)
        ph = rng.uniform(0, 2 * np.pi, 2)
        f += np.sin(kx * x + ph[0]) * np.cos(kz * z + ph[1])
    return mean + amp * f / 6.0


def inject(L, npol, nelx, nelz, nt, seed):
    core = sys.modules[L.__name__ + ".core"]
    cap = _capture_projection(core)
    state = {}

    def fake_builder(nodes_xy, **kw):
        v = state["v"]
        n = len(v)
        ex = {"u_star": np.zeros(n), "closest": np.zeros((n, 2)), "tangent": np.zeros((n, 2)),
              "normal_out": np.zeros((n, 2))}
        return v.copy(), np.full(n, 1e6), ex

    core.build_velocity_layered_with_anomaly = fake_builder
    Lx, Lz = 40.0 * nelx, 40.0 * nelz
    rng = np.random.default_rng(seed)
    nrec = 7
    rec = np.stack([rng.uniform(0.2 * Lx, 0.8 * Lx, nrec), rng.uniform(0.1 * Lz, 0.7 * Lz, nrec)], 1)
    rec[0] = [0.5 * Lx, 0.5 * Lz]               # one receiver exactly on a node line
    cfg = {
        "domain": {"xmin": 0.0, "xmax": Lx, "zmin": 0.0, "zmax": Lz,
                   "nelem_x": nelx, "nelem_z": nelz},
        "time": {"total_time": 0.0, "dt": 1.0},
        "source": {"position": (0.37 * Lx, 0.41 * Lz), "frequency": 25.0, "amplitude": 2.0},
        "receivers": {"positions": rec.tolist()},
        "method": {"polynomial_order": npol, "pml_thickness": 100.0},
        "velocity": {"vmin": 1500.0, "vmax": 2600.0, "control_points": [[0, 0]] * 6,
                     "tau": 10.0, "spline_samples": 50,
                     "layers": {"interfaces_z": [], "velocities": [2000.0]},
                     "anomaly": {"v_inside": 2000.0}},
        "output": {"visualize": False, "save_wavefield": False},
    }
    dx, dz = Lx / nelx, Lz / nelz
    dt = _cfl_dt(npol, dx, dz, 2600.0)
    cfg["time"]["total_time"] = (nt - 0.5) * dt
    # build the mesh once to know the node coordinates
    coords, _, _ = sys.modules[L.__name__ + ".mesh"].create_global_mesh(
        0.0, Lx, 0.0, Lz, nelx, nelz, npol)
    state["v"] = np.clip(_smooth_field(np.asarray(coords), seed, 2100.0, 450.0), 1500.0, 2600.0)
    sim = L.SEMSimulation(cfg)
    run = sim.run(ctrl_offsets_flat=np.zeros(12))
    dt_run, nt_run = sim.dt, sim.nt
    v_obs = np.clip(_smooth_field(np.asarray(coords), seed + 100, 2100.0, 450.0), 1500.0, 2600.0)
    state["v"] = v_obs
    y_native = sim.run_forward_and_adjoint({"bspline_ctrl": np.zeros(12), "y_obs":
                                            np.zeros((sim.nt, nrec)), "obs_dt": sim.dt,
                                            "obs_nt": sim.nt, "noise_std": 0.0,
                                            "verbose": False})["clean_data"]
    # observations on a coarser grid (1.5 dt) -> exercises _align_observation_data
    obs_dt = 1.5 * sim.dt
    obs_nt = int(sim.nt / 1.5)
    t_obs = np.arange(obs_nt) * obs_dt
    t_sim = np.arange(sim.nt) * sim.dt
    y_obs = np.stack([np.interp(t_obs, t_sim, y_native[:, r]) for r in range(nrec)], 1)
    state["v"] = np.clip(_smooth_field(np.asarray(coords), seed, 2100.0, 450.0), 1500.0, 2600.0)
    res = sim.run_forward_and_adjoint({"bspline_ctrl": np.zeros(12), "y_obs": y_obs,
                                       "obs_dt": obs_dt, "obs_nt": obs_nt, "noise_std": 3e-9,
                                       "verbose": False})
    import torch
    dJ = torch.from_numpy(-cap["dL_dv"])
    dot = sim.dot_test_nodes_fd(dJ, y_obs, obs_dt, obs_nt, 3e-9, nvec=1, eps=1e-2, seed=seed,
                                use_roi=False, verbose=False)
    return cfg, dict(coords=sim.global_coords, velocity=state["v"], dt=sim.dt, nt=sim.nt,
                     dt_run=dt_run, nt_run=nt_run, rec_run=run["receiver_data"], y_obs=y_obs, obs_dt=obs_dt, obs_nt=obs_nt,
                     clean=res["clean_data"], loglik=res["loglik"], dL_dv=cap["dL_dv"],
                     sigma=3e-9, src_node=sim.src_node,
                     dot_lhs=dot[0][0], dot_rhs=dot[0][1], dot_seed=seed, dot_eps=1e-2)


def _save(name, cfg, data):
    meta = {"config": cfg, "numpy": np.__version__,
            "scipy": __import__("scipy").__version__, "torch": __import__("torch").__version__}
    np.savez_compressed(OUT / f"{name}.npz", meta=json.dumps(meta, default=float), **data)
    print("wrote", name, {k: np.shape(v) for k, v in data.items()})


def main():
    global REF
    if not os.environ.get("MUN_REFERENCE"):
        sys.exit("set MUN_REFERENCE to the root of the MUN sources")
    REF = _P(os.environ["MUN_REFERENCE"])
    _install_stubs()
    import torch
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    L = _load(REF / "CO2_plume/layered_model/inversion/sem_waveform", "mun_ref_layered")
    B = _load(REF / "Bspline_Coupling/SEM/sem_waveform", "mun_ref_canonical")
    which = sys.argv[1:] or ["layered_cfg0", "circle_n5", "inject"]
    if "layered_cfg0" in which:
        _save("layered_cfg0", *layered_cfg0(L))
    if "circle_n5" in which:
        _save("circle_n5", *circle_n5(B))
    if "inject" in which:
        for npol, nx, nz, nt, seed in ((1, 30, 20, 250, 11), (2, 16, 10, 200, 12),
                                       (3, 12, 9, 200, 13), (6, 7, 5, 150, 14)):
            L = _load(REF / "CO2_plume/layered_model/inversion/sem_waveform",
                      f"mun_ref_layered_{npol}")
            _save(f"inject_n{npol}", *inject(L, npol, nx, nz, nt, seed))


if __name__ == "__main__":
    main()
