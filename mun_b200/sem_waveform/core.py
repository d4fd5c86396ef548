"""``SEMSimulation`` — drop-in for MUN's ``sem_waveform.core.SEMSimulation``.

Same config dict, methods, return dicts, side effects and exceptions as the reference
(``Bspline_Coupling/SEM/sem_waveform/core.py:88-1583`` and its layered and gridded
variants ``CO2_plume/layered_model/inversion/sem_waveform/core.py``,
``CO2_plume/one_stage/single_cubic/sem_waveform/core.py``); the variant is picked from
the velocity config (``layers`` -> layered background, ``background_2d`` /
``background`` -> gridded background, otherwise inside/outside velocity).  Model
building, CFL, observation alignment and the control-point projection run on the host
in float64 as in the reference; every time loop runs on the GPU through the C ABI
(``mun_b200._lib``): forward in float32, misfit and gradient time-sum in float64.

One deliberate difference: the reference keeps the whole forward history
(``u_hist``, nt x npoints); here the forward is checkpointed and replayed, so memory is
O((nt/k + k) npoints) and results do not depend on k (bitwise).
"""
from __future__ import annotations

import collections
import os
import threading
import time
import warnings

import numpy as np
import torch

from .. import _lib
from ..obs import align_observation, misfit_window
from ..plan import SEMPlan
from ..solver import Batch, SolveSpec
from . import velocity as vel
from .mesh import create_global_mesh, find_closest_node
from .operators import precompute_sem_operators
from .receivers import receiver_matrix, circle_positions
from .boundary import setup_pml
from .sources import create_source_wavelet
from .utils import adjust_time_step_for_stability, check_cfl_condition


# Plans (device tables of one mesh / dt / nt / source / receiver set) shared by every
# simulation in the process: MUN's MCMC constructs a new simulation for each proposal
# (Bspline_Coupling/MCMC/MCMC.py:193-208), which then finds its plan here.  LRU-bounded.
# MUN's CO2 drivers call run_forward_and_adjoint from several threads at once, each on its
# own cached simulation (CO2_plume/one_stage/single_cubic/RQS_NF.py:1064-1072): the lookup, insertion and
# eviction happen under one lock.
_PLAN_CACHE = collections.OrderedDict()
_PLAN_CACHE_MAX = 64
_PLAN_LOCK = threading.Lock()


class SEMSimulation:
    def __init__(self, config, device=None):
        self.config = config
        self._validate_config()
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device() if torch.cuda.is_available() else 0)
        self._plans = {}
        self._batch = None
        self._initialize_components()
        self.visualize = self.config["output"].get("visualize", False)
        self.frames = []
        self.adj_history_dtype = self.config.get("method", {}).get("adj_history_dtype", "float64")
        if self.adj_history_dtype not in ("float32", "float64"):
            self.adj_history_dtype = "float64"

    # ------------------------------------------------------------------ config
    def _validate_config(self):
        for key in ("domain", "time", "source", "receivers", "method", "velocity", "output"):
            if key not in self.config:
                raise ValueError(f"Missing required config key: {key}")

    def _initialize_components(self):
        c = self.config
        d, tp, sp, rp, mp, vp = (c["domain"], c["time"], c["source"], c["receivers"], c["method"],
                                 c["velocity"])
        self.xmin, self.xmax = float(d["xmin"]), float(d["xmax"])
        self.zmin, self.zmax = float(d["zmin"]), float(d["zmax"])
        self.nelem_x, self.nelem_z = int(d["nelem_x"]), int(d["nelem_z"])
        self.npol = int(mp["polynomial_order"])
        self.ngll = self.npol + 1
        self.total_time = float(tp["total_time"])
        self.dt = float(tp["dt"])
        self.nt = int(np.ceil(self.total_time / self.dt))
        self.dt2 = self.dt * self.dt
        self.src_x, self.src_z = [float(v) for v in sp["position"]]
        self.src_f0 = float(sp["frequency"])
        self.src_amp = float(sp["amplitude"])
        if "positions" in rp:
            pos = np.asarray(rp["positions"], dtype=np.float64)
            if pos.ndim != 2 or pos.shape[1] != 2:
                raise ValueError("config['receivers']['positions'] must be of shape (nrec, 2)")
            self.receiver_positions = pos
            self.num_receivers = pos.shape[0]
            self.receiver_radius = None
        else:
            self.num_receivers = int(rp["num_receivers"])
            self.receiver_radius = float(rp["radius"])
            self.receiver_positions = None

        if "background_2d" in vp or "background" in vp:
            self.variant = "grid2d"
        elif "layers" in vp:
            self.variant = "layered"
        else:
            self.variant = "canonical"
        anom = vp.get("anomaly", {}) if isinstance(vp.get("anomaly", {}), dict) else {}
        if self.variant == "canonical":
            self.vmin = float(vp["inside_velocity"])
            self.vmax = float(vp["outside_velocity"])
            ctrl = vp.get("control_points", None)
            perts = vp.get("perturbations", None)
            self.anomaly_enabled = True
        else:
            self.vmin = float(vp.get("vmin", 2000.0))
            self.vmax = float(vp.get("vmax", 3000.0))
            ctrl = anom.get("control_points", vp.get("control_points", None))
            perts = anom.get("perturbations", vp.get("perturbations", None))
            self.anomaly_enabled = bool(anom.get("enabled", True))
        self.ctrl_pts_original = None if ctrl is None else np.asarray(ctrl, dtype=np.float64)
        if perts is None:
            self.true_offset = None
        else:
            a = np.asarray(perts, dtype=np.float64)
            self.true_offset = None if a.size == 0 else a
        o = c["output"]
        self.output_dir = o.get("output_dir", "sem_output")
        self.save_wavefield = bool(o.get("save_wavefield", False))
        self.save_seismograms = bool(o.get("save_seismograms", True))
        self.visualize = bool(o.get("visualize", False))

        self.global_coords, self.global_connectivity, self.node_map = create_global_mesh(
            self.xmin, self.xmax, self.zmin, self.zmax, self.nelem_x, self.nelem_z, self.npol)
        self.node_grid = self.node_map.node_grid
        self.npoints = int(len(self.global_coords))
        self.Lx, self.Lz = self.xmax - self.xmin, self.zmax - self.zmin
        self.dx_elem, self.dz_elem = self.Lx / self.nelem_x, self.Lz / self.nelem_z

        if self.variant == "layered":
            lay = vp.get("layers", {})
            self.interfaces_z = np.asarray(lay.get("interfaces_z", []), dtype=np.float64)
            self.layer_velocities = np.asarray(lay.get("velocities", []), dtype=np.float64)
            self.v_layer_background = vel.build_layered_background(
                self.global_coords, self.interfaces_z, self.layer_velocities)
        if self.variant == "grid2d":
            self._load_background(vp)

        # initial velocity for the CFL check (core.py:238-270)
        base = None
        if self.ctrl_pts_original is not None and self.anomaly_enabled:
            base = self.ctrl_pts_original.reshape(-1, 2)
            if self.true_offset is not None:
                base = base + self.true_offset.reshape(-1, 2)
        if base is not None:
            v0, _, _ = self._build_velocity(base)
        elif self.variant == "grid2d":
            v0 = self.v_background.copy()
        else:
            v0 = np.full(self.npoints, self.vmax)
        self.velocity_model = v0
        self.dt, self.nt = adjust_time_step_for_stability(
            self.velocity_model, self.dt, self.total_time, self.npol, self.dx_elem,
            self.dz_elem, self.vmax)
        self.dt2 = self.dt * self.dt
        self.time_array = np.arange(self.nt, dtype=np.float64) * self.dt
        self.src_wavelet = create_source_wavelet(self.nt, self.dt, f0=self.src_f0, t0=0.1,
                                                 gate_time=0.3, amp=self.src_amp)
        self.src_wavelet_torch = torch.from_numpy(self.src_wavelet)
        self.src_node = find_closest_node(self.src_x, self.src_z, self.global_coords)
        self.src_pos = self.global_coords[self.src_node]
        if self.receiver_positions is None:
            self.receiver_coords_sem = [tuple(p) for p in circle_positions(
                self.src_x, self.src_z, self.receiver_radius, self.num_receivers)]
        else:
            self.receiver_coords_sem = [tuple(p) for p in self.receiver_positions]
        self.R_sparse, self.R_torch = receiver_matrix(
            np.asarray(self.receiver_coords_sem), self.xmin, self.zmin, self.dx_elem, self.dz_elem,
            self.nelem_x, self.nelem_z, self.global_connectivity, self.npol, self.npoints)
        self.Gx_global, self.Gz_global, self.S_interp_global, self.w2D_global = \
            precompute_sem_operators(self.dx_elem, self.dz_elem, self.npol)
        self._setup_sponge()
        o = c["output"]
        self.roi_xmin = o.get("roi_xmin", self.xmin + 100.0)
        self.roi_xmax = o.get("roi_xmax", self.xmax - 100.0)
        self.roi_zmin = o.get("roi_zmin", self.zmin + 100.0)
        self.roi_zmax = o.get("roi_zmax", self.zmax - 100.0)
        x, z = self.global_coords[:, 0], self.global_coords[:, 1]
        self.roi_mask = ((x >= self.roi_xmin) & (x <= self.roi_xmax) &
                         (z >= self.roi_zmin) & (z <= self.roi_zmax))

    def _load_background(self, vp):
        bg = vp.get("background_2d", None) or vp.get("background", None)
        if bg is None:
            raise ValueError("velocity.background_2d is required for 2D background mode.")
        if bg.get("vp", None) is not None:
            grid = np.asarray(bg["vp"], dtype=np.float64)
        else:
            if bg.get("vp_path", None) is None:
                raise ValueError("background_2d must provide either 'vp' array or 'vp_path'.")
            grid = np.load(bg["vp_path"]).astype(np.float64)
        if bg.get("x", None) is not None:
            xg = np.asarray(bg["x"], dtype=np.float64).reshape(-1)
        elif bg.get("x_path", None) is not None:
            xg = np.load(bg["x_path"]).astype(np.float64).reshape(-1)
        else:
            xg = np.linspace(float(bg.get("xmin", self.xmin)), float(bg.get("xmax", self.xmax)),
                             int(bg.get("nx", grid.shape[1])))
        if bg.get("z", None) is not None:
            zg = np.asarray(bg["z"], dtype=np.float64).reshape(-1)
        elif bg.get("z_path", None) is not None:
            zg = np.load(bg["z_path"]).astype(np.float64).reshape(-1)
        else:
            zg = np.linspace(float(bg.get("zmin", self.zmin)), float(bg.get("zmax", self.zmax)),
                             int(bg.get("nz", grid.shape[0])))
        if xg.size < 2 or zg.size < 2:
            raise ValueError("background_2d grid x/z must have at least 2 points each.")
        if xg[0] > xg[-1]:
            xg, grid = xg[::-1], grid[:, ::-1]
        if zg[0] > zg[-1]:
            zg, grid = zg[::-1], grid[::-1, :]
        method = str(bg.get("interp", "linear"))
        self.background_2d = {"x": xg, "z": zg, "vp": grid, "interp": method}
        self.v_background = vel.build_background_from_grid(self.global_coords, xg, zg, grid,
                                                           method=method, clip=True)
        self.vmin = float(min(self.vmin, np.nanmin(self.v_background)))
        self.vmax = float(max(self.vmax, np.nanmax(self.v_background)))

    def _setup_sponge(self):
        self.pml_indices_sem, self.pml_mask_sem, self.decay_sem_torch = setup_pml(
            self.xmin, self.xmax, self.zmin, self.zmax, self.config["method"]["pml_thickness"],
            self.global_coords, self.dt, c_max=self.vmax)
        self.decay_sem = self.decay_sem_torch.numpy()

    # ------------------------------------------------------------------ model building
    def _build_velocity(self, ctrl_abs):
        """Velocity (and signed distance, extras) for absolute control points.  On a CUDA
        device the model is built there (``sem_velocity_from_curve``); the host builders
        compute the same numbers (``method.velocity_on_device = False`` selects them)."""
        vp = self.config["velocity"]
        tau, samples = float(vp["tau"]), int(vp["spline_samples"])
        anom = vp.get("anomaly", {}) if isinstance(vp.get("anomaly", {}), dict) else {}
        ctrl = np.reshape(ctrl_abs, (6, 2) if self.variant == "canonical" else (-1, 2))
        v_in = self.vmin if self.variant == "canonical" else float(anom.get("v_inside", self.vmin))
        blend = "smooth" if self.variant == "canonical" else str(anom.get("blend", "smooth"))
        if self.device.type == "cuda" and self.config["method"].get("velocity_on_device", True):
            if not hasattr(self, "_coords_dev"):
                self._coords_dev = torch.as_tensor(self.global_coords, device=self.device)
                bg = self._background()
                self._bg_dev = None if bg is None else torch.as_tensor(bg, device=self.device)
            vel_d, sd_d, us_d, nr_d = vel.build_velocity_device(
                self._coords_dev, ctrl, tau, samples, v_in, v_outside=self.vmax,
                v_background_dev=self._bg_dev, periodic=(self.variant == "grid2d"), blend=blend)
            return (vel_d.cpu().numpy(), sd_d.cpu().numpy(),
                    {"u_star": us_d.cpu().numpy(), "normal_out": nr_d.cpu().numpy()})
        if self.variant == "canonical":
            return vel.build_velocity_on_sem_nodes(self.global_coords, ctrl, self.vmin, self.vmax, tau,
                                                   samples, 7)
        if self.variant == "layered":
            return vel.build_velocity_layered_with_anomaly(
                self.global_coords, self.interfaces_z, self.layer_velocities, ctrl, v_in, tau, samples, 7,
                blend)
        return vel.build_velocity_2d_background_with_anomaly(
            self.global_coords, self.v_background, ctrl, v_in, tau, samples, 7, blend)

    def _velocity_on_device(self):
        return self.device.type == "cuda" and self.config["method"].get("velocity_on_device", True)

    def _build_velocity_dev(self, ctrl_abs, sync=False):
        """Device tensors (velocity, sd, u_star, normal) of ``_build_velocity``'s on-device
        branch, left on the GPU."""
        vp = self.config["velocity"]
        tau, samples = float(vp["tau"]), int(vp["spline_samples"])
        anom = vp.get("anomaly", {}) if isinstance(vp.get("anomaly", {}), dict) else {}
        ctrl = np.reshape(ctrl_abs, (6, 2) if self.variant == "canonical" else (-1, 2))
        v_in = self.vmin if self.variant == "canonical" else float(anom.get("v_inside", self.vmin))
        blend = "smooth" if self.variant == "canonical" else str(anom.get("blend", "smooth"))
        if not hasattr(self, "_coords_dev"):
            self._coords_dev = torch.as_tensor(self.global_coords, device=self.device)
            bg = self._background()
            self._bg_dev = None if bg is None else torch.as_tensor(bg, device=self.device)
        return vel.build_velocity_device(
            self._coords_dev, ctrl, tau, samples, v_in, v_outside=self.vmax, v_background_dev=self._bg_dev,
            periodic=(self.variant == "grid2d"), blend=blend, sync=sync)

    def _project_dev(self, ctrl_abs, dL, sd, us, nrm):
        """(S, 2K) interleaved [x0, z0, x1, z1, ...] control-point gradients on the device
        (the same projection as ``_analytical_gradient_projection_improved``)."""
        vp = self.config["velocity"]
        anom = vp.get("anomaly", {}) if isinstance(vp.get("anomaly", {}), dict) else {}
        ctrl = np.reshape(ctrl_abs, (-1, 2))
        K = ctrl.shape[0]
        if self.variant == "canonical":
            g = vel.project_ctrl_device(ctrl, False, dL, sd, us, nrm, self.vmin, float(vp["tau"]),
                                        v_background_const=self.vmax, floor_one=False)
        else:
            g = vel.project_ctrl_device(ctrl, self.variant == "grid2d", dL, sd, us, nrm,
                                        float(anom.get("v_inside", self.vmin)), float(vp["tau"]),
                                        v_background_dev=self._bg_dev, floor_one=True)
        out = torch.empty_like(g)
        out[:, 0::2] = g[:, :K]
        out[:, 1::2] = g[:, K:]
        return out

    def _background(self):
        if self.variant == "layered":
            return self.v_layer_background
        if self.variant == "grid2d":
            return self.v_background
        return None

    # ------------------------------------------------------------------ device plumbing
    def _boundary(self):
        """``method.boundary``: 'sponge' (the reference's, default) or 'stacey' (extension:
        Stacey absorbing sides and bottom, free surface on top, no sponge)."""
        b = str(self.config["method"].get("boundary", "sponge"))
        if b not in ("sponge", "stacey"):
            raise ValueError(f"method.boundary must be 'sponge' or 'stacey', got {b!r}")
        return b

    def _plan(self):
        key = (float(self.dt), int(self.nt))
        p = self._plans.get(key)
        if p is None:
            rec = np.ascontiguousarray(self.receiver_coords_sem, dtype=np.float64)
            gkey = (torch.cuda.current_device(), float(self.xmin), float(self.xmax), float(self.zmin),
                    float(self.zmax), int(self.nelem_x), int(self.nelem_z), int(self.npol), float(self.dt),
                    int(self.nt), float(self.src_x), float(self.src_z), float(self.src_f0),
                    float(self.src_amp), rec.tobytes(), float(self.config["method"]["pml_thickness"]),
                    float(self.vmax), self._boundary())
            with _PLAN_LOCK:
                p = _PLAN_CACHE.get(gkey)
                if p is not None:
                    _PLAN_CACHE.move_to_end(gkey)
            if p is None:
                p = SEMPlan(xmin=self.xmin, xmax=self.xmax, zmin=self.zmin, zmax=self.zmax,
                            nelx=self.nelem_x, nelz=self.nelem_z, npol=self.npol, dt=self.dt, nt=self.nt,
                            src_xz=(self.src_x, self.src_z), f0=self.src_f0, amp=self.src_amp,
                            receivers=rec, pml_thickness=float(self.config["method"]["pml_thickness"]),
                            sponge_cmax=self.vmax, coords=self.global_coords, node_grid=self.node_grid,
                            boundary=self._boundary())
                with _PLAN_LOCK:
                    # another thread may have built the same plan meanwhile: keep the first
                    p = _PLAN_CACHE.setdefault(gkey, p)
                    _PLAN_CACHE.move_to_end(gkey)
                    while len(_PLAN_CACHE) > _PLAN_CACHE_MAX:
                        _PLAN_CACHE.popitem(last=False)
            self._plans[key] = p
        return p

    def _get_batch(self):
        if self._batch is None:
            self._batch = Batch()
        return self._batch

    def _dev(self, a):
        return torch.as_tensor(np.asarray(a, dtype=np.float64), device=self.device)

    def _cfl_update(self):
        self.dt, self.nt = adjust_time_step_for_stability(
            self.velocity_model, self.dt, self.total_time, self.npol, self.dx_elem, self.dz_elem,
            self.vmax)
        self.dt2 = self.dt * self.dt
        self._setup_sponge()
        self.time_array = np.arange(self.nt, dtype=np.float64) * self.dt
        self.src_wavelet = create_source_wavelet(self.nt, self.dt, f0=self.src_f0, t0=0.1,
                                                 gate_time=0.3, amp=self.src_amp)
        self.src_wavelet_torch = torch.from_numpy(self.src_wavelet)

    # ------------------------------------------------------------------ forward
    def run(self, ctrl_offsets_flat=None, use_torch=True):
        """Forward simulation (core.py:334-435): rebuilds the velocity from the
        control-point offsets, applies the CFL rule, records R u before each update."""
        if self.variant == "grid2d" and (not self.anomaly_enabled or self.ctrl_pts_original is None):
            self.velocity_model = self.v_background.copy()
            self.signed_dist, self.spline_extras = None, None
        else:
            if self.ctrl_pts_original is None:
                raise ValueError("run() needs velocity.control_points")
            if ctrl_offsets_flat is None:
                if self.true_offset is not None:
                    ctrl_offsets_flat = self.true_offset.reshape(-1)
                else:
                    ctrl_offsets_flat = np.zeros(self.ctrl_pts_original.size)
            if isinstance(ctrl_offsets_flat, torch.Tensor):
                ctrl_offsets_flat = ctrl_offsets_flat.detach().cpu().numpy()
            perts = np.asarray(ctrl_offsets_flat, dtype=np.float64).reshape(-1, 2)
            ctrl_abs = self.ctrl_pts_original.reshape(-1, 2) + perts
            self.velocity_model, self.signed_dist, self.spline_extras = self._build_velocity(ctrl_abs)
        self._cfl_update()
        self.velocity_model_torch = torch.from_numpy(self.velocity_model)
        rec = self._forward_rec(self.velocity_model, shift=False)
        self.receiver_data = rec
        out = {"dt": float(self.dt), "nt": int(self.nt), "receiver_data": rec,
               "receiver_coords": self.receiver_coords_sem}
        return out

    def _forward_rec(self, velocity, shift):
        if not np.all(np.isfinite(velocity)):
            raise ValueError("[CFL] velocity_model contains non-finite values (NaN/Inf).")
        s = SolveSpec(self._plan(), self._dev(velocity), shift=shift)
        self._get_batch().run([s])
        self._check_status([s])
        return s.rec.double().cpu().numpy()

    def _check_status(self, specs):
        st = torch.cat([s.status for s in specs]).cpu().numpy()
        if np.any(st != 0):
            raise FloatingPointError(f"non-finite wavefield in {int(np.sum(st != 0))} solve(s)")

    def _forward_pred_with_velocity(self, velocity_torch):
        """Predicted receiver data for a given nodal velocity (core.py:1373-1438)."""
        v = velocity_torch.detach().cpu().numpy() if isinstance(velocity_torch, torch.Tensor) \
            else np.asarray(velocity_torch, dtype=np.float64)
        if self.num_receivers == 0:
            return None
        return self._forward_rec(v, shift=False)

    # ------------------------------------------------------------------ forward + adjoint
    def _align_observation_data(self, y_obs, obs_dt, obs_nt):
        return align_observation(y_obs, obs_dt, obs_nt, self.dt, self.nt)

    def _solve_spec(self, velocity, y_obs, obs_dt, obs_nt, sigma2, exact=False, ckpt_k=0, y_cache=None,
                    y_key=None):
        it0, it1, decim = misfit_window(self.config.get("method", {}).get("misfit_window", None),
                                        self.dt, self.nt)
        nt_eff = it1 - it0
        nt_dec = -(-nt_eff // decim)
        dt_eff = self.dt * decim
        if y_cache is not None and y_key in y_cache:
            y_dev = y_cache[y_key]
        else:
            y = np.asarray(y_obs, dtype=np.float64)
            if abs(dt_eff - obs_dt) < 1e-12 and nt_dec == obs_nt and y.shape[0] == nt_dec:
                ya = y
            else:
                ya = align_observation(y, obs_dt, obs_nt, dt_eff, nt_dec)
            if ya.shape[1] != self.num_receivers:
                raise ValueError(f"y_obs has {ya.shape[1]} receivers, expected {self.num_receivers}")
            y_dev = self._dev(ya)
            if y_cache is not None:
                y_cache[y_key] = y_dev
        v_dev = velocity if isinstance(velocity, torch.Tensor) else self._dev(velocity)
        return SolveSpec(self._plan(), v_dev, adjoint=True, exact=exact,
                         y_obs=y_dev, window=(it0, it1, decim), inv_sigma2=1.0 / sigma2,
                         ckpt_k=ckpt_k), (it0, it1)

    def run_forward_and_adjoint(self, params_dict):
        """Forward + adjoint log-likelihood and its gradient w.r.t. the control points
        (core.py:1067-1371).  Returns {'loglik', 'grad_wrt_ctrl' (2K,) interleaved
        [x0,z0,x1,z1,...], 'clean_data' (nt,nrec), 'dt', 'nt'}."""
        perts = np.asarray(params_dict["bspline_ctrl"], dtype=np.float64)
        if perts.ndim == 1:
            if perts.size % 2:
                raise ValueError(f"bspline_ctrl 1D array length {perts.size} is not even; "
                                 "cannot reshape to (K,2)")
            perts = perts.reshape(-1, 2)
        elif not (perts.ndim == 2 and perts.shape[1] == 2):
            raise ValueError(f"bspline_ctrl must be shape (2*K,) or (K,2), got {perts.shape}")
        if self.variant == "canonical" and perts.shape != (6, 2):
            raise ValueError("canonical model uses 6 control points")
        y_obs = np.asarray(params_dict["y_obs"], dtype=np.float64)
        obs_dt = float(params_dict["obs_dt"])
        obs_nt = int(params_dict["obs_nt"])
        sigma = float(params_dict.get("noise_std", 0.0))
        sigma2 = sigma * sigma + 1e-24
        dev_build = None
        if self._velocity_on_device():
            dev_build = self._build_velocity_dev(perts)
            velocity_model = dev_build[0].cpu().numpy()
            signed_dist = dev_build[1].cpu().numpy()
            extras = {"u_star": dev_build[2].cpu().numpy(), "normal_out": dev_build[3].cpu().numpy()}
        else:
            velocity_model, signed_dist, extras = self._build_velocity(perts)
        self.velocity_model, self.signed_dist, self.spline_extras = velocity_model, signed_dist, extras
        self.velocity_model_torch = torch.from_numpy(velocity_model)
        self._cfl_update()
        mode = self.config.get("method", {}).get("adjoint_mode", "reference")
        spec, (it0, it1) = self._solve_spec(dev_build[0] if dev_build is not None else velocity_model,
                                            y_obs, obs_dt, obs_nt, sigma2, exact=(mode == "exact"))
        self._get_batch().run([spec])
        self._check_status([spec])
        loglik = float(spec.loglik.item())
        dJ_dv = spec.grad.cpu().numpy()
        clean = spec.rec.double().cpu().numpy()[it0:it1]
        self.dJ_dv = dJ_dv
        dL_dv = -dJ_dv
        if dev_build is not None:  # projection on the device, as in the batch path
            G = self._project_dev(perts, -spec.grad[None], dev_build[1][None], dev_build[2][None],
                                  dev_build[3][None]).cpu().numpy()[0]
            proj = {"grad_ctrl_x": G[0::2], "grad_ctrl_z": G[1::2]}
        else:
            proj = self._analytical_gradient_projection_improved(
                dL_dv_np=dL_dv, bspline_ctrl=perts, tau=float(self.config["velocity"]["tau"]),
                signed_dist=signed_dist, extras=extras,
                spline_samples=int(self.config["velocity"]["spline_samples"]))
        if self.config["method"].get("VERIFY_PROJECTION", False):
            self._verify_projection(perts, dL_dv, proj, sigma2, obs_dt, obs_nt, y_obs)
        gx = np.asarray(proj["grad_ctrl_x"], dtype=np.float64).reshape(-1)
        gz = np.asarray(proj["grad_ctrl_z"], dtype=np.float64).reshape(-1)
        g = np.empty(2 * gx.size)
        g[0::2], g[1::2] = gx, gz
        return {"loglik": loglik, "grad_wrt_ctrl": g, "clean_data": clean, "dt": float(self.dt),
                "nt": int(self.nt)}

    def run_forward_and_adjoint_batch(self, params_list, ckpt_k=0):
        """Many ``run_forward_and_adjoint`` requests in one batched launch sequence.
        All requests share this simulation's mesh; dt follows the CFL rule applied to
        the fastest model of the batch (the reference would lower ``self.dt`` the same
        way when the calls run one after another).  With the on-device velocity builder
        the models, solves and control-point projection stay on the GPU; only the
        per-sample outputs come back (one copy each for all samples)."""
        if not self._velocity_on_device():
            return self._run_forward_and_adjoint_batch_host(params_list, ckpt_k)
        ctrls = [np.asarray(prm["bspline_ctrl"], dtype=np.float64).reshape(-1, 2) for prm in params_list]
        builds = [self._build_velocity_dev(c) for c in ctrls]
        V = torch.stack([b[0] for b in builds])
        imax = int(torch.argmax(V.max(dim=1).values).item())
        self.velocity_model = V[imax].cpu().numpy()
        self._cfl_update()
        specs, wins, ycache = [], [], {}
        for i, prm in enumerate(params_list):
            sigma = float(prm.get("noise_std", 0.0))
            key = (id(prm["y_obs"]), float(prm["obs_dt"]), int(prm["obs_nt"]))
            sp, win = self._solve_spec(V[i], prm["y_obs"], float(prm["obs_dt"]), int(prm["obs_nt"]),
                                       sigma * sigma + 1e-24, ckpt_k=ckpt_k, y_cache=ycache, y_key=key)
            specs.append(sp)
            wins.append(win)
        self._get_batch().run(specs)
        self._check_status(specs)
        dL = -torch.stack([sp.grad for sp in specs])
        G = self._project_dev(ctrls[0], dL, torch.stack([b[1] for b in builds]),
                              torch.stack([b[2] for b in builds]), torch.stack([b[3] for b in builds])).cpu().numpy()
        ll = torch.cat([sp.loglik for sp in specs]).cpu().numpy()
        it0, it1 = wins[0]
        rec = torch.stack([sp.rec for sp in specs]).double().cpu().numpy()
        return [{"loglik": float(ll[i]), "grad_wrt_ctrl": G[i], "clean_data": rec[i, it0:it1],
                 "dt": float(self.dt), "nt": int(self.nt)} for i in range(len(specs))]

    def _run_forward_and_adjoint_batch_host(self, params_list, ckpt_k=0):
        """Batch path with the host velocity builders and host projection."""
        builds = []
        for prm in params_list:
            perts = np.asarray(prm["bspline_ctrl"], dtype=np.float64).reshape(-1, 2)
            builds.append((perts,) + tuple(self._build_velocity(perts)))
        self.velocity_model = builds[int(np.argmax([np.max(b[1]) for b in builds]))][1]
        self._cfl_update()
        specs, wins = [], []
        for (perts, v, sd, ex), prm in zip(builds, params_list):
            sigma = float(prm.get("noise_std", 0.0))
            sp, win = self._solve_spec(v, prm["y_obs"], float(prm["obs_dt"]), int(prm["obs_nt"]),
                                       sigma * sigma + 1e-24, ckpt_k=ckpt_k)
            specs.append(sp)
            wins.append(win)
        self._get_batch().run(specs)
        self._check_status(specs)
        outs = []
        tau = float(self.config["velocity"]["tau"])
        for (perts, v, sd, ex), sp, (it0, it1) in zip(builds, specs, wins):
            dL = -sp.grad.cpu().numpy()
            proj = self._analytical_gradient_projection_improved(dL, perts, tau, sd, ex)
            gx, gz = proj["grad_ctrl_x"].reshape(-1), proj["grad_ctrl_z"].reshape(-1)
            g = np.empty(2 * gx.size)
            g[0::2], g[1::2] = gx, gz
            outs.append({"loglik": float(sp.loglik.item()), "grad_wrt_ctrl": g,
                         "clean_data": sp.rec.double().cpu().numpy()[it0:it1],
                         "dt": float(self.dt), "nt": int(self.nt)})
        return outs

    def run_forward_only_for_loglik(self, ctrl12, sigma2, obs_dt, obs_nt, y_obs):
        """Log-likelihood for FD checks (core.py:1440-1492): velocity from the control
        points, forward with receivers read before each update, no state change."""
        perts = np.asarray(ctrl12, dtype=np.float64).reshape(-1, 2)
        v, _, _ = self._build_velocity(perts)
        d = self._forward_pred_with_velocity(torch.from_numpy(v))
        if d is None:
            return -0.0
        if abs(self.dt - obs_dt) < 1e-12 and self.nt == obs_nt:
            r = d - np.asarray(y_obs, dtype=np.float64)
        else:
            r = (align_observation(d, self.dt, self.nt, self.dt, self.nt)
                 - align_observation(y_obs, obs_dt, obs_nt, self.dt, self.nt))
        return -0.5 * float(np.sum(r * r)) / float(sigma2)

    def dot_test_nodes_fd(self, dJ_dc_torch, y_obs, obs_dt, obs_nt, sigma, nvec=1, eps=1e-4,
                          seed=0, use_roi=True, verbose=True):
        """<dJ/dc, dc> against [J(c+eps dc) - J(c-eps dc)]/(2 eps) (core.py:1494-1551)."""
        y = np.asarray(y_obs, dtype=np.float64)
        if abs(obs_dt - self.dt) > 1e-15 or int(obs_nt) != int(self.nt):
            y = align_observation(y, obs_dt, obs_nt, self.dt, self.nt)
        sigma2 = float(sigma) ** 2 + 1e-24
        rng = np.random.RandomState(seed)
        c0 = np.asarray(self.velocity_model, dtype=np.float64)
        roi = np.asarray(self.roi_mask, dtype=bool) if use_roi else np.ones(self.npoints, bool)
        g = dJ_dc_torch.detach().cpu().numpy() if isinstance(dJ_dc_torch, torch.Tensor) else \
            np.asarray(dJ_dc_torch, dtype=np.float64)
        results = []
        for _ in range(int(nvec)):
            delta = np.zeros(self.npoints)
            idx = np.where(roi)[0]
            v = rng.randn(idx.size)
            v /= np.linalg.norm(v) + 1e-24
            delta[idx] = v
            lhs = float(np.dot(g, delta))
            rp = self._forward_pred_with_velocity(torch.from_numpy(c0 + eps * delta)) - y
            rm = self._forward_pred_with_velocity(torch.from_numpy(c0 - eps * delta)) - y
            Jp = 0.5 / sigma2 * float(np.sum(rp * rp))
            Jm = 0.5 / sigma2 * float(np.sum(rm * rm))
            rhs = (Jp - Jm) / (2.0 * eps)
            results.append((lhs, rhs, lhs / (rhs + 1e-30)))
        return results

    # ------------------------------------------------------------------ projection
    def _analytical_gradient_projection_improved(self, dL_dv_np, bspline_ctrl, tau, signed_dist,
                                                 extras, spline_samples=200):
        """dL/dv -> dL/d(control points): sigmoid slope x outward normal x curve basis
        at the closest-point parameter (core.py:902-970; layered core.py:1047-1117;
        gridded core.py:1128-1202)."""
        ctrl = np.asarray(bspline_ctrl, dtype=np.float64).reshape(-1, 2)
        K = ctrl.shape[0]
        dL = np.asarray(dL_dv_np, dtype=np.float64).reshape(-1)
        sd = np.asarray(signed_dist, dtype=np.float64).reshape(-1)
        u = np.asarray(extras["u_star"], dtype=np.float64).reshape(-1)
        nrm = np.asarray(extras["normal_out"], dtype=np.float64).reshape(-1, 2)
        tau_safe = max(float(tau), 1e-12)
        sig = 1.0 / (1.0 + np.exp(np.clip(sd / tau_safe, -50.0, 50.0)))
        if self.variant == "canonical":
            dv = (self.vmin - self.vmax) * sig * (1.0 - sig) * (-1.0 / tau_safe)
            mask = np.abs(dv) > 1e-8 * (self.vmax - self.vmin)
        else:
            anom = self.config["velocity"].get("anomaly", {})
            v_in = float(anom.get("v_inside", self.vmin))
            bgv = self._background()
            dv = (v_in - bgv) * sig * (1.0 - sig) * (-1.0 / tau_safe)
            mask = np.abs(dv) > 1e-8 * np.maximum(1.0, np.abs(v_in - bgv))
        if not np.any(mask):
            return {"grad_ctrl_x": np.zeros(K), "grad_ctrl_z": np.zeros(K)}
        w = (dL[mask] * dv[mask])[:, None]
        B = self._curve_basis(ctrl, u[mask])
        return {"grad_ctrl_x": np.sum(w * B * nrm[mask, 0:1], axis=0),
                "grad_ctrl_z": np.sum(w * B * nrm[mask, 1:2], axis=0)}

    def _curve_basis(self, ctrl, u):
        """Basis of the free control points at curve parameters u (duplicated closing
        controls folded back onto the points they copy)."""
        K = ctrl.shape[0]
        if self.variant == "grid2d":
            sp = vel.closed_spline_periodic(ctrl)
            lo, hi = sp.lo, sp.hi
            t = np.clip(lo + np.mod(u, 1.0) * (hi - lo), lo, np.nextafter(hi, lo))
            Bc = sp.basis_matrix(t)
            B = Bc[:, :K].copy()
            for j in range(Bc.shape[1] - K):
                B[:, j] += Bc[:, K + j]
            return B
        sp = vel.closed_spline_clamped(ctrl)
        Bc = sp.basis_matrix(u)
        B = Bc[:, :K].copy()
        B[:, 0] += Bc[:, K:].sum(axis=1)
        return B

    def _finite_difference_gradient_projection(self, perturbations, dJ_dv, spline_samples, tau,
                                               fd_eps):
        ctrl = np.asarray(perturbations, dtype=np.float64).reshape(-1, 2)
        K = ctrl.shape[0]
        out = np.zeros(2 * K)
        for j in range(2 * K):
            dp = np.zeros_like(ctrl)
            dp[j % K, j // K] = fd_eps
            vp_, _, _ = self._build_velocity(ctrl + dp)
            vm_, _, _ = self._build_velocity(ctrl - dp)
            out[j] = float(np.sum(np.asarray(dJ_dv) * (vp_ - vm_) / (2.0 * fd_eps)))
        return out

    def _verify_projection(self, perts, dL_dv, proj, sigma2, obs_dt, obs_nt, y_obs):
        pa = np.concatenate([proj["grad_ctrl_x"], proj["grad_ctrl_z"]])
        pf = -self._finite_difference_gradient_projection(
            perts, dL_dv, int(self.config["velocity"]["spline_samples"]),
            float(self.config["velocity"]["tau"]), 1e-6)
        print("\nPer-dimension gradient comparison:")
        for i in range(len(pa)):
            ratio = pa[i] / pf[i] if pf[i] != 0 else float("inf")
            print(f"{i:2d}   | {pa[i]:14.6e} | {pf[i]:14.6e} | {ratio:11.3f}")


def run_forward_and_adjoint_sources(sims, params_list):
    """Several ``run_forward_and_adjoint`` requests on different simulations (e.g. one
    per source position, as MUN's multi-source likelihood builds them:
    ``CO2_plume/one_stage/single_cubic/RQS_NF.py:1028-1091``) in one batched launch
    sequence instead of one solve per thread.  Each simulation keeps its own plan, CFL
    update and side effects; the returned dicts are those of the separate calls, bitwise.
    The simulations must live on one CUDA device and build their velocity on it."""
    if len(sims) != len(params_list):
        raise ValueError("one parameter dict per simulation")
    if not sims:
        return []
    for s in sims:
        if not s._velocity_on_device():
            raise ValueError("run_forward_and_adjoint_sources needs the on-device velocity builder")
    reqs = []
    for sim, prm in zip(sims, params_list):
        perts = np.asarray(prm["bspline_ctrl"], dtype=np.float64).reshape(-1, 2)
        build = sim._build_velocity_dev(perts)
        sim.velocity_model = build[0].cpu().numpy()
        sim.signed_dist = build[1].cpu().numpy()
        sim.spline_extras = {"u_star": build[2].cpu().numpy(), "normal_out": build[3].cpu().numpy()}
        sim.velocity_model_torch = torch.from_numpy(sim.velocity_model)
        sim._cfl_update()
        sigma = float(prm.get("noise_std", 0.0))
        mode = sim.config.get("method", {}).get("adjoint_mode", "reference")
        spec, win = sim._solve_spec(build[0], prm["y_obs"], float(prm["obs_dt"]), int(prm["obs_nt"]),
                                    sigma * sigma + 1e-24, exact=(mode == "exact"))
        reqs.append((sim, perts, build, spec, win))
    specs = [r[3] for r in reqs]
    sims[0]._get_batch().run(specs)
    for sim, _, _, spec, _ in reqs:
        sim._check_status([spec])
    outs = []
    for sim, perts, build, spec, (it0, it1) in reqs:
        sim.dJ_dv = spec.grad.cpu().numpy()
        G = sim._project_dev(perts, -spec.grad[None], build[1][None], build[2][None], build[3][None])
        outs.append({"loglik": float(spec.loglik.item()), "grad_wrt_ctrl": G.cpu().numpy()[0],
                     "clean_data": spec.rec.double().cpu().numpy()[it0:it1], "dt": float(sim.dt),
                     "nt": int(sim.nt)})
    return outs
