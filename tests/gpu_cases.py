"""Helpers shared by the GPU tests: plans and device inputs built from golden configs."""
import numpy as np
import torch

from mun_b200 import SEMPlan
from mun_b200.obs import align_observation


def receivers_of(cfg):
    rc = cfg["receivers"]
    if "positions" in rc:
        return np.asarray(rc["positions"], dtype=np.float64)
    sx, sz = cfg["source"]["position"]
    ang = np.linspace(0, 2 * np.pi, int(rc["num_receivers"]), endpoint=False)
    return np.stack([sx + rc["radius"] * np.cos(ang), sz + rc["radius"] * np.sin(ang)], 1)


def sponge_cmax(cfg):
    v = cfg["velocity"]
    return float(v.get("outside_velocity", v.get("vmax", 3000.0)))


def plan_for(cfg, dt, nt):
    d = cfg["domain"]
    return SEMPlan(xmin=d["xmin"], xmax=d["xmax"], zmin=d["zmin"], zmax=d["zmax"],
                   nelx=d["nelem_x"], nelz=d["nelem_z"], npol=cfg["method"]["polynomial_order"],
                   dt=float(dt), nt=int(nt), src_xz=cfg["source"]["position"],
                   f0=cfg["source"]["frequency"], amp=cfg["source"]["amplitude"],
                   receivers=receivers_of(cfg), pml_thickness=cfg["method"]["pml_thickness"],
                   sponge_cmax=sponge_cmax(cfg))


def dev(x):
    return torch.as_tensor(np.asarray(x, dtype=np.float64), device="cuda")


def aligned_obs(g):
    if "obs_dt" in g:
        return align_observation(g["y_obs"], float(g["obs_dt"]), int(g["obs_nt"]),
                                 float(g["dt"]), int(g["nt"]))
    return np.asarray(g["y_obs"], dtype=np.float64)
