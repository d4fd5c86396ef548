"""The plan's boundary tables of the Stacey / free-surface mode against the float64
oracle's own boundary weights (host arithmetic only, no GPU): slot layout, the node each
slot refers to, a = c alpha and the impedance factor gamma = beta / (4 dt)."""
import numpy as np
import pytest

from mun_b200.plan import boundary_slots, build_plan_arrays
from oracle import sem_oracle as so


@pytest.mark.parametrize("N,nelx,nelz", [(4, 10, 5), (3, 7, 4), (1, 9, 3)])
def test_boundary_tables_match_oracle(N, nelx, nelz):
    xmax, zmax, dt = 700.0, 400.0, 1e-4
    rec = np.array([[100.0, 10.0], [600.0, 10.0]])
    a = build_plan_arrays(0.0, xmax, 0.0, zmax, nelx, nelz, N, dt, 20, (350.0, 20.0), 10.0, 1.0, rec,
                          100.0, 3000.0, boundary="stacey")
    cfg = {"domain": {"xmin": 0.0, "xmax": xmax, "zmin": 0.0, "zmax": zmax, "nelem_x": nelx, "nelem_z": nelz},
           "time": {"total_time": 20 * dt, "dt": dt}, "source": {"position": (350.0, 20.0), "frequency": 10.0,
                                                                 "amplitude": 1.0},
           "receivers": {"positions": rec}, "method": {"polynomial_order": N, "pml_thickness": 100.0,
                                                       "boundary": "stacey"},
           "velocity": {"outside_velocity": 3000.0}}
    rng = np.random.default_rng(0)
    nxg, nzg = nelx * N + 1, nelz * N + 1
    c = 1500.0 + 1000.0 * rng.random(nxg * nzg)
    sim = so.build_sim(cfg, c, dt=dt, dt_cfl_velocity=np.full(len(c), 1.0))
    nb, gx, gz, used = boundary_slots(nelx, nelz, N)
    assert a["bnd_n"] == nb == 2 * nzg + nxg
    ref = a["bnd_ref"]
    # every absorbing-edge node below the surface appears in exactly one slot
    on_edge = (sim.extra["beta"] > 0) & ~sim.extra["top"]
    assert sorted(ref[ref >= 0].tolist()) == sorted(np.nonzero(on_edge)[0].tolist())
    k = np.nonzero(ref >= 0)[0]
    r = ref[k]
    assert np.array_equal(sim.grid[r, 0], gx[k]) and np.array_equal(sim.grid[r, 1], gz[k])
    a_oracle = 0.5 * dt * c[r] * sim.extra["beta"][r] / sim.M[r]
    assert np.allclose(c[r] * a["bnd_alpha"][k], a_oracle, rtol=1e-13, atol=0)
    assert np.allclose(a["bnd_gamma"][k], sim.extra["beta"][r] / (4 * dt), rtol=1e-13, atol=0)
    # no sponge in this mode
    assert np.all(a["tab_x"][2 * nxg:] == 0.0) and np.all(a["tab_z"][2 * nzg:] == 0.0)


def test_kernel_recurrence_in_stacey_mode_matches_oracle():
    """The kernels' one-field Stacey update w = e1 v + e2 F (e1, e2 from the plan's slot
    tables, free surface zeroed), run in float64 from the plan tables alone, against the
    oracle's three-level recurrence (1 + a) u+ = 2u - (1 - a) u- + dt^2 M^-1 (f - K u)."""
    from tests import kernel_model as km
    N, nelx, nelz, nt = 4, 10, 6, 400
    xmax, zmax = 500.0, 300.0
    rec = np.stack([np.linspace(30.0, 470.0, 9), np.full(9, 15.0)], 1)
    cfg = {"domain": {"xmin": 0.0, "xmax": xmax, "zmin": 0.0, "zmax": zmax, "nelem_x": nelx, "nelem_z": nelz},
           "time": {"total_time": 1.0, "dt": 1.0},
           "source": {"position": (250.0, 30.0), "frequency": 25.0, "amplitude": 1.0},
           "receivers": {"positions": rec},
           "method": {"polynomial_order": N, "pml_thickness": 100.0, "boundary": "stacey"},
           "velocity": {"outside_velocity": 2600.0}}
    sim0 = so.build_sim(cfg)
    x, z = sim0.coords[:, 0], sim0.coords[:, 1]
    c = 2000.0 + 300.0 * np.sin(x / 90.0) * np.cos(z / 70.0)
    sim = so.build_sim(cfg, c, dt_cfl_velocity=np.full(len(c), 2600.0))
    sim.nt = nt
    sim.src = so.ricker_source(nt, sim.dt, 25.0, 1.0)
    ref, _ = so.forward(sim, c, convention="fwdadj")
    a = build_plan_arrays(0.0, xmax, 0.0, zmax, nelx, nelz, N, sim.dt, nt, (250.0, 30.0), 25.0, 1.0, rec,
                          100.0, 2600.0, boundary="stacey")
    mine, _ = km.forward(a, c, shift=True)
    err = float(np.linalg.norm(mine - ref) / np.linalg.norm(ref))
    assert np.abs(ref[-100:]).max() > 1e-3 * np.abs(ref).max()   # the edges are reached in the window
    assert err < 1e-11, err
