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
