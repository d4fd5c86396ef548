"""The float64 oracle's extension boundary mode (Stacey absorbing sides and bottom, free
surface on top; the reference has only the all-sides sponge):

* its adjoint gradient is the exact derivative of its own log-likelihood: central
  differences along random directions, one of them supported on the absorbing-boundary
  nodes only (where the boundary-impedance term of the gradient lives), agree to 1e-5
  (without that term the edge direction's derivative has the wrong sign);
* the absorbing edges reflect little: against a run on a domain three times as wide and
  deep (whose edges are too far to be seen in the window), the energy the Stacey edges
  send back to the receivers is under 1 % of what rigid edges send back (4e-4 here).
"""
import numpy as np

from oracle import sem_oracle as so


def _cfg(xmin=0.0, xmax=1000.0, zmax=500.0, nelx=20, nelz=10, T=0.3, nrec=11):
    return {"domain": {"xmin": xmin, "xmax": xmax, "zmin": 0.0, "zmax": zmax, "nelem_x": nelx,
                       "nelem_z": nelz},
            "time": {"total_time": T, "dt": 1.0},
            "source": {"position": (500.0, 25.0), "frequency": 15.0, "amplitude": 1.0},
            "receivers": {"positions": np.stack([np.linspace(100.0, 900.0, nrec), np.full(nrec, 12.5)], 1)},
            "method": {"polynomial_order": 4, "pml_thickness": 100.0, "boundary": "stacey"},
            "velocity": {"outside_velocity": 2600.0}}


def test_stacey_adjoint_matches_finite_differences():
    cfg = _cfg(nelx=12, nelz=8, T=0.25, xmax=600.0, zmax=400.0, nrec=7)
    cfg["source"]["position"] = (300.0, 25.0)
    cfg["receivers"]["positions"][:, 0] = np.linspace(40.0, 560.0, 7)
    sim0 = so.build_sim(cfg)
    x, z = sim0.coords[:, 0], sim0.coords[:, 1]
    v = 2000.0 + 300.0 * np.sin(x / 130.0) * np.cos(z / 90.0)
    v_obs = v + 60.0 * np.exp(-((x - 350.0) ** 2 + (z - 250.0) ** 2) / 8e3)
    sim = so.build_sim(cfg, v, dt_cfl_velocity=np.full(len(v), 2600.0))
    y, _ = so.forward(sim, v_obs, convention="fwdadj")
    sigma = 1e-3
    out = so.forward_adjoint(sim, y, sigma)
    g = out["dJ_dv"]                      # d loglik / d c
    rng = np.random.default_rng(1)
    beta = sim.extra["beta"]
    dirs = [rng.standard_normal(len(v)),
            np.where(beta > 0, rng.standard_normal(len(v)), 0.0),   # absorbing-edge nodes only
            np.cos(x / 200.0) * np.sin(z / 150.0)]
    for k, d in enumerate(dirs):
        d = d / np.abs(d).max()
        eps = 0.01   # m/s; the central difference converges as eps^2 down to ~1e-9 here
        lp = so.misfit_loglik(sim, v + eps * d, y, sigma)
        lm = so.misfit_loglik(sim, v - eps * d, y, sigma)
        fd = (lp - lm) / (2 * eps)
        ad = float(g @ d)
        rel = abs(ad - fd) / abs(fd)
        print(f"direction {k}: adjoint {ad:.8e} FD {fd:.8e} rel {rel:.1e}")
        assert rel < 1e-5


def test_stacey_edges_reflect_little():
    h = 50.0
    # edge echoes of the 1000x500 m domain reach the receivers from about 0.5 s on; those
    # of the 3000x1500 m domain only after 1.3 s
    small = _cfg(T=0.7)
    big = _cfg(xmin=-1000.0, xmax=2000.0, zmax=1500.0, nelx=60, nelz=30, T=0.7)
    assert (big["domain"]["xmax"] - big["domain"]["xmin"]) / big["domain"]["nelem_x"] == h
    c0 = 2000.0
    s_small = so.build_sim(small, np.full((20 * 4 + 1) * (10 * 4 + 1), c0))
    s_big = so.build_sim(big, np.full((60 * 4 + 1) * (30 * 4 + 1), c0), dt=s_small.dt)
    assert s_big.dt == s_small.dt and s_big.nt == s_small.nt
    assert np.allclose(s_small.coords[s_small.src_node], s_big.coords[s_big.src_node])
    ref, _ = so.forward(s_big, convention="fwdadj")
    stacey, _ = so.forward(s_small, convention="fwdadj")
    s_small.extra["beta"] = np.zeros_like(s_small.extra["beta"])   # rigid sides and bottom
    rigid, _ = so.forward(s_small, convention="fwdadj")
    e_st = float(np.sum((stacey - ref) ** 2))
    e_rg = float(np.sum((rigid - ref) ** 2))
    print(f"reflected energy at the receivers: Stacey {e_st:.3e}, rigid {e_rg:.3e}, "
          f"ratio {e_st / e_rg:.1e}; direct {float(np.sum(ref ** 2)):.3e}")
    assert e_rg > 1e-3 * float(np.sum(ref ** 2))   # the rigid edges do reflect in the window
    assert e_st < 0.01 * e_rg
