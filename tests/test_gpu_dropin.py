"""The drop-in SEMSimulation on the GPU against the reference's own outputs (same
config dicts, same call sequence as tests/golden/make_golden.py)."""
import numpy as np
import pytest

from mun_b200.sem_waveform import SEMSimulation
from tests.goldens import load, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-4


def test_layered_cfg0_call_sequence():
    g = load("layered_cfg0")
    sim = SEMSimulation(g["config"])
    run = sim.run(ctrl_offsets_flat=np.zeros(12))
    e_run = rel_l2(run["receiver_data"], g["rec_run"])
    nt = int(g["nt"])
    obs = sim.run_forward_and_adjoint({"bspline_ctrl": np.asarray(g["ctrl_true"]).reshape(-1),
                                       "y_obs": np.zeros((nt, 50)), "obs_dt": sim.dt, "obs_nt": nt,
                                       "noise_std": 1e-9, "verbose": False})
    e_obs = rel_l2(obs["clean_data"], g["y_obs"])
    res = sim.run_forward_and_adjoint({"bspline_ctrl": np.asarray(g["ctrl"]).reshape(-1),
                                       "y_obs": g["y_obs"], "obs_dt": sim.dt, "obs_nt": nt,
                                       "noise_std": 1e-9, "verbose": False})
    e_clean = rel_l2(res["clean_data"], g["clean"])
    e_ll = abs(res["loglik"] - float(g["loglik"])) / abs(float(g["loglik"]))
    e_g = rel_l2(res["grad_wrt_ctrl"], g["grad_ctrl"])
    e_dv = rel_l2(-sim.dJ_dv, g["dL_dv"])
    print(f"layered cfg0: run {e_run:.2e} obs {e_obs:.2e} clean {e_clean:.2e} loglik {e_ll:.2e} "
          f"dL/dv {e_dv:.2e} grad_ctrl {e_g:.2e}")
    assert max(e_run, e_obs, e_clean, e_ll, e_dv, e_g) <= TOL
    assert res["dt"] == float(g["dt"]) and res["nt"] == nt


def test_canonical_circle_call_sequence():
    g = load("circle_n5")
    sim = SEMSimulation(g["config"])
    run = sim.run()
    e_run = rel_l2(run["receiver_data"], g["rec_run"])
    ctrl0 = np.asarray(g["ctrl"])
    y = sim.run_forward_and_adjoint({"bspline_ctrl": (ctrl0 + 25.0).reshape(-1),
                                     "y_obs": np.zeros((sim.nt, 24)), "obs_dt": sim.dt,
                                     "obs_nt": sim.nt, "noise_std": 0.0})["clean_data"]
    res = sim.run_forward_and_adjoint({"bspline_ctrl": ctrl0.reshape(-1), "y_obs": g["y_obs"],
                                       "obs_dt": sim.dt, "obs_nt": sim.nt, "noise_std": 1e-8})
    e_y = rel_l2(y, g["y_obs"])
    e_ll = abs(res["loglik"] - float(g["loglik"])) / abs(float(g["loglik"]))
    e_g = rel_l2(res["grad_wrt_ctrl"], g["grad_ctrl"])
    print(f"circle n5: run {e_run:.2e} y {e_y:.2e} loglik {e_ll:.2e} grad_ctrl {e_g:.2e}")
    assert max(e_run, e_y, e_ll, e_g) <= TOL


def test_batch_method_equals_single_calls():
    g = load("layered_cfg0")
    sim = SEMSimulation(g["config"])
    nt = int(g["nt"])
    rng = np.random.default_rng(0)
    params = [{"bspline_ctrl": (np.asarray(g["ctrl"]) + rng.normal(0, 10, (6, 2))).reshape(-1),
               "y_obs": g["y_obs"], "obs_dt": float(g["dt"]), "obs_nt": nt, "noise_std": 1e-9}
              for _ in range(4)]
    batched = sim.run_forward_and_adjoint_batch(params, ckpt_k=64)
    for p, b in zip(params, batched):
        s = sim.run_forward_and_adjoint(p)
        assert s["loglik"] == b["loglik"]
        np.testing.assert_array_equal(s["grad_wrt_ctrl"], b["grad_wrt_ctrl"])


def test_multi_source_batch_equals_separate_calls():
    # one simulation per source position (MUN's multi-source likelihood), batched
    import copy
    from mun_b200.sem_waveform import run_forward_and_adjoint_sources
    g = load("layered_cfg0")
    nt = int(g["nt"])
    sims, params = [], []
    for k, x in enumerate((700.0, 1000.0, 1300.0)):
        cfg = copy.deepcopy(g["config"])
        cfg["source"]["position"] = [x, float(cfg["source"]["position"][1])]
        sims.append(SEMSimulation(cfg))
        params.append({"bspline_ctrl": np.asarray(g["ctrl"]).reshape(-1), "y_obs": g["y_obs"],
                       "obs_dt": float(g["dt"]), "obs_nt": nt, "noise_std": 1e-9})
    batched = run_forward_and_adjoint_sources(sims, params)
    for sim, p, b in zip(sims, params, batched):
        s = sim.run_forward_and_adjoint(p)
        assert s["loglik"] == b["loglik"]
        np.testing.assert_array_equal(s["grad_wrt_ctrl"], b["grad_wrt_ctrl"])
        np.testing.assert_array_equal(s["clean_data"], b["clean_data"])
        assert s["dt"] == b["dt"] and s["nt"] == b["nt"]


def test_concurrent_threads_on_separate_simulations():
    """MUN's multi-source likelihood runs one simulation per source on up to three Python
    threads (CO2_plume/one_stage/single_cubic/RQS_NF.py:1064-1072).  The same pattern here,
    with fresh simulations so the threads also race on the shared plan cache, gives bitwise
    the serial results."""
    import copy
    from concurrent.futures import ThreadPoolExecutor
    from mun_b200.sem_waveform import core
    g = load("layered_cfg0")
    nt = int(g["nt"])
    xs = (500.0, 800.0, 1000.0, 1200.0, 1500.0)

    def cfg_for(x):
        cfg = copy.deepcopy(g["config"])
        cfg["source"]["position"] = [x, float(cfg["source"]["position"][1])]
        return cfg

    def params(k):
        return {"bspline_ctrl": (np.asarray(g["ctrl"]) + 5.0 * k).reshape(-1), "y_obs": g["y_obs"],
                "obs_dt": float(g["dt"]), "obs_nt": nt, "noise_std": 1e-9}

    serial = [SEMSimulation(cfg_for(x)).run_forward_and_adjoint(params(k)) for k, x in enumerate(xs)]
    with core._PLAN_LOCK:
        core._PLAN_CACHE.clear()

    def one(task):
        k, x = task
        return SEMSimulation(cfg_for(x)).run_forward_and_adjoint(params(k))

    for _ in range(2):
        with ThreadPoolExecutor(max_workers=3) as ex:
            threaded = list(ex.map(one, enumerate(xs)))
        for s, t in zip(serial, threaded):
            assert s["loglik"] == t["loglik"]
            np.testing.assert_array_equal(s["grad_wrt_ctrl"], t["grad_wrt_ctrl"])
            np.testing.assert_array_equal(s["clean_data"], t["clean_data"])
