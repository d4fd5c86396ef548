"""Benchmark: SEM forward+adjoint solves/s, batched vs plain, on one B200 per rank.

Workload (default): batched ELBO sampling — 256 velocity models on one 100x50-element,
order-4 mesh over 2000x1000 m (80,601 nodes), each the three-layer 1500/2200/3000 m/s
base (interfaces at 300/650 m) plus a cubic tensor B-spline perturbation on a 10x6
node grid with N(0, 100^2) m/s node values drawn from a seed; Ricker 10 Hz at
(1000, 20), 100 receivers at 10 m depth, 3000 steps at the CFL limit, sponge 200 m on
all sides, float32 wavefields, float64 gradient time-sum (float32 partial sums of at
most 16 ticks folded into float64) and float64 misfit.  Observed data come from a
seeded "true" perturbation.  Inputs are synthetic (no dataset involved).

A step = one batched forward+adjoint pass over all 256 models.  ``value`` is
device-timed with CUDA events (inputs resident), ``e2e`` is the same step through the
public API with host arrays copied in and gradients/logliks copied out inside the
timed region.  ``plain`` times one-at-a-time solves of the same models.  Outside the
timed region, two of the models are solved again by the float64 oracle on the host
(``parity``), and compact runs of the single large solve, the uneven batch and the
serving mix are added as ``single``, ``uneven`` and ``serving``.

``--impl reference`` times the oracle restatement of MUN's CPU path (torch-CPU float64,
same library calls as the reference) on the host cores: one full 3000-step solve of
one model per step (``--ref-nt N`` fits set-up + per-step cost from N- and 2N-step runs
instead).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

# the metric both arms report (the driver pairs the two lines by it)
METRIC = "SEM fwd+adjoint solves/s (batched vs plain, same GPU, <=1e-4 rel); p50/p99 ms"
# algorithmic bytes per node and fwd+adj step (float32 state): forward 16 (u_curr, u_prev
# and c^2 read, u_next written), forward-state store/load 8, adjoint 16, float64 gradient
# read-modify-write 16; a forward tick carries 20 of them, an adjoint tick 36
BYTES_PER_NODE_STEP_FWDADJ = 56
BYTES_PER_NODE_FWD_TICK = 20
BYTES_PER_NODE_ADJ_TICK = 36
# bytes the strip kernel itself moves per node: forward tick 20 (reads b, v, c^2, writes
# b, v); adjoint tick 32.5 (reads lambda, mu, c^2 and the forward b, writes lambda and mu,
# float32 partial gradient read-modify-write, and a float64 fold every 16 ticks)
IMPL_BYTES_PER_NODE = {"forward_tick": 20, "adjoint_tick": 32.5}
# DRAM bytes per node and tick of the strip kernel from one ncu capture (dram__bytes_read +
# dram__bytes_write of one forward and one adjoint tick of a 128-model group, 10.3 M nodes),
# scaled to a launch by its nodes
TRAFFIC_B_PER_NODE = {"fwd": 17.0, "adj": 29.3}


WORKLOAD_ELBO = ("batched ELBO sampling (256 models, 100x50 el, N=4, 80601 nodes, 3000 steps, "
                 "100 receivers)")


def workload(nmodels=256, nelx=100, nelz=50, nt=3000, nrec=100, seed0=0, boundary="sponge"):
    from mun_b200.bspline import grid_basis, layered_velocity
    from mun_b200.mesh import create_global_mesh
    xmin, xmax, zmin, zmax, N = 0.0, 2000.0, 0.0, 1000.0, 4
    coords, _, node_grid = create_global_mesh(xmin, xmax, zmin, zmax, nelx, nelz, N)
    base = layered_velocity(coords[:, 1], [300.0, 650.0], [1500.0, 2200.0, 3000.0])
    B = grid_basis(coords, (xmin, xmax), (zmin, zmax), 10, 6)
    thetas = np.stack([np.random.default_rng(seed0 + i).normal(0.0, 100.0, 60) for i in range(nmodels)])
    vels = base[None, :] + thetas @ B.T
    theta_true = np.random.default_rng(12345).normal(0.0, 100.0, 60)
    v_true = base + B @ theta_true
    cmax = max(float(vels.max()), float(v_true.max()))
    dt = 0.35 * (min((xmax - xmin) / nelx, (zmax - zmin) / nelz) / (N + 1)) / (cmax * (N + 1) * np.sqrt(2.0))
    rec = np.stack([np.linspace(xmin, xmax, nrec), np.full(nrec, 10.0)], 1)
    plan_kw = dict(xmin=xmin, xmax=xmax, zmin=zmin, zmax=zmax, nelx=nelx, nelz=nelz, npol=N, dt=dt,
                   nt=nt, src_xz=(1000.0, 20.0), f0=10.0, amp=1.0, receivers=rec,
                   pml_thickness=200.0, sponge_cmax=3000.0, coords=coords, node_grid=node_grid,
                   boundary=boundary)
    return dict(plan_kw=plan_kw, vels=vels, v_true=v_true, thetas=thetas, B=B, coords=coords,
                npoints=len(coords), dt=dt, nt=nt, sigma=1e-3)


def max_over_ranks(x, world, device=None):
    """Largest value of x over the ranks of the job (the job's time is its slowest rank's);
    every rank must call it at the same point."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def parse_tile(t):
    """'8x4' -> (8, 4); 'auto' -> (0, 0) (the library picks the shape)."""
    return (0, 0) if t == "auto" else tuple(int(x) for x in t.split("x"))


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    def __init__(self, path):
        self.path = path
        self.p = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self, device_index=0):
        try:
            rows = [l.split(",") for l in open(self.path).read().strip().splitlines()]
            rows = [[x.strip() for x in r] for r in rows if len(r) >= 9 and r[0].strip() == str(device_index)]
            sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
            mx = float(rows[0][2]) if rows else None
            reasons = set()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for r in rows:
                for nm, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
            return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                    "reasons": sorted(reasons), "samples": len(sm)}
        except Exception as exc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "error": str(exc)}


def peaks():
    try:
        return json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def cpu_baseline(W, nt_sample, threads):
    """Oracle restatement of the reference's CPU path on one model.  nt_sample <= 0 (or
    >= nt): one full-length solve, timed as is.  Otherwise runs nt_sample and
    2*nt_sample steps and fits set-up + per-step cost, so the full-length solve time is
    set-up + nt * per-step (the reference's loops are linear in nt)."""
    if nt_sample <= 0 or nt_sample >= W["nt"]:
        t = oracle_solve_s(W, W["nt"], threads)
        return t, t
    t1 = oracle_solve_s(W, nt_sample, threads)
    t2 = oracle_solve_s(W, 2 * nt_sample, threads)
    per_step = max((t2 - t1) / nt_sample, 1e-9)
    setup = max(t1 - per_step * nt_sample, 0.0)
    return setup + per_step * W["nt"], t1 + t2


def oracle_solve_s(W, nts, threads):
    """Wall time of one oracle fwd+adj solve of nts steps (set-up included)."""
    import torch
    from oracle import sem_oracle as so
    torch.set_num_threads(threads)
    kw = W["plan_kw"]
    cfg = {"domain": {"xmin": kw["xmin"], "xmax": kw["xmax"], "zmin": kw["zmin"],
                      "zmax": kw["zmax"], "nelem_x": kw["nelx"], "nelem_z": kw["nelz"]},
           "time": {"total_time": (nts - 0.5) * W["dt"], "dt": W["dt"]},
           "source": {"position": kw["src_xz"], "frequency": kw["f0"], "amplitude": kw["amp"]},
           "receivers": {"positions": kw["receivers"]},
           "method": {"polynomial_order": kw["npol"], "pml_thickness": kw["pml_thickness"],
                      "boundary": kw.get("boundary", "sponge")},
           "velocity": {"outside_velocity": kw["sponge_cmax"]}}
    t0 = time.perf_counter()
    sim = so.build_sim(cfg, W["vels"][0], dt=W["dt"])
    y = np.zeros((sim.nt, len(kw["receivers"])))
    so.forward_adjoint(sim, y, W["sigma"])
    return time.perf_counter() - t0


def cpu_estimate(plan_kw, dt, nt, velocity, nt_sample, threads, sigma=1e-3):
    """Oracle CPU time of one full fwd+adj solve, fitted from nt_sample and 2*nt_sample
    step runs (set-up + per-step cost); exact when nt_sample >= nt."""
    W = {"plan_kw": plan_kw, "dt": dt, "nt": nt, "vels": [velocity], "sigma": sigma}
    if nt_sample >= nt:
        el = oracle_solve_s(W, nt, threads)
        return el, el
    return cpu_baseline(W, nt_sample, threads)


def run_plain(args):
    """Plain method (CPU-runnable case): 2000x1000 m, 40x20 elements, order 4 (161x81
    nodes), three-layer 1500/2200/3000 m/s (interfaces 300/650 m), Ricker 10 Hz at
    (1000, 20), 50 receivers at 10 m depth, dt at the CFL limit, 2000 steps, forward +
    adjoint; observations from the model with +100 m/s on the central B-spline nodes.
    One GPU solve at a time (events) and the oracle's full CPU run on the host cores."""
    import torch
    from mun_b200 import Batch, SEMPlan, SolveSpec
    from mun_b200.bspline import grid_basis, layered_velocity
    from mun_b200.mesh import create_global_mesh
    xmin, xmax, zmin, zmax, nelx, nelz, N = 0.0, 2000.0, 0.0, 1000.0, 40, 20, 4
    coords, _, ng = create_global_mesh(xmin, xmax, zmin, zmax, nelx, nelz, N)
    v = layered_velocity(coords[:, 1], [300.0, 650.0], [1500.0, 2200.0, 3000.0])
    B = grid_basis(coords, (xmin, xmax), (zmin, zmax), 8, 4)
    th = np.zeros(32)
    th[[10, 11, 13, 14, 18, 19, 21, 22]] = 100.0
    v_obs = v + B @ th
    # "CFL 0.4" asks for the reference's stability limit, which it clamps to:
    # 0.35 (h / (N+1)) / (c_max (N+1) sqrt 2) = 1.650e-4 s at c_max 3000, h 50 m
    h = min((xmax - xmin) / nelx, (zmax - zmin) / nelz)
    dt = 0.35 * (h / (N + 1)) / (3000.0 * (N + 1) * np.sqrt(2.0))
    nt = 2000
    rec = np.stack([np.linspace(xmin, xmax, 50), np.full(50, 10.0)], 1)
    kw = dict(xmin=xmin, xmax=xmax, zmin=zmin, zmax=zmax, nelx=nelx, nelz=nelz, npol=N, dt=dt, nt=nt,
              src_xz=(1000.0, 20.0), f0=10.0, amp=1.0, receivers=rec, pml_thickness=200.0,
              sponge_cmax=3000.0, coords=coords, node_grid=ng, boundary=args.boundary)
    plan = SEMPlan(**kw)
    dev = torch.device("cuda")
    obs = SolveSpec(plan, torch.as_tensor(v_obs, device=dev), shift=True)
    Batch().run([obs])
    y = obs.rec.double()
    tex, tez = parse_tile(args.tile)
    b = Batch(tile=(tex, tez), graph_chunk=args.graph_chunk, kernel=args.kernel)
    stream = torch.cuda.Stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for it in range(args.warmup + max(args.steps, 5)):
        s = SolveSpec(plan, torch.as_tensor(v, device=dev), adjoint=True, y_obs=y, inv_sigma2=1e6)
        with torch.cuda.stream(stream):
            ev0.record(stream)
            b.run([s])
            ev1.record(stream)
        ev1.synchronize()
        if it >= args.warmup:
            ms.append(ev0.elapsed_time(ev1))
    ms = np.array(ms)
    out = {"workload": "plain: 40x20 el, N=4, 13041 nodes, 2000 steps, 50 receivers, fwd+adj",
           "boundary": args.boundary,
           "gpu_ms_per_solve": float(ms.mean()), "gpu_solves_per_s": 1e3 / float(ms.mean()),
           "p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)),
           "kernel": b.last_kernel, "shape": b.last_shape, "graph_chunk": args.graph_chunk,
           "groups": b.last_groups, "status": int(s.status.item())}
    if not args.no_cpu:
        threads = os.cpu_count() or 1
        kw_o = {k: kw[k] for k in kw if k not in ("coords", "node_grid")}
        t0 = time.perf_counter()
        per, _ = cpu_estimate(kw_o, dt, nt, v, nt, threads)
        out["cpu"] = {"s_per_solve": per, "solves_per_s": 1.0 / per, "cores": threads, "kind": "port",
                      "sample": "one full 2000-step run, set-up included",
                      "wall_s": time.perf_counter() - t0}
        out["gpu_over_cpu"] = per / (ms.mean() / 1e3)
    print(json.dumps(out), flush=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    W = workload(nmodels=1)
    nt_sample = args.ref_nt
    for _ in range(args.warmup):
        cpu_baseline(W, nt_sample, threads)
    times = []
    for _ in range(args.steps):
        per, _ = cpu_baseline(W, nt_sample, threads)
        times.append(per)
    per = float(np.mean(times))
    val = 1.0 / per
    sample_txt = ("1 model, one full 3000-step fwd+adj solve per step (set-up included)"
                  if nt_sample <= 0 or nt_sample >= W["nt"] else
                  f"1 model, {nt_sample}- and {2 * nt_sample}-step runs (of 3000) fitted to set-up + "
                  "per-step cost")
    out = {"metric": METRIC, "value": val, "unit": "solves/s",
           "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": per * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic",
           "config": {"workload": WORKLOAD_ELBO, "sample": sample_txt},
           "cpu_baseline": {"value": val, "unit": "solves/s", "cores": threads, "kind": "port",
                            "sample": sample_txt},
           "e2e": {"value": val, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def _layered_plume(coords, cx, cz, ax, az, drop=0.08):
    from mun_b200.bspline import layered_velocity
    base = layered_velocity(coords[:, 1], [300.0, 650.0], [1500.0, 2200.0, 3000.0])
    r2 = ((coords[:, 0] - cx) / ax) ** 2 + ((coords[:, 1] - cz) / az) ** 2
    w = 1.0 / (1.0 + np.exp((r2 - 1.0) * 8.0))   # smooth ellipse indicator
    return base * (1.0 - drop * w)


def uneven_specs(n=64, seed=3):
    """Uneven batch: n solves, meshes 40x20..200x100 (2:1), orders {3,4,5}, 8-20 Hz, nt from
    each mesh's CFL for T = 0.5 s clamped to [1500, 6000], layered base with a seeded
    elliptical -8% plume; observations from each model's own forward at 2% lower velocity."""
    from mun_b200.mesh import create_global_mesh
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nelx = int(rng.integers(40, 201))
        nelz = max(1, nelx // 2)
        N = int(rng.choice([3, 4, 5]))
        f0 = float(rng.uniform(8.0, 20.0))
        coords, _, ng = create_global_mesh(0.0, 2000.0, 0.0, 1000.0, nelx, nelz, N)
        v = _layered_plume(coords, rng.uniform(600, 1400), rng.uniform(400, 700), rng.uniform(150, 400),
                           rng.uniform(150, 400))
        h = min(2000.0 / nelx, 1000.0 / nelz)
        dt = 0.35 * (h / (N + 1)) / (float(v.max()) * (N + 1) * np.sqrt(2.0))
        nt = int(min(6000, max(1500, np.ceil(0.5 / dt))))
        rec = np.stack([np.linspace(0.0, 2000.0, 100), np.full(100, 10.0)], 1)
        out.append(dict(plan=dict(xmin=0.0, xmax=2000.0, zmin=0.0, zmax=1000.0, nelx=nelx, nelz=nelz,
                                  npol=N, dt=dt, nt=nt, src_xz=(1000.0, 20.0), f0=f0, amp=1.0,
                                  receivers=rec, pml_thickness=200.0, sponge_cmax=3000.0,
                                  coords=coords, node_grid=ng), v=v))
    return out


def run_uneven(args, steps=None, warmup=None, plain=None, cpu_sample=None, emit=True):
    """Uneven batch (64 solves of uneven meshes, orders and step counts), batched through
    the autotuned launch configuration vs one solve at a time."""
    import torch
    from mun_b200 import Batch, SEMPlan, SolveSpec
    from mun_b200.autotune import tuned_batch
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    plain = args.plain if plain is None else plain
    cpu_sample = args.cpu_sample if cpu_sample is None else cpu_sample
    specs_args = uneven_specs(args.models if (emit and args.models != 256) else 64)
    plans = [SEMPlan(**a["plan"]) for a in specs_args]
    dev = torch.device("cuda")
    stream = torch.cuda.Stream()
    ys = []
    ob = Batch()
    with torch.cuda.stream(stream):
        for p, a in zip(plans, specs_args):
            s = SolveSpec(p, torch.as_tensor(a["v"] * 0.98, device=dev), shift=True)
            ob.run([s])
            ys.append(s.rec.double())
    stream.synchronize()
    node_steps = sum(p.npoints * p.nt for p in plans)

    def specs():
        return [SolveSpec(p, torch.as_tensor(a["v"], device=dev), adjoint=True, y_obs=y, inv_sigma2=1e6,
                          ckpt_k=0) for p, a, y in zip(plans, specs_args, ys)]
    t0 = time.perf_counter()
    if args.kernel == 0 and args.graph_chunk == 0:
        b, tuned = tuned_batch(specs())
    else:
        b, tuned = Batch(kernel=args.kernel, graph_chunk=args.graph_chunk), None
    tune_s = time.perf_counter() - t0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for it in range(warmup + steps):
        sp = specs()
        with torch.cuda.stream(stream):
            ev0.record(stream)
            b.run(sp)
            ev1.record(stream)
        ev1.synchronize()
        if it >= warmup:
            ms.append(ev0.elapsed_time(ev1))
    status = max(int(s.status.item()) for s in sp)
    batched = len(plans) / (np.mean(ms) / 1e3)
    plain_ms = []
    pb = Batch()
    for sp1 in specs()[: max(4, plain)]:
        with torch.cuda.stream(stream):
            ev0.record(stream)
            pb.run([sp1])
            ev1.record(stream)
        ev1.synchronize()
        plain_ms.append(ev0.elapsed_time(ev1))
    # plain time of the whole set, scaled by node-steps of the timed subset
    sub = plans[: len(plain_ms)]
    plain_total = sum(plain_ms) * node_steps / sum(p.npoints * p.nt for p in sub)
    cpu = None
    if cpu_sample > 0:
        threads = os.cpu_count() or 1
        per_ns, el = [], 0.0
        for p, a in list(zip(plans, specs_args))[:2]:
            kw_o = {k: a["plan"][k] for k in a["plan"] if k not in ("coords", "node_grid", "dt", "nt")}
            per, e = cpu_estimate(kw_o, a["plan"]["dt"], p.nt, a["v"], cpu_sample, threads)
            per_ns.append(per / (p.npoints * p.nt))
            el += e
        total = float(np.mean(per_ns)) * node_steps
        cpu = {"solves_per_s": len(plans) / total, "s_all": total, "cores": threads, "kind": "port",
               "sample": f"first 2 solves, {cpu_sample}/{2 * cpu_sample}-step runs, per node-step "
                         f"cost scaled to all 64 ({el:.0f} s)"}
    out = {"workload": "uneven batch: 64 solves, 40x20..200x100 el, N in {3,4,5}, nt 1500-6000",
           "metric": "SEM fwd+adjoint solves/s", "unit": "solves/s", "batched": batched,
           "batched_ms": float(np.mean(ms)), "kernel": b.last_kernel, "groups": b.last_groups,
           "autotuned": None if tuned is None else {"kernel": tuned["kernel"], "tile": list(tuned["tile"]),
                                                    "graph_chunk": tuned["graph_chunk"],
                                                    "strip_bands": tuned["strip_bands"],
                                                    "ckpt_k": "automatic schedule (memory-budget cost model)",
                                                    "tuning_s": round(tune_s, 1)},
           "shape (tile_ex, tile_ez, strip_bands)": list(b.last_shape),
           "plain_estimated": len(plans) / (plain_total / 1e3), "plain_solves_timed": len(plain_ms),
           "batched_over_plain": batched / (len(plans) / (plain_total / 1e3)),
           "mnode_steps_per_s": node_steps / (np.mean(ms) / 1e3) / 1e6,
           "orders": sorted(set(p.npol for p in plans)),
           "nt_range": [min(p.nt for p in plans), max(p.nt for p in plans)], "cpu": cpu, "status": status}
    if emit:
        print(json.dumps(out), flush=True)
    return out


def run_serving(args, requests=None, emit=True):
    """Serving: Poisson request stream of forward-only likelihoods from 16 random-walk MCMC
    chains (meshes 60x30..120x60, order 4) mixed with flow-trainer batches of 32
    forward+adjoint solves (100x50, order 4, 10x6 B-spline perturbations); continuous
    batching in the engine; p50/p99 latency and solves/s vs the same requests served one
    at a time."""
    import torch
    from mun_b200 import Batch, SEMPlan, SolveSpec
    from mun_b200.mesh import create_global_mesh
    from mun_b200.serving import Engine, Request, serve
    rng = np.random.default_rng(4)
    dev = torch.device("cuda")
    T = args.serve_T
    chains = []
    for c in range(16):
        nelx = int(rng.integers(60, 121))
        nelz = nelx // 2
        coords, _, ng = create_global_mesh(0.0, 2000.0, 0.0, 1000.0, nelx, nelz, 4)
        v0 = _layered_plume(coords, rng.uniform(800, 1200), 550.0, 250.0, 150.0)
        h = 2000.0 / nelx
        dt = 0.35 * (h / 5) / (3300.0 * 5 * np.sqrt(2.0))
        nt = int(np.ceil(T / dt))
        rec = np.stack([np.linspace(0.0, 2000.0, 50), np.full(50, 10.0)], 1)
        p = SEMPlan(xmin=0.0, xmax=2000.0, zmin=0.0, zmax=1000.0, nelx=nelx, nelz=nelz, npol=4, dt=dt, nt=nt,
                    src_xz=(1000.0, 20.0), f0=10.0, amp=1.0, receivers=rec, pml_thickness=200.0,
                    sponge_cmax=3000.0, coords=coords, node_grid=ng)
        s = SolveSpec(p, torch.as_tensor(v0, device=dev))
        Batch().run([s])
        chains.append((p, v0, s.rec.double(), coords))
    W = workload(nmodels=32, nt=int(np.ceil(T / workload(nmodels=1, nt=10)["dt"])))
    fplan = SEMPlan(**W["plan_kw"])
    obs = SolveSpec(fplan, torch.as_tensor(W["v_true"], device=dev), shift=True)
    Batch().run([obs])
    fy = obs.rec.double()
    reqs = []
    t = 0.0
    rate = args.serve_rate
    n_req = args.serve_requests if requests is None else requests
    k_flow = 0
    while len(reqs) < n_req:
        t += rng.exponential(1.0 / rate)
        if rng.uniform() < 0.8:   # MCMC proposal
            c = int(rng.integers(16))
            p, v0, y, coords = chains[c]
            v = v0 + rng.normal(0, 20.0) * np.exp(-((coords[:, 0] - 1000) ** 2 + (coords[:, 1] - 550) ** 2) / 2e5)
            reqs.append(Request(t, SolveSpec(p, torch.as_tensor(v, device=dev), misfit=True, y_obs=y,
                                             inv_sigma2=1e6), "mcmc"))
        else:                      # flow-trainer batch of 32 samples
            for i in range(32):
                reqs.append(Request(t, SolveSpec(fplan, torch.as_tensor(W["vels"][(32 * k_flow + i) % 32], device=dev),
                                                 adjoint=True, y_obs=fy, inv_sigma2=1e6, ckpt_k=fplan.nt),
                                    "flow"))
            k_flow += 1
    free, _ = torch.cuda.mem_get_info()
    cap = min(int(args.serve_cap_gb * (1 << 30)), int(free) - (8 << 30))
    eng = Engine(max_solves=args.serve_slots, memory_cap_bytes=cap,
                 ticks_per_step=args.serve_ticks, kernel=args.kernel)
    done, lat, wall = serve(eng, reqs)
    # serialized reference: the same requests one at a time, back to back
    b = Batch()
    t0 = time.perf_counter()
    for r in reqs:
        s = r.spec
        s2 = SolveSpec(s.plan, s.velocity, adjoint=s.adjoint, misfit=s.misfit, shift=s.shift,
                       y_obs=s.y_obs, inv_sigma2=s.inv_sigma2, ckpt_k=s.ckpt_k)
        b.run([s2])
    torch.cuda.synchronize()
    serial = time.perf_counter() - t0
    kinds = np.array([r.kind for r in done])
    out = {"workload": f"serving: Poisson {rate:.0f} req/s, 16 MCMC chains (fwd likelihood, 60x30..120x60) "
                       f"+ flow batches of 32 fwd+adj (100x50), T={T} s",
           "requests": len(done), "wall_s": wall, "solves_per_s": len(done) / wall,
           "p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99)),
           "p50_ms_mcmc": 1e3 * float(np.percentile(lat[kinds == "mcmc"], 50)),
           "p99_ms_mcmc": 1e3 * float(np.percentile(lat[kinds == "mcmc"], 99)),
           "p50_ms_flow": 1e3 * float(np.percentile(lat[kinds == "flow"], 50)) if (kinds == "flow").any() else None,
           "serialized_solves_per_s": len(reqs) / serial, "served_over_serialized": (len(done) / wall) / (len(reqs) / serial),
           "memory_cap_gb": cap / (1 << 30), "engine": eng.stats()}
    if emit:
        print(json.dumps(out), flush=True)
    return out


def single_model(nelx=400, nelz=200, N=4):
    """Single large solve inputs: 8000x4000 m, order 4 (1601x801 nodes at 400x200), GRF
    velocity (mean 2500, std 300, correlation 200 m, clipped [1500, 4000], seed 1), dt at
    the CFL limit."""
    from mun_b200.mesh import create_global_mesh
    from mun_b200.sem_waveform.velocity import build_background_from_grid
    coords, _, ng = create_global_mesh(0.0, 8000.0, 0.0, 4000.0, nelx, nelz, N)
    rng = np.random.default_rng(1)
    nx, nz = 801, 401
    w = rng.standard_normal((nz, nx))
    kx = np.fft.fftfreq(nx, d=10.0)
    kz = np.fft.fftfreq(nz, d=10.0)
    K2 = kx[None, :] ** 2 + kz[:, None] ** 2
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * np.exp(-2 * (np.pi ** 2) * (200.0 ** 2) * K2)))
    f = (f - f.mean()) / f.std() * 300.0 + 2500.0
    grid = np.clip(f, 1500.0, 4000.0)
    v = build_background_from_grid(coords, np.linspace(0, 8000, nx), np.linspace(0, 4000, nz), grid)
    h = min(8000.0 / nelx, 4000.0 / nelz)
    dt = 0.35 * (h / (N + 1)) / (float(v.max()) * (N + 1) * np.sqrt(2.0))
    return coords, ng, v, dt


def run_single(args, steps=None, warmup=None, cpu_sample=None, emit=True):
    """Single large solve: 400x200 elements, order 4, GRF velocity, Ricker 15 Hz at the
    surface centre, 400 surface receivers, 5000 steps, checkpoint every 250."""
    import torch
    from mun_b200 import Batch, SEMPlan, SolveSpec
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    cpu_sample = args.cpu_sample if cpu_sample is None else cpu_sample
    nelx, nelz, N = 400, 200, 4
    coords, ng, v, dt = single_model(nelx, nelz, N)
    nt = args.nt if (emit and args.nt != 3000) else 5000
    rec = np.stack([np.linspace(0.0, 8000.0, 400), np.full(400, 1e-3)], 1)
    plan = SEMPlan(xmin=0.0, xmax=8000.0, zmin=0.0, zmax=4000.0, nelx=nelx, nelz=nelz, npol=N, dt=dt, nt=nt,
                   src_xz=(4000.0, 1e-3), f0=15.0, amp=1.0, receivers=rec, pml_thickness=400.0,
                   sponge_cmax=4000.0, coords=coords, node_grid=ng)
    dev = torch.device("cuda")
    obs = SolveSpec(plan, torch.as_tensor(v * 1.01, device=dev), shift=True)
    Batch().run([obs])
    stream = torch.cuda.Stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b = Batch(kernel=args.kernel)

    def timed(k):
        ms = []
        for it in range(warmup + steps):
            s = SolveSpec(plan, torch.as_tensor(v, device=dev), adjoint=True, y_obs=obs.rec.double(),
                          inv_sigma2=1e6, ckpt_k=k)
            with torch.cuda.stream(stream):
                ev0.record(stream)
                b.run([s])
                ev1.record(stream)
            ev1.synchronize()
            if it >= warmup:
                ms.append(ev0.elapsed_time(ev1))
        return float(np.mean(ms)), s, b.last_ticks, b.last_tick_ms()
    m, s, ticks_k250, tick_ms = timed(250)
    # the same solve under the automatic schedule: its float32 forward history (25.6 GB)
    # fits, so there is no replay
    m_auto, s2, ticks_auto, tick_ms_auto = timed(0)
    same = bool(torch.equal(s.grad, s2.grad) and torch.equal(s.rec, s2.rec))
    # the same automatic schedule in one cooperative launch (persistent strip kernel)
    b_auto = b
    b = Batch(kernel=4)
    m_pers, s3, _, _ = timed(0)
    pers = {"ms_per_solve": m_pers, "solves_per_s": 1e3 / m_pers, "kernel": b.last_kernel,
            "bitwise_equal": bool(torch.equal(s3.grad, s2.grad) and torch.equal(s3.rec, s2.rec)),
            "hbm_frac_56B": BYTES_PER_NODE_STEP_FWDADJ * plan.npoints * nt / (m_pers / 1e3) / 1e9
            / float(peaks()[0].get("hbm_gbs", 6650.0))}
    b = b_auto
    alg = BYTES_PER_NODE_STEP_FWDADJ * plan.npoints * nt
    pk, pk_kind = peaks()
    peak = float(pk.get("hbm_gbs", 6650.0))
    auto = {"ms_per_solve": m_auto, "solves_per_s": 1e3 / m_auto, "ticks": ticks_auto,
            "groups": b.last_groups, "bitwise_equal_to_k250": same,
            "achieved_gbs_56B": alg / (m_auto / 1e3) / 1e9,
            "hbm_frac_56B": alg / (m_auto / 1e3) / 1e9 / peak,
            "tick_loop_ms": tick_ms_auto}
    cpu = None
    if cpu_sample > 0:
        kw_o = dict(xmin=0.0, xmax=8000.0, zmin=0.0, zmax=4000.0, nelx=nelx, nelz=nelz, npol=N,
                    src_xz=(4000.0, 1e-3), f0=15.0, amp=1.0, receivers=rec, pml_thickness=400.0,
                    sponge_cmax=4000.0)
        threads = os.cpu_count() or 1
        per, el = cpu_estimate(kw_o, dt, nt, v, cpu_sample, threads)
        cpu = {"s_per_solve": per, "solves_per_s": 1.0 / per, "cores": threads, "kind": "port",
               "sample": f"{cpu_sample}- and {2 * cpu_sample}-step runs of {nt}, linear fit "
                         f"(float64 state, no checkpointing: {el:.0f} s)"}
    out = {"workload": "single large solve: 400x200 el, N=4, 1,282,401 nodes, 5000 steps, k=250",
           "nt": nt, "ms_per_solve": m, "solves_per_s": 1e3 / m, "kernel": b.last_kernel,
           "shape (tile_ex, tile_ez, strip_bands)": list(b.last_shape),
           "mnode_steps_per_s": plan.npoints * nt / (m / 1e3) / 1e6,
           "achieved_gbs_56B": alg / (m / 1e3) / 1e9, "hbm_frac_56B": alg / (m / 1e3) / 1e9 / peak,
           "peak_kind": pk_kind, "ticks": ticks_k250, "tick_loop_ms": tick_ms,
           "auto_schedule": auto, "persistent_strip": pers, "cpu": cpu,
           "status": int(s.status.item()) | int(s2.status.item()) | int(s3.status.item())}
    if emit:
        print(json.dumps(out), flush=True)
    return out


def stacey_leg(args, steps=2, warmup=1):
    """The batched ELBO step with the boundary the configuration states: Stacey absorbing
    sides and bottom, free surface on top (an extension mode; the reference has only the
    sponge).  Device-timed steps of the 256 models and float64-oracle parity of one."""
    import torch
    from mun_b200 import Batch, SEMPlan, SolveSpec
    W = workload(nmodels=args.models, nt=args.nt, boundary="stacey")
    plan = SEMPlan(**W["plan_kw"])
    dev = torch.device("cuda")
    stream = torch.cuda.Stream()
    batch = Batch(kernel=args.kernel)
    with torch.cuda.stream(stream):
        obs = SolveSpec(plan, torch.as_tensor(W["v_true"], device=dev), shift=True)
        batch.run([obs])
    stream.synchronize()
    y = obs.rec.double()
    inv_s2 = 1.0 / (W["sigma"] ** 2 + 1e-24)
    vel = torch.as_tensor(W["vels"], device=dev)
    specs = [SolveSpec(plan, vel[i], adjoint=True, y_obs=y, inv_sigma2=inv_s2) for i in range(args.models)]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for it in range(warmup + steps):
        with torch.cuda.stream(stream):
            ev0.record(stream)
            batch.run(specs)
            ev1.record(stream)
        ev1.synchronize()
        if it >= warmup:
            ms.append(ev0.elapsed_time(ev1))
    out = {"workload": "batched ELBO sampling, 256 models, Stacey absorbing sides and bottom, free surface "
                       "on top (no sponge)",
           "value": args.models / (np.mean(ms) / 1e3), "unit": "solves/s", "ms_per_step": float(np.mean(ms)),
           "kernel": batch.last_kernel, "groups": batch.last_groups, "ticks": batch.last_ticks,
           "tick_loop_ms": batch.last_tick_ms(),
           "status": int(torch.cat([s.status for s in specs]).max().item())}
    out["parity"] = parity_leg(W, specs, y, [1])
    return out


def parity_leg(W, specs, y, which):
    """Relative errors of solves ``which`` of the timed batch (their last run) against the
    float64 oracle on the host, same velocity and observations: seismogram (rel. L2),
    gradient dJ/dv (rel. L2), log-likelihood (rel.).  Outside the timed region."""
    import torch
    from oracle import sem_oracle as so
    torch.set_num_threads(os.cpu_count() or 1)
    kw = W["plan_kw"]
    cfg = {"domain": {"xmin": kw["xmin"], "xmax": kw["xmax"], "zmin": kw["zmin"],
                      "zmax": kw["zmax"], "nelem_x": kw["nelx"], "nelem_z": kw["nelz"]},
           "time": {"total_time": (W["nt"] - 0.5) * W["dt"], "dt": W["dt"]},
           "source": {"position": kw["src_xz"], "frequency": kw["f0"], "amplitude": kw["amp"]},
           "receivers": {"positions": kw["receivers"]},
           "method": {"polynomial_order": kw["npol"], "pml_thickness": kw["pml_thickness"],
                      "boundary": kw.get("boundary", "sponge")},
           "velocity": {"outside_velocity": kw["sponge_cmax"]}}
    yy = y.cpu().numpy()
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
    t0 = time.perf_counter()
    rows = []
    for i in which:
        sim = so.build_sim(cfg, W["vels"][i], dt=W["dt"])
        assert sim.nt == W["nt"]
        ref = so.forward_adjoint(sim, yy, W["sigma"])
        s = specs[i]
        rows.append((rel(s.rec.cpu().numpy(), ref["clean"]), rel(s.grad.cpu().numpy(), ref["dJ_dv"]),
                     abs(float(s.loglik.item()) - ref["loglik"]) / abs(ref["loglik"])))
    e = np.array(rows).max(axis=0)
    return {"models": list(which), "seis_rel_l2": float(e[0]), "grad_rel_l2": float(e[1]),
            "loglik_rel": float(e[2]), "tolerance": 1e-4, "pass": bool((e <= 1e-4).all()),
            "oracle": "float64 CPU restatement of the reference path, full 3000 steps"
                      + ("" if kw.get("boundary", "sponge") == "sponge" else
                         " (its Stacey / free-surface extension mode)"),
            "wall_s": time.perf_counter() - t0}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mun", choices=["mun", "reference"])
    ap.add_argument("--models", type=int, default=256)
    ap.add_argument("--nt", type=int, default=3000)
    ap.add_argument("--plain", type=int, default=10, help="one-at-a-time solves timed")
    ap.add_argument("--tile", default="auto", help="tile kernel shape EXxEZ, or auto")
    ap.add_argument("--graph-chunk", type=int, default=0)
    ap.add_argument("--kernel", type=int, default=0, help="0 auto, 1 tile, 2 strip")
    ap.add_argument("--ckpt-k", type=int, default=0)
    ap.add_argument("--ref-nt", type=int, default=0, help="reference arm sample steps (0 = full solve)")
    ap.add_argument("--cpu-nt", type=int, default=0, help="cpu_baseline sample steps (0 = full solve)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="single/uneven workloads: oracle CPU estimate from this many steps (0 = none)")
    ap.add_argument("--workload", default="elbo", choices=["elbo", "plain", "uneven", "serving", "single"])
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-requests", type=int, default=400)
    ap.add_argument("--serve-T", type=float, default=0.25)
    ap.add_argument("--serve-slots", type=int, default=256)
    ap.add_argument("--serve-cap-gb", type=float, default=150.0)
    ap.add_argument("--serve-ticks", type=int, default=32)
    ap.add_argument("--clocks-log", default="", help="nvidia-smi clock samples (default: a temp file)")
    ap.add_argument("--boundary", default="sponge", choices=["sponge", "stacey"],
                    help="the reference's sponge, or Stacey sides/bottom with a free surface (plain and "
                         "default workloads)")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload: skip the parity, single, uneven and serving legs")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "plain":
        return run_plain(args)
    if args.workload == "uneven":
        return run_uneven(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "single":
        return run_single(args)

    import torch
    import torch.distributed as dist
    from mun_b200 import Batch, SEMPlan, SolveSpec

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    W = workload(nmodels=args.models, nt=args.nt, seed0=1000 * rank, boundary=args.boundary)
    plan = SEMPlan(**W["plan_kw"])
    dev = torch.device("cuda", local)
    tex, tez = parse_tile(args.tile)
    batch = Batch(tile=(tex, tez), graph_chunk=args.graph_chunk, kernel=args.kernel)
    stream = torch.cuda.Stream()

    # observed data from the "true" model, once
    with torch.cuda.stream(stream):
        obs = SolveSpec(plan, torch.as_tensor(W["v_true"], device=dev), shift=True)
        batch.run([obs])
    stream.synchronize()
    y = obs.rec.double()
    inv_s2 = 1.0 / (W["sigma"] ** 2 + 1e-24)
    vel_dev = torch.as_tensor(W["vels"], device=dev)
    n = args.models

    def make_specs(v):
        return [SolveSpec(plan, v[i], adjoint=True, y_obs=y, inv_sigma2=inv_s2, ckpt_k=args.ckpt_k)
                for i in range(n)]

    def barrier():
        if world > 1:
            dist.barrier()

    # ---------------- device-resident batched step
    specs = make_specs(vel_dev)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            batch.run(specs)
    stream.synchronize()
    launches_per_step = batch.last_launches
    kernel_used = batch.last_kernel
    groups_used = batch.last_groups
    shape_used = batch.last_shape
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_ms, tick_ms = [], []
    clocks = Clocks(args.clocks_log or os.path.join(tempfile.gettempdir(), f"mun_b200_clocks_r{rank}.csv"))
    barrier()
    torch.cuda.synchronize()
    with clocks:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                ev0.record(stream)
                batch.run(specs)
                ev1.record(stream)
            ev1.synchronize()
            step_ms.append(ev0.elapsed_time(ev1))
            tick_ms.append(batch.last_tick_ms())
    torch.cuda.synchronize()
    barrier()
    ms = float(np.mean(step_ms))
    ticks_per_step = batch.last_ticks
    # node-ticks of each kind per step: every group runs nt adjoint ticks, a read-out and
    # a scale tick; its remaining ticks are forward or replay ticks
    fwd_like = ticks_per_step - groups_used * (W["nt"] + 2)
    # algorithmic bytes of the step's tick launches: 56 B per node-step (replay ticks are
    # overhead and carry none)
    kern_bytes = BYTES_PER_NODE_STEP_FWDADJ * W["npoints"] * W["nt"] * n
    tick_loop_ms = float(np.mean(tick_ms))
    ms = max_over_ranks(ms, world, dev)
    status = torch.cat([s.status for s in specs]).max().item()
    value = n * world / (ms / 1e3)

    # ---------------- end to end through the public API with host buffers
    pin_v = torch.as_tensor(W["vels"]).pin_memory()
    pin_y = y.cpu().pin_memory()
    out_g = torch.empty((n, W["npoints"]), dtype=torch.float64).pin_memory()
    out_l = torch.empty(n, dtype=torch.float64).pin_memory()
    e2e_ms = []
    for it in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            ev0.record(stream)
            v = pin_v.to(dev, non_blocking=True)
            yy = pin_y.to(dev, non_blocking=True)
            sp = [SolveSpec(plan, v[i], adjoint=True, y_obs=yy, inv_sigma2=inv_s2, ckpt_k=args.ckpt_k)
                  for i in range(n)]
            batch.run(sp)
            out_g.copy_(torch.stack([s.grad for s in sp]), non_blocking=True)
            out_l.copy_(torch.cat([s.loglik for s in sp]), non_blocking=True)
            ev1.record(stream)
        ev1.synchronize()
        if it >= args.warmup:
            e2e_ms.append(ev0.elapsed_time(ev1))
    e2e = max_over_ranks(float(np.mean(e2e_ms)), world, dev)
    h2d = pin_v.numel() * 8 + pin_y.numel() * 8
    d2h = out_g.numel() * 8 + out_l.numel() * 8

    # ---------------- plain: one solve at a time (same models, best single-solve kernel)
    plain_ms = []
    pbatch = Batch(tile=(tex, tez), graph_chunk=args.graph_chunk, kernel=0)
    with torch.cuda.stream(stream):
        for i in range(args.warmup + args.plain):
            s = SolveSpec(plan, vel_dev[i % n], adjoint=True, y_obs=y, inv_sigma2=inv_s2,
                          ckpt_k=args.ckpt_k)
            ev0.record(stream)
            pbatch.run([s])
            ev1.record(stream)
            ev1.synchronize()
            if i >= args.warmup:
                plain_ms.append(ev0.elapsed_time(ev1))
    plain_kernel = pbatch.last_kernel
    plain_shape = pbatch.last_shape
    plain_ms = np.array(plain_ms)
    # a single solve's ticks are short, so a late host launch stalls the GPU: the median solve
    # is the plain path's figure (the mean is reported beside it)
    plain_value = 1e3 / float(np.median(plain_ms))

    # ---------------- roofline of the dominant kernel (the tick kernel, one launch per tick)
    pk, pk_kind = peaks()
    alg_bytes = BYTES_PER_NODE_STEP_FWDADJ * W["npoints"] * W["nt"] * n
    step_achieved = alg_bytes / (ms / 1e3) / 1e9
    achieved = kern_bytes / (tick_loop_ms / 1e3) / 1e9
    peak = float(pk.get("hbm_gbs", 6650.0))
    # DRAM traffic per node of each tick kind from the ncu capture of the strip kernel
    # (128 models, per node), averaged over the step's ticks like the algorithmic bytes
    traffic = None
    if kernel_used == "strip" and TRAFFIC_B_PER_NODE:
        traffic = W["npoints"] * (n // groups_used) * (
            TRAFFIC_B_PER_NODE["fwd"] * fwd_like + TRAFFIC_B_PER_NODE["adj"] * groups_used * W["nt"]
        ) / ticks_per_step

    # ---------------- parity of two of the models against the float64 oracle (host)
    parity = None
    if rank == 0 and not args.no_extras:
        parity = parity_leg(W, specs, y, [0, n - 1])

    # ---------------- compact runs of the other workloads (device-timed, one solve set each)
    extras = {}
    # the batches' arenas (the 256-model step keeps ~128 GB) go back before the other legs
    del batch, pbatch
    import gc
    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    if rank == 0 and not args.no_extras:
        extras["stacey"] = stacey_leg(args)
        gc.collect()
        torch.cuda.empty_cache()
        extras["single"] = run_single(args, steps=2, warmup=1, cpu_sample=0, emit=False)
        extras["uneven"] = run_uneven(args, steps=1, warmup=1, plain=4, cpu_sample=0, emit=False)
        extras["serving"] = run_serving(args, requests=100, emit=False)

    cpu = None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        per, el = cpu_baseline(W, args.cpu_nt, threads)
        full = args.cpu_nt <= 0 or args.cpu_nt >= W["nt"]
        cpu = {"value": 1.0 / per, "unit": "solves/s", "cores": threads, "kind": "port",
               "sample": (f"1 model, one full {W['nt']}-step fwd+adj solve ({el:.1f} s)" if full else
                          f"1 model, {args.cpu_nt}- and {2 * args.cpu_nt}-step runs of {W['nt']} "
                          f"({el:.1f} s), fitted set-up + per-step cost")}
    if rank == 0:
        out = {
            "metric": "SEM fwd+adjoint solves/s (batched vs plain, same GPU, <=1e-4 rel); p50/p99 ms",
            "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 state / f64 gradient time-sum (f32 partials of <=16 ticks folded into f64) / f64 misfit",
            "data": "synthetic",
            "config": {"workload": WORKLOAD_ELBO,
                       "models_per_gpu": n, "nodes": W["npoints"], "nt": W["nt"],
                       "kernel": kernel_used, "shape (tile_ex, tile_ez, strip_bands)": shape_used,
                       "graph_chunk": args.graph_chunk,
                       "ckpt_k": args.ckpt_k or "auto", "groups": groups_used,
                       "l2": "inputs larger than L2 (state+c2 of 256 models ~250 MB per field set)",
                       "parallelism": f"replicas x{world}"},
            "plain": {"value": plain_value, "unit": "solves/s", "statistic": "median solve",
                      "kernel": plain_kernel, "shape": plain_shape,
                      "p50_ms": float(np.percentile(plain_ms, 50)), "mean_ms": float(plain_ms.mean()),
                      "p99_ms": float(np.percentile(plain_ms, 99)), "solves": int(len(plain_ms))},
            "batched_over_plain": value / world / plain_value,
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99))},
            "mnode_steps_per_s": W["npoints"] * W["nt"] * n * world / (ms / 1e3) / 1e6,
            "e2e": {"value": n * world / (e2e / 1e3), "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": pk_kind,
                         "kernel": f"sem_{kernel_used}_kernel<4>",
                         "bytes_per_node_step": BYTES_PER_NODE_STEP_FWDADJ,
                         "bytes_per_node": {"forward_tick": BYTES_PER_NODE_FWD_TICK,
                                            "adjoint_tick": BYTES_PER_NODE_ADJ_TICK},
                         "kernel_bytes_per_node": IMPL_BYTES_PER_NODE,
                         "launch_us_avg": 1e3 * tick_loop_ms / ticks_per_step,
                         "ticks_per_step": ticks_per_step, "forward_like_ticks": fwd_like,
                         "note": "algorithmic bytes (56 per fwd+adj node-step) of the step's tick "
                                 "launches over the CUDA-event time of the tick loops (one "
                                 "tick-kernel launch per tick, chained by programmatic dependent "
                                 "launch); traffic = ncu DRAM bytes per launch",
                         "step_level": {"bytes_per_node_step": BYTES_PER_NODE_STEP_FWDADJ,
                                        "achieved": step_achieved,
                                        "frac": step_achieved / peak}},
            "cpu_baseline": cpu,
            "parity": parity,
            **extras,
            "gpu_launches": int(launches_per_step * args.steps),
            "status": int(status),
            "clocks": clocks.summary(local),
        }
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
