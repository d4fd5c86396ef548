"""Launch-configuration autotuner.

Picks the kernel variant (tile kernel with a tile shape, persistent tile kernel, strip
kernel or persistent strip kernel, with the strip chunk height) and the CUDA-graph chunk for a batch by timing candidates on a short proxy of the
batch: the same meshes, orders, receivers and velocities with a few dozen time steps.
The checkpoint interval and group split stay with the library's memory-budget schedule.
The choice is cached per batch signature (mesh sizes, orders, solve count, adjoint or
not).  Results never depend on the choice: every variant computes bitwise the same
numbers, so tuning only moves time.
"""
from __future__ import annotations

import time

import torch

from .plan import SEMPlan
from .solver import Batch, SolveSpec

# (0, 0): automatic.  4x3 and 3x3 tiles own at most 256 nodes at order 4 (one per thread of
# the 256-thread CTA), so a tick's node update is one pass
TILE_CANDIDATES = [(0, 0), (8, 8), (16, 8), (8, 4), (16, 4), (4, 4), (4, 3), (3, 3), (2, 2)]
GRAPH_CANDIDATES = [0, 32]
STRIP_BAND_CANDIDATES = [0, 4, 5, 6, 8, 10]  # strip kernel: element rows per CTA (0: automatic)
PERSIST_STRIP_BAND_CANDIDATES = [0, 2, 4]  # persistent strip kernel (one launch for all ticks)

_cache = {}


def signature(specs):
    shapes = tuple(sorted((s.plan.nelx, s.plan.nelz, s.plan.npol) for s in specs))
    return (shapes, len(specs), any(s.adjoint for s in specs))


def _proxy_plan(plan, nt_proxy):
    kw = dict(plan.kwargs)
    kw["nt"] = min(int(nt_proxy), plan.nt)
    return SEMPlan(**kw)


def group_count(specs):
    """Consecutive groups the library's automatic schedule is expected to run ``specs``
    in: the solves' workspaces with full forward histories (k = nt, no replay; the
    library's own layout, ``SEMPlan.workspace_bytes``) against the budget the schedule
    uses, 85 % of free device memory less 512 MiB."""
    free, _ = torch.cuda.mem_get_info()
    budget = 0.85 * free - (512 << 20)
    total = sum(s.plan.workspace_bytes(s.flags, s.plan.nt if s.adjoint else 2) for s in specs)
    return max(1, min(len(specs), -(-int(total) // max(int(budget), 1))))


def tune(specs, nt_proxy=48, repeats=2, candidates=None, verbose=False):
    """Return ``dict(kernel=..., tile=..., graph_chunk=..., strip_bands=..., ckpt_k=...)``
    for ``specs``: the elements per CTA (tile shape, or strip chunk height), the kernel
    variant and the graph chunk, timed; ``ckpt_k = 0`` leaves the checkpoint interval and
    the group split to the library's memory-budget cost model at run time."""
    key = signature(specs)
    if key in _cache:
        return _cache[key]
    # the proxy keeps the batch's shape over time: each solve's step count in proportion to
    # its own (the shortest at least 8 steps; a group lasts as long as its longest solve),
    # and the solves in the consecutive groups the real run's memory budget will split it into
    nt_max = max(s.plan.nt for s in specs)
    proxies = {}
    for s in specs:
        if id(s.plan) not in proxies:
            proxies[id(s.plan)] = _proxy_plan(s.plan, max(8, -(-nt_proxy * s.plan.nt // nt_max)))
    ngroups = group_count(specs)
    gsize = -(-len(specs) // ngroups)

    def proxy_specs():
        out = []
        for s in specs:
            p = proxies[id(s.plan)]
            y = None if s.y_obs is None else s.y_obs[:p.nt]
            out.append(SolveSpec(p, s.velocity, adjoint=s.adjoint, exact=s.exact, shift=s.shift,
                                 misfit=s.misfit, y_obs=y, inv_sigma2=s.inv_sigma2, ckpt_k=p.nt))
        return out

    # the persistent kernel is one launch per run (graphs do not apply); it falls back to
    # per-tick tile launches by itself when the tiles are not all resident
    cands = candidates or ([(1, t, g, 0) for t in TILE_CANDIDATES for g in GRAPH_CANDIDATES]
                           + [(3, t, 0, 0) for t in TILE_CANDIDATES]
                           + [(2, (0, 0), g, sb) for g in GRAPH_CANDIDATES for sb in STRIP_BAND_CANDIDATES]
                           + [(4, (0, 0), 0, sb) for sb in PERSIST_STRIP_BAND_CANDIDATES])
    best, best_t = None, float("inf")
    stream = torch.cuda.Stream()
    for cand in cands:
        kernel, tile, chunk, bands = tuple(cand) + (0,) * (4 - len(cand))
        b = Batch(tile=tile if kernel in (1, 3) else (8, 8), graph_chunk=chunk, kernel=kernel,
                  strip_bands=bands)
        def run_groups(sp):
            with torch.cuda.stream(stream):
                for g0 in range(0, len(sp), gsize):
                    b.run(sp[g0:g0 + gsize])

        try:
            run_groups(proxy_specs())  # warm-up (plan lists, graph instantiation)
            stream.synchronize()
            times = []
            for _ in range(repeats):
                sp = proxy_specs()
                t0 = time.perf_counter()
                run_groups(sp)
                stream.synchronize()
                times.append(time.perf_counter() - t0)
            el = min(times)
        except (ValueError, RuntimeError):
            continue
        if verbose:
            print(f"kernel={kernel} tile={tile} graph_chunk={chunk} strip_bands={bands}: {1e3 * el:.2f} ms")
        if el < best_t:
            best_t, best = el, (kernel, tile, chunk, bands)
    kernel, tile, chunk, bands = best
    # ckpt_k 0: the library picks the checkpoint interval and group split at run time
    res = {"kernel": kernel, "tile": tile, "graph_chunk": chunk, "strip_bands": bands, "ckpt_k": 0,
           "proxy_ms": 1e3 * best_t, "proxy_groups": ngroups}
    _cache[key] = res
    return res


def tuned_batch(specs, **kw):
    """A ``Batch`` configured by ``tune`` (checkpointing stays automatic)."""
    cfg = tune(specs, **kw)
    return Batch(tile=cfg["tile"] if cfg["kernel"] in (1, 3) else (8, 8), graph_chunk=cfg["graph_chunk"],
                 kernel=cfg["kernel"], strip_bands=cfg["strip_bands"]), cfg
