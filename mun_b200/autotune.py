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
STRIP_BAND_CANDIDATES = [0, 4, 8]  # strip kernel: element rows per CTA (0: automatic)
PERSIST_STRIP_BAND_CANDIDATES = [0, 2, 4]  # persistent strip kernel (one launch for all ticks)

_cache = {}


def signature(specs):
    shapes = tuple(sorted((s.plan.nelx, s.plan.nelz, s.plan.npol) for s in specs))
    return (shapes, len(specs), any(s.adjoint for s in specs))


def _proxy_plan(plan, nt_proxy):
    a = plan.arrays
    kw = dict(plan.kwargs)
    kw["nt"] = min(int(nt_proxy), plan.nt)
    return SEMPlan(**kw)


def tune(specs, nt_proxy=48, repeats=2, candidates=None, verbose=False):
    """Return ``dict(kernel=..., tile=..., graph_chunk=..., strip_bands=..., ckpt_k=...)``
    for ``specs``: the elements per CTA (tile shape, or strip chunk height), the kernel
    variant and the graph chunk, timed; ``ckpt_k = 0`` leaves the checkpoint interval and
    the group split to the library's memory-budget cost model at run time."""
    key = signature(specs)
    if key in _cache:
        return _cache[key]
    proxies = {}
    for s in specs:
        if id(s.plan) not in proxies:
            proxies[id(s.plan)] = _proxy_plan(s.plan, nt_proxy)

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
        try:
            with torch.cuda.stream(stream):
                b.run(proxy_specs())  # warm-up (plan lists, graph instantiation)
            stream.synchronize()
            times = []
            for _ in range(repeats):
                sp = proxy_specs()
                t0 = time.perf_counter()
                with torch.cuda.stream(stream):
                    b.run(sp)
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
           "proxy_ms": 1e3 * best_t}
    _cache[key] = res
    return res


def tuned_batch(specs, **kw):
    """A ``Batch`` configured by ``tune`` (checkpointing stays automatic)."""
    cfg = tune(specs, **kw)
    return Batch(tile=cfg["tile"] if cfg["kernel"] in (1, 3) else (8, 8), graph_chunk=cfg["graph_chunk"],
                 kernel=cfg["kernel"], strip_bands=cfg["strip_bands"]), cfg
