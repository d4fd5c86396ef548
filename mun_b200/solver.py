"""Batched solve API over the C ABI (``sem_run``).

A ``SolveSpec`` describes one solve: a plan, a nodal velocity on the device (float64,
reference node order) and what to compute.  ``Batch.run`` executes any list of specs
— mixed meshes, orders, step counts — as one tick-driven launch sequence, optionally
replayed from captured CUDA graphs, and fills the specs' output tensors.
"""
import ctypes as C
from dataclasses import dataclass, field

import torch

from . import _lib


@dataclass
class SolveSpec:
    plan: object
    velocity: torch.Tensor
    adjoint: bool = False
    exact: bool = False
    shift: bool = False          # record R u after the update (run_forward_and_adjoint)
    misfit: bool = False
    y_obs: torch.Tensor = None   # (n_obs, nrec) float64 on the device, misfit grid
    window: tuple = None         # (it0, it1, decim)
    inv_sigma2: float = 1.0
    ckpt_k: int = 0              # 0: the library picks k and the group split (memory budget)
    rec: torch.Tensor = None     # outputs
    loglik: torch.Tensor = None
    grad: torch.Tensor = None
    status: torch.Tensor = None
    tag: object = field(default=None, repr=False)

    @property
    def flags(self):
        f = 0
        if self.adjoint:
            f |= _lib.SEM_F_ADJOINT | _lib.SEM_F_SHIFT | _lib.SEM_F_MISFIT
        if self.exact:
            f |= _lib.SEM_F_EXACT
        if self.shift:
            f |= _lib.SEM_F_SHIFT
        if self.misfit:
            f |= _lib.SEM_F_MISFIT
        return f


def choose_ckpt_k(plan, n_solves, budget_bytes=None):
    """Largest checkpoint interval whose per-solve workspace fits the budget (k = nt
    stores the whole forward and skips the replay)."""
    if budget_bytes is None:
        free, _ = torch.cuda.mem_get_info()
        budget_bytes = int(0.7 * free)
    per = budget_bytes // max(1, n_solves)
    nt = plan.nt
    flags = _lib.SEM_F_ADJOINT | _lib.SEM_F_SHIFT
    if plan.workspace_bytes(flags, nt) <= per:
        return nt
    lo, hi = 2, nt
    while lo < hi:
        mid = (lo + hi + 1) // 2
        if plan.workspace_bytes(flags, mid) <= per:
            lo = mid
        else:
            hi = mid - 1
    # the workspace is minimal near sqrt(2 nt); never go below that
    return max(lo, min(nt, int((2 * nt) ** 0.5)))


class Batch:
    """Owns a ``sem_batch_t`` (workspace arena, descriptors, tick counter)."""

    def __init__(self, tile=(0, 0), threads=256, graph_chunk=0, kernel=0, strip_bands=0, autotune=False):
        """``autotune=True``: each ``run`` takes its kernel, tile shape or strip chunk height
        and graph chunk from ``mun_b200.autotune.tune`` for the batch's signature (timed once
        per signature on a short proxy, then cached); results do not depend on the choice."""
        lib = _lib.load()
        h = C.c_void_p()
        _lib.check(lib.sem_batch_create(C.byref(h)))
        self.handle, self._lib = h, lib
        self.tile, self.threads, self.graph_chunk = tuple(tile), int(threads), int(graph_chunk)
        self.kernel = int(kernel)  # 0 auto, 1 tile, 2 strip, 3 persistent tile, 4 persistent strip
        self.strip_bands = int(strip_bands)  # strip kernel: element rows per CTA (0 auto)
        self.autotune = bool(autotune)
        self.last_tuned = None
        self._side = None

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                torch.cuda.synchronize()
                self._lib.sem_batch_destroy(h)
            except Exception:
                pass
            self.handle = None

    @property
    def last_launches(self):
        return int(self._lib.sem_batch_last_launches(self.handle))

    @property
    def last_groups(self):
        """Consecutive groups the last run used (automatic checkpointing may split a
        batch so that each group's forward history fits the memory budget)."""
        return int(self._lib.sem_batch_last_groups(self.handle))

    @property
    def last_shape(self):
        """(tile_ex, tile_ez, strip_bands) of the last run (strip_bands 0: tile kernel)."""
        v = [C.c_int32() for _ in range(3)]
        _lib.check(self._lib.sem_batch_last_shape(self.handle, *[C.byref(x) for x in v]))
        return tuple(int(x.value) for x in v)

    @property
    def last_ticks(self):
        """Tick rounds the last run launched (summed over its groups)."""
        return int(self._lib.sem_batch_last_ticks(self.handle))

    def last_tick_ms(self):
        """Device time (ms) of the last run's tick loops, from CUDA events the library
        records on the run's stream around them; waits for those events."""
        ms = C.c_double()
        _lib.check(self._lib.sem_batch_last_tick_ms(self.handle, C.byref(ms)))
        return float(ms.value)

    @property
    def last_kernel(self):
        return {1: "tile", 2: "strip", 3: "persistent", 4: "persistent strip"}.get(
            int(self._lib.sem_batch_last_kernel(self.handle)), "none")

    def run(self, specs, tile=None, graph_chunk=None, memory_budget=None, kernel=None):
        n = len(specs)
        strip_bands = self.strip_bands
        if self.autotune and n:
            from .autotune import tune
            cfg = tune(specs)
            self.last_tuned = cfg
            kernel = cfg["kernel"] if kernel is None else kernel
            tile = (cfg["tile"] if cfg["kernel"] in (1, 3) else (8, 8)) if tile is None else tile
            graph_chunk = cfg["graph_chunk"] if graph_chunk is None else graph_chunk
            strip_bands = cfg["strip_bands"]
        arr = (_lib.Solve * max(n, 1))()
        keep = []
        for i, s in enumerate(specs):
            p = s.plan
            v = s.velocity
            if not (v.is_cuda and v.dtype == torch.float64 and v.numel() == p.npoints):
                raise ValueError("velocity must be a float64 CUDA tensor with npoints entries")
            v = v.contiguous()
            keep.append(v)
            dev = v.device
            if s.rec is None:
                s.rec = torch.empty((p.nt, p.nrec), dtype=torch.float32, device=dev)
            elif (tuple(s.rec.shape) != (p.nt, p.nrec) or s.rec.dtype != torch.float32
                  or not s.rec.is_contiguous() or s.rec.device != dev):
                raise ValueError("rec must be a contiguous float32 (nt, nrec) tensor on the device")
            flags = s.flags
            it0, it1, dec = s.window if s.window is not None else (0, p.nt, 1)
            if not (0 <= it0 < it1 <= p.nt and dec >= 1):
                raise ValueError(f"bad misfit window {(it0, it1, dec)} for nt={p.nt}")
            if flags & (_lib.SEM_F_MISFIT | _lib.SEM_F_ADJOINT):
                if s.y_obs is None:
                    raise ValueError("y_obs required for misfit/adjoint solves")
                y = s.y_obs.to(device=dev, dtype=torch.float64).contiguous()
                n_obs = -(-(it1 - it0) // dec)
                if y.dim() != 2 or y.shape[1] != p.nrec or y.shape[0] < n_obs:
                    raise ValueError(f"y_obs must be ({n_obs}, {p.nrec}) on the misfit grid, "
                                     f"got {tuple(y.shape)}")
                keep.append(y)
                if s.loglik is None:
                    s.loglik = torch.empty(1, dtype=torch.float64, device=dev)
            else:
                y = None
            if s.adjoint and s.grad is None:
                s.grad = torch.empty(p.npoints, dtype=torch.float64, device=dev)
            if s.status is None:
                s.status = torch.zeros(1, dtype=torch.int32, device=dev)
            # 0: the library picks the checkpoint interval and the group split
            k = s.ckpt_k if s.ckpt_k else (0 if s.adjoint else 2)
            a = arr[i]
            a.plan = p.handle.value
            a.velocity = v.data_ptr()
            a.flags = flags
            a.ckpt_k = int(k)
            a.y_obs = y.data_ptr() if y is not None else None
            a.it0, a.it1, a.decim = int(it0), int(it1), int(dec)
            a.inv_sigma2 = float(s.inv_sigma2)
            a.rec_out = s.rec.data_ptr()
            a.loglik_out = s.loglik.data_ptr() if s.loglik is not None else None
            a.grad_out = s.grad.data_ptr() if s.grad is not None else None
            a.status_out = s.status.data_ptr()
        t = tile or self.tile
        cfg = _lib.LaunchCfg(int(t[0]), int(t[1]), self.threads,
                             int(self.graph_chunk if graph_chunk is None else graph_chunk),
                             int(self.kernel if kernel is None else kernel), int(strip_bands),
                             int(memory_budget or 0))
        cur = torch.cuda.current_stream()
        if cfg.graph_chunk > 0 and cur.cuda_stream == 0:
            # graphs cannot be captured on the legacy default stream: use a side stream
            if self._side is None:
                self._side = torch.cuda.Stream()
            side = self._side
            side.wait_stream(cur)
            with torch.cuda.stream(side):
                rc = self._lib.sem_run(self.handle, arr, n, C.byref(cfg), C.c_void_p(side.cuda_stream))
            cur.wait_stream(side)
            for tt in keep:
                tt.record_stream(side)
            for s in specs:
                for o in (s.rec, s.loglik, s.grad, s.status):
                    if o is not None:
                        o.record_stream(side)
        else:
            rc = self._lib.sem_run(self.handle, arr, n, C.byref(cfg), C.c_void_p(cur.cuda_stream))
        _lib.check(rc)
        return specs


_default = {}


def _batch():
    dev = torch.cuda.current_device()
    if dev not in _default:
        _default[dev] = Batch()
    return _default[dev]


def forward(plan, velocity, shift=False):
    """Receiver traces (nt, nrec) float32 on the device."""
    s = SolveSpec(plan, velocity, shift=shift)
    _batch().run([s])
    return s.rec


def forward_adjoint(plan, velocity, y_obs, sigma, exact=False, ckpt_k=0, window=None):
    """dict(loglik, clean, grad = reference dJ_dv = d loglik / d c, status)."""
    s = SolveSpec(plan, velocity, adjoint=True, exact=exact, y_obs=y_obs,
                  inv_sigma2=1.0 / (float(sigma) ** 2 + 1e-24), ckpt_k=ckpt_k, window=window)
    _batch().run([s])
    return {"loglik": s.loglik, "clean": s.rec, "grad": s.grad, "status": s.status}
