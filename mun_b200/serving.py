"""Continuous-batching request loop over the native serving engine (``sem_engine_*``).

Requests are forward-only likelihoods (MCMC proposals: forward with the misfit summed on
the device) and forward+adjoint gradients (flow-trainer samples).  The engine keeps
every admitted solve's wavefields and checkpoints resident in its arena and admits a
queued request at the next tick boundary as soon as a slot and enough device memory
(its workspace footprint, under the engine's byte cap) are free, so requests that
arrive while others run overlap with them on the device.  Each solve's result is
bitwise identical alone and in any mix (deterministic kernels, per-solve time
program).
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .solver import SolveSpec


class Engine:
    """Owns a ``sem_engine_t``."""

    def __init__(self, max_solves=512, memory_cap_bytes=8 << 30, ticks_per_step=16, kernel=0,
                 tile=(0, 0), stream=None):
        """kernel 0 / tile (0, 0): chosen per step for the running set (as in sem_run)."""
        lib = _lib.load()
        cfg = _lib.EngineCfg(int(max_solves), int(memory_cap_bytes), int(ticks_per_step), int(kernel),
                             int(tile[0]), int(tile[1]))
        h = C.c_void_p()
        _lib.check(lib.sem_engine_create(C.byref(cfg), C.byref(h)))
        self.handle, self._lib = h, lib
        self.stream = stream or torch.cuda.Stream()
        self._keep = {}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.sem_engine_destroy(h)
            except Exception:
                pass
            self.handle = None

    def submit(self, spec: SolveSpec) -> int:
        """Queue a solve; its output tensors are allocated here and stay alive until
        ``release``."""
        p = spec.plan
        dev = spec.velocity.device
        with torch.cuda.stream(self.stream):
            v = spec.velocity.contiguous()
            if spec.rec is None:
                spec.rec = torch.empty((p.nt, p.nrec), dtype=torch.float32, device=dev)
            y = None
            if spec.flags & (_lib.SEM_F_MISFIT | _lib.SEM_F_ADJOINT):
                y = spec.y_obs.to(device=dev, dtype=torch.float64).contiguous()
                spec.loglik = torch.empty(1, dtype=torch.float64, device=dev)
            if spec.adjoint:
                spec.grad = torch.empty(p.npoints, dtype=torch.float64, device=dev)
            spec.status = torch.zeros(1, dtype=torch.int32, device=dev)
        it0, it1, dec = spec.window if spec.window is not None else (0, p.nt, 1)
        s = _lib.Solve()
        s.plan = p.handle.value
        s.velocity = v.data_ptr()
        s.flags = spec.flags
        s.ckpt_k = int(spec.ckpt_k or p.nt)
        s.y_obs = y.data_ptr() if y is not None else None
        s.it0, s.it1, s.decim = int(it0), int(it1), int(dec)
        s.inv_sigma2 = float(spec.inv_sigma2)
        s.rec_out = spec.rec.data_ptr()
        s.loglik_out = spec.loglik.data_ptr() if spec.loglik is not None else None
        s.grad_out = spec.grad.data_ptr() if spec.grad is not None else None
        s.status_out = spec.status.data_ptr()
        t = C.c_int64()
        _lib.check(self._lib.sem_engine_submit(self.handle, C.byref(s), C.byref(t)))
        self._keep[t.value] = (spec, v, y)
        return t.value

    def step(self):
        _lib.check(self._lib.sem_engine_step(self.handle, C.c_void_p(self.stream.cuda_stream)))

    def state(self, ticket) -> int:
        st = C.c_int32()
        _lib.check(self._lib.sem_engine_status(self.handle, C.c_int64(ticket), C.byref(st)))
        return st.value

    def release(self, ticket):
        _lib.check(self._lib.sem_engine_release(self.handle, C.c_int64(ticket)))
        return self._keep.pop(ticket)[0]

    def stats(self):
        out = (C.c_int64 * 5)()
        _lib.check(self._lib.sem_engine_stats(self.handle, out))
        return {"queued": out[0], "running": out[1], "bytes_in_use": out[2], "tick": out[3],
                "launches": out[4]}

    def run_until_done(self, tickets, max_steps=10_000_000):
        pending = set(tickets)
        for _ in range(max_steps):
            if not pending:
                return
            self.step()
            for t in list(pending):
                if self.state(t) == 2:
                    pending.discard(t)
        raise RuntimeError("engine did not finish")


@dataclass
class Request:
    arrival: float          # seconds after the start of the stream
    spec: SolveSpec
    kind: str               # "mcmc" or "flow"
    ticket: int = -1
    done: float = field(default=None)


def serve(engine: Engine, requests, time_scale=1.0):
    """Play a request stream in (wall-clock) time: submit each request when its arrival
    time has passed, step the engine, record completion times.  Returns per-request
    latencies (s) and the wall time of the whole stream."""
    reqs = sorted(requests, key=lambda r: r.arrival)
    t0 = time.perf_counter()
    nxt = 0
    inflight = {}
    done = []
    while nxt < len(reqs) or inflight:
        now = time.perf_counter() - t0
        while nxt < len(reqs) and reqs[nxt].arrival * time_scale <= now:
            r = reqs[nxt]
            r.ticket = engine.submit(r.spec)
            inflight[r.ticket] = r
            nxt += 1
        if inflight:
            engine.step()
            for tk in list(inflight):
                if engine.state(tk) == 2:
                    r = inflight.pop(tk)
                    engine.release(tk)
                    r.done = time.perf_counter() - t0
                    done.append(r)
        elif nxt < len(reqs):
            time.sleep(max(0.0, reqs[nxt].arrival * time_scale - now))
    wall = time.perf_counter() - t0
    lat = np.array([r.done - r.arrival * time_scale for r in done])
    return done, lat, wall
