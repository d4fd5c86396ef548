"""The allocation-free forward entry point, ``sem_forward_noalloc``, against the
allocating ``sem_forward``.

Some callers of this solver cannot allocate device memory while they run: a
framework whose memory pool owns the whole GPU, a real-time request loop that must not
hit cudaMalloc's implicit device synchronisation, or an embedding that brings its own
allocator.  ``sem_forward_noalloc`` serves them from a fixed scratch array compiled
into the library.  Both calls go through the C ABI.  Two calls in a row with different
velocities must each match the allocating path, which shows that the second call does
not see the state the first call left in the shared scratch.  The tile kernel's
arithmetic per node does not depend on the tile shape, so the traces are bitwise those
of the allocating call; they are also checked against the reference's own traces (the
golden ``rec_run``) at the parity tolerance, and the device's free memory must not
change across a call.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from mun_b200 import SEMPlan, _lib
from tests.goldens import load, rel_l2
from tests.gpu_cases import dev, plan_for

pytestmark = pytest.mark.gpu
TOL = 1e-4  # relative L2, as in the other GPU parity tests


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _noalloc(lib, plan, v):
    rec = torch.full((plan.nt, plan.nrec), float("nan"), dtype=torch.float32, device="cuda")
    st = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    _lib.check(lib.sem_forward_noalloc(plan.handle, C.c_void_p(v.data_ptr()),
                                       C.c_void_p(rec.data_ptr()), C.c_void_p(st.data_ptr()),
                                       _stream()))
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return rec


def _allocating(lib, batch, plan, v):
    rec = torch.empty((plan.nt, plan.nrec), dtype=torch.float32, device="cuda")
    _lib.check(lib.sem_forward(batch, plan.handle, C.c_void_p(v.data_ptr()),
                               C.c_void_p(rec.data_ptr()), _stream()))
    torch.cuda.synchronize()
    return rec


def test_no_alloc_forward_matches_allocating_entry_point_twice():
    lib = _lib.load()
    batch = C.c_void_p()
    _lib.check(lib.sem_batch_create(C.byref(batch)))
    try:
        for name in ("inject_n3", "layered_cfg0"):
            g = load(name)
            plan = plan_for(g["config"], g["dt_run"], g["nt_run"])
            v1 = dev(g["velocity"])
            v2 = dev(np.asarray(g["velocity"]) * 0.93 + 40.0)  # a different model
            for v in (v1, v2):  # two calls in a row on the shared scratch
                a = _noalloc(lib, plan, v)
                b = _allocating(lib, batch, plan, v)
                assert torch.isfinite(a).all()
                err = rel_l2(a.cpu().numpy(), b.cpu().numpy())
                assert err <= TOL, (name, err)
                assert torch.equal(a, b), name
            # the reference's own traces of the first model
            err_ref = rel_l2(_noalloc(lib, plan, v1).cpu().numpy(), g["rec_run"])
            assert err_ref <= TOL, (name, err_ref)
            # and the traces of the two models differ (the test would notice stale state)
            assert rel_l2(_noalloc(lib, plan, v1).cpu().numpy(),
                          _noalloc(lib, plan, v2).cpu().numpy()) > 1e-3
    finally:
        lib.sem_batch_destroy(batch)


def test_no_alloc_call_takes_no_device_memory():
    lib = _lib.load()
    g = load("inject_n3")
    plan = plan_for(g["config"], g["dt_run"], g["nt_run"])
    v = dev(g["velocity"])
    rec = torch.empty((plan.nt, plan.nrec), dtype=torch.float32, device="cuda")
    st = torch.empty((1,), dtype=torch.int32, device="cuda")
    args = (plan.handle, C.c_void_p(v.data_ptr()), C.c_void_p(rec.data_ptr()), C.c_void_p(st.data_ptr()))
    _lib.check(lib.sem_forward_noalloc(*args, _stream()))  # warm-up: kernels loaded
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        _lib.check(lib.sem_forward_noalloc(*args, _stream()))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert int(st.item()) == 0


def test_no_alloc_rejects_meshes_beyond_the_scratch():
    lib = _lib.load()
    rec = np.array([[1000.0, 500.0]])
    plan = SEMPlan(xmin=0.0, xmax=10000.0, zmin=0.0, zmax=5400.0, nelx=500, nelz=270, npol=4,
                   dt=1e-4, nt=4, src_xz=(5000.0, 100.0), f0=10.0, amp=1.0, receivers=rec,
                   pml_thickness=200.0, sponge_cmax=3000.0)
    v = torch.full((plan.npoints,), 2000.0, dtype=torch.float64, device="cuda")
    out = torch.empty((plan.nt, 1), dtype=torch.float32, device="cuda")
    rc = lib.sem_forward_noalloc(plan.handle, C.c_void_p(v.data_ptr()), C.c_void_p(out.data_ptr()),
                                 None, _stream())
    assert rc == _lib.SEM_ERR_ARG
    assert b"too large" in lib.sem_last_error()
