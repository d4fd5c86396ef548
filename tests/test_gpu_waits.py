"""Time limits of the device waits, exercised without a GPU fault: a ring wait whose
bytes never arrive and a grid barrier one arrival short give up after about 2 s with
SEM_ERR_TIMEOUT in the status, and the context stays usable (a solve runs after them)."""
import ctypes as C
import time

import pytest
import torch

from mun_b200 import Batch, SolveSpec, _lib
from tests.goldens import load
from tests.gpu_cases import dev, plan_for

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which,expect", [(0, _lib.SEM_ERR_TIMEOUT), (1, _lib.SEM_ERR_TIMEOUT), (2, 0)])
def test_wait_gives_up_with_status(which, expect):
    lib = _lib.load()
    st = C.c_int32(-1)
    t0 = time.perf_counter()
    _lib.check(lib.sem_selftest_wait(which, C.byref(st)))
    dt = time.perf_counter() - t0
    assert st.value == expect
    if expect:
        assert 1.5 < dt < 30.0
    # the context is still usable
    g = load("inject_n2")
    plan = plan_for(g["config"], g["dt"], g["nt"])
    s = SolveSpec(plan, dev(g["velocity"]))
    Batch().run([s])
    torch.cuda.synchronize()
    assert int(s.status.item()) == 0
