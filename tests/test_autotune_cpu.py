"""Host logic of the autotuner's proxy (no GPU): the number of consecutive groups a batch's
workspaces with full forward histories need under the library's memory budget (85 % of
free device memory less 512 MiB), with the free-memory query and the plans' workspace
sizes faked."""
from types import SimpleNamespace

import pytest
import torch

from mun_b200 import autotune


def _history_bytes(nelx, nelz, npol, k):
    nxg, nzg = nelx * npol + 1, nelz * npol + 1
    return (k + 8) * ((nxg + 31) // 32 * 32) * nzg * 4


def _spec(nelx, nelz, npol, nt, adjoint=True):
    plan = SimpleNamespace(nelx=nelx, nelz=nelz, npol=npol, nt=nt,
                           workspace_bytes=lambda flags, k: _history_bytes(nelx, nelz, npol, k))
    return SimpleNamespace(plan=plan, adjoint=adjoint, flags=1 if adjoint else 0)


@pytest.mark.parametrize("free_gb,expect", [(179.0, 2), (400.0, 1), (60.0, 5)])
def test_group_count_follows_the_memory_budget(monkeypatch, free_gb, expect):
    free = int(free_gb * (1 << 30))
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda *a: (free, free))
    specs = [_spec(100, 50, 4, 3000) for _ in range(256)]
    per = _history_bytes(100, 50, 4, 3000)
    budget = 0.85 * free - (512 << 20)
    assert -(-256 * per // int(budget)) == expect
    assert autotune.group_count(specs) == expect


def test_group_count_bounds(monkeypatch):
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda *a: (1 << 30, 1 << 30))
    # forward-only solves keep no history: one group
    assert autotune.group_count([_spec(100, 50, 4, 3000, adjoint=False) for _ in range(8)]) == 1
    # never more groups than solves
    assert autotune.group_count([_spec(400, 200, 4, 5000) for _ in range(3)]) == 3
