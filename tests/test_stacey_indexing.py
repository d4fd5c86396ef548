"""CPU audit of the Stacey mode's table indexing (mirrors bnd_slot, bnd_sens and the
history writes in sem_kernels.cu): every absorbing-edge node below the free surface has
one slot inside the table row, no two nodes share a slot, the coefficient reads stay in
their rows, and the history rows written by forward ticks (t + 1 <= nt) and read by
adjoint ticks (t and t + 2, t <= nt - 2) lie inside the nt + 1 rows the workspace holds;
the plan's slot layout agrees with the kernel's."""
import numpy as np
import pytest

from mun_b200.plan import boundary_slots


def bnd_slot(gx, gz, nxg, nzg):
    if gx == 0:
        return gz
    if gx == nxg - 1:
        return nzg + gz
    if gz == nzg - 1:
        return 2 * nzg + gx
    return -1


@pytest.mark.parametrize("N,nelx,nelz,nt", [(4, 100, 50, 3000), (4, 400, 200, 5000), (1, 3, 2, 5),
                                            (3, 7, 4, 40), (7, 2, 1, 3)])
def test_slots_and_history_rows(N, nelx, nelz, nt):
    nxg, nzg = nelx * N + 1, nelz * N + 1
    nb = 2 * nzg + nxg
    pitch = (nb + 63) // 64 * 64
    nb_plan, pgx, pgz, used = boundary_slots(nelx, nelz, N)
    assert nb_plan == nb
    seen = {}
    for gz in range(1, nzg):                 # gz = 0 is the free surface: no slot is used
        for gx in range(nxg):
            k = bnd_slot(gx, gz, nxg, nzg)
            edge = gx == 0 or gx == nxg - 1 or gz == nzg - 1
            assert (k >= 0) == edge
            if k >= 0:
                assert 0 <= k < nb <= pitch and k not in seen
                seen[k] = (gx, gz)
                assert used[k] and pgx[k] == gx and pgz[k] == gz
                for row in (0, 1, 2):        # e1, e2, g
                    assert row * pitch + k < 3 * pitch
    # slots the kernels never address are the plan's unused ones or top-row side slots
    for k in range(nb):
        if k not in seen:
            assert (not used[k]) or pgz[k] == 0
    # history: forward / replay tick t writes row t + 1; adjoint tick t <= nt - 2 reads t, t + 2
    rows = nt + 1
    for t in (0, nt // 2, nt - 1):
        assert 0 <= t + 1 < rows
    for t in (0, max(0, nt - 2)):
        if t <= nt - 2:
            assert 0 <= t and t + 2 < rows
