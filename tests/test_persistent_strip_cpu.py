"""CPU audit of the persistent strip kernel's neighbour map (mirrors
sem_strip_persist_kernel): each CTA waits for the eight CTAs around it; those indices stay
inside the solve's own CTAs, the relation is symmetric, and every other CTA that owns a
node the chunk's bands use (halo columns of its rows, the halo band above, the shared row
below, and the corner node a receiver element read out of the last band can reach) is
among them.  The four edge neighbours alone would miss that corner."""
import pytest


def neighbours(local, ns, nzc, base):
    strip, chunk = divmod(local, nzc)
    out = []
    for ds in (-1, 0, 1):
        for dc in (-1, 0, 1):
            st, ch = strip + ds, chunk + dc
            if (ds or dc) and 0 <= st < ns and 0 <= ch < nzc:
                out.append(base + local + ds * nzc + dc)
    return out


def owner(gx, gz, ew, zch, N, nxg, nzg, ns, nzc):
    """CTA (local index) owning grid node (gx, gz): strip by owned columns, chunk by rows."""
    strip = min(gx // (ew * N), ns - 1) if gx < nxg - 1 else ns - 1
    chunk = min(gz // (zch * N), nzc - 1) if gz < nzg - 1 else nzc - 1
    return strip * nzc + chunk


@pytest.mark.parametrize("N,nelx,nelz,ew,zch", [(4, 100, 50, 25, 50), (4, 400, 200, 29, 5), (2, 12, 9, 5, 2),
                                                (3, 7, 4, 7, 4), (1, 9, 6, 3, 3)])
def test_neighbour_map(N, nelx, nelz, ew, zch):
    ns = -(-nelx // ew)
    nzc = -(-nelz // zch)
    nxg, nzg = nelx * N + 1, nelz * N + 1
    base = 17  # the solve's first CTA inside the group's grid
    total = ns * nzc
    for local in range(total):
        nb = neighbours(local, ns, nzc, base)
        assert all(base <= x < base + total for x in nb) and len(set(nb)) == len(nb)
        for x in nb:
            assert base + local in neighbours(x - base, ns, nzc, base)
        strip, chunk = divmod(local, nzc)
        e0, e1 = strip * ew, min(strip * ew + ew, nelx)
        zb0, zb1 = chunk * zch, min(chunk * zch + zch, nelz)
        used = set()
        # rows of the owned element rows (and the shared row below, which a receiver element
        # of the last element row spans): halo columns N to the left, the shared column right
        for gz in range(zb0 * N, zb1 * N + 1):
            for gx in range(max(e0 * N - N, 0), min(e1 * N, nxg - 1) + 1):
                used.add((gx, gz))
        # the halo band above (element row zb0 - 1), owned columns only
        if zb0 > 0:
            for gz in range((zb0 - 1) * N, zb0 * N):
                for gx in range(e0 * N, min(e1 * N, nxg - 1) + 1):
                    used.add((gx, gz))
        others = {owner(gx, gz, ew, zch, N, nxg, nzg, ns, nzc) for gx, gz in used} - {local}
        assert others <= {x - base for x in nb}, (local, others, nb)
