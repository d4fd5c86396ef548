"""CPU audit of the tick kernel's tile index arithmetic (mirrors sem_kernels.cu).

For a range of orders, tile shapes and mesh sizes it checks that every shared-memory
read lies inside the staged halo region and the allocation, that segment results are
only read where they were written, that every node is owned by exactly one tile, and
that the receiver tile lists cover recording and injection."""
import itertools

import numpy as np
import pytest


def region_w(tex, N):
    return ((tex + 2) * N + 1) | 1


def region_h(tez, N):
    return (tez + 2) * N + 1


def smem_floats(N, tex, tez, adj):
    NP = N + 1
    reg = region_w(tex, N) * region_h(tez, N)
    nro, nco = (tez * N + 1) | 1, (tex * N + 1) | 1
    xseg, zseg = (tex + 1) * NP * nro, (tez + 1) * NP * nco
    f = 96 + 2 * reg + xseg + zseg
    if adj:
        f += reg + xseg + zseg + nro * nco + 1024
    return f


def audit(N, nelx, nelz, tex, tez):
    NP = N + 1
    nxg, nzg = nelx * N + 1, nelz * N + 1
    ntx, ntz = -(-nelx // tex), -(-nelz // tez)
    owner = np.zeros((nzg, nxg), dtype=int)
    SW, SH = region_w(tex, N), region_h(tez, N)
    nrop_max, ncop_max = (tez * N + 1) | 1, (tex * N + 1) | 1
    for tz, tx in itertools.product(range(ntz), range(ntx)):
        ex0, ex1 = tx * tex, min(tx * tex + tex, nelx)
        ez0, ez1 = tz * tez, min(tz * tez + tez, nelz)
        gxo0, gxo1 = ex0 * N, (nxg if ex1 == nelx else ex1 * N)
        gzo0, gzo1 = ez0 * N, (nzg if ez1 == nelz else ez1 * N)
        nco, nro = gxo1 - gxo0, gzo1 - gzo0
        gxs, gzs = gxo0 - N, gzo0 - N
        segx0, nsx = max(ex0 - 1, 0), ex1 - max(ex0 - 1, 0)
        segz0, nsz = max(ez0 - 1, 0), ez1 - max(ez0 - 1, 0)
        nrop, ncop = nro | 1, nco | 1
        assert nro <= tez * N + 1 and nco <= tex * N + 1
        assert nsx <= tex + 1 and nsz <= tez + 1
        r0, r1 = max(gzs, 0), min(gzs + SH, nzg)
        c0, c1 = max(gxs, 0), min(gxs + (ex1 - ex0 + 2) * N + 1, nxg)
        assert c1 - gxs <= SW and r1 - gzs <= SH
        loaded = lambda gz, gx: r0 <= gz < r1 and c0 <= gx < c1  # noqa: E731
        owner[gzo0:gzo1, gxo0:gxo1] += 1
        xw, zw = set(), set()
        for r in range(nro):
            for sg in range(nsx):
                ex = segx0 + sg
                for a in range(NP):
                    gz, gx = gzo0 + r, ex * N + a
                    assert loaded(gz, gx), (gz, gx)
                    assert 0 <= (gz - gzs) * SW + (gx - gxs) < SW * SH
                    idx = (sg * NP + a) * nrop + r
                    assert idx < (tex + 1) * NP * nrop_max
                    xw.add(idx)
        for cc in range(nco):
            for sg in range(nsz):
                ez = segz0 + sg
                for a in range(NP):
                    gz, gx = ez * N + a, gxo0 + cc
                    assert loaded(gz, gx), (gz, gx)
                    idx = (sg * NP + a) * ncop + cc
                    assert idx < (tez + 1) * NP * ncop_max
                    zw.add(idx)
        for r in range(nro):
            for cc in range(nco):
                gx, gz = gxo0 + cc, gzo0 + r
                assert loaded(gz, gx)
                exr, ia = divmod(gx, N)
                ezr, ja = divmod(gz, N)
                reads_x, reads_z = [], []
                if ia:
                    reads_x.append(((exr - segx0) * NP + ia) * nrop + r)
                else:
                    if exr >= 1:
                        reads_x.append(((exr - 1 - segx0) * NP + N) * nrop + r)
                    if exr < nelx:
                        reads_x.append(((exr - segx0) * NP) * nrop + r)
                if ja:
                    reads_z.append(((ezr - segz0) * NP + ja) * ncop + cc)
                else:
                    if ezr >= 1:
                        reads_z.append(((ezr - 1 - segz0) * NP + N) * ncop + cc)
                    if ezr < nelz:
                        reads_z.append(((ezr - segz0) * NP) * ncop + cc)
                assert reads_x and reads_z
                assert all(i in xw for i in reads_x), (gx, gz)
                assert all(i in zw for i in reads_z), (gx, gz)
                assert r * nco + cc < nrop_max * ncop_max
    assert (owner == 1).all()
    return ntx, ntz


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("tiles", [(8, 8), (4, 2), (1, 1), (16, 4), (3, 5)])
def test_tile_index_arithmetic(N, tiles):
    for nelx, nelz in ((7, 5), (1, 1), (16, 9), (13, 3)):
        audit(N, nelx, nelz, *tiles)
    assert smem_floats(N, *tiles, True) * 4 <= 227 * 1024 or max(tiles) > 8


def test_receiver_tile_lists_cover_elements():
    rng = np.random.default_rng(0)
    for N, nelx, nelz, tex, tez in ((4, 40, 20, 8, 8), (3, 13, 7, 4, 3), (5, 9, 9, 2, 5)):
        nxg, nzg = nelx * N + 1, nelz * N + 1
        ntx, ntz = -(-nelx // tex), -(-nelz // tez)
        for _ in range(50):
            ex, ez = rng.integers(nelx), rng.integers(nelz)
            bx, bz = ex * N, ez * N
            rec_tile = (ez // tez) * ntx + (ex // tex)
            tx, tz = rec_tile % ntx, rec_tile // ntx
            # recording tile stages the whole element
            gxs, gzs = tx * tex * N - N, tz * tez * N - N
            ex1 = min(tx * tex + tex, nelx)
            assert bx - gxs >= 0 and bx + N <= min(gxs + (ex1 - tx * tex + 2) * N, nxg - 1)
            assert bz - gzs >= 0
            # injection: every element node has an owner among the listed tiles
            tiles = set()
            for j in range(N + 1):
                for i in range(N + 1):
                    ox = min((bx + i) // (tex * N), ntx - 1)
                    oz = min((bz + j) // (tez * N), ntz - 1)
                    tiles.add((ox, oz))
                    gxo0 = ox * tex * N
                    gxo1 = nxg if min(ox * tex + tex, nelx) == nelx else (ox * tex + tex) * N
                    assert gxo0 <= bx + i < gxo1
            assert 1 <= len(tiles) <= 4
