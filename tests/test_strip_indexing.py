"""CPU audit of the strip kernel's index arithmetic (mirrors sem_strip_kernel in
sem_kernels.cu): TMA copy ranges and alignment, shared-memory reads inside the copied
columns, phase-B flux reads only where phase A wrote, exact partition of the owned
columns, and coverage of the per-band receiver lists."""
import numpy as np
import pytest

THREADS = 128


def bw(N):
    return (THREADS + 3 + 3) & ~3


def ew_max(N):
    return (THREADS - N - 1) // N


def strips_of(nelx, N):
    ns = -(-nelx // ew_max(N))
    ew = -(-nelx // ns)
    ns = -(-nelx // ew)
    return ns, ew


def pitch_of(nxg):
    return -(-nxg // 32) * 32


def audit(N, nelx, nelz):
    NP = N + 1
    nxg = nelx * N + 1
    pitch = pitch_of(nxg)
    ns, EW = strips_of(nelx, N)
    BW = bw(N)
    SEGS = (THREADS - N - 1) // N + 1
    owner = np.zeros(nxg, dtype=int)
    for strip in range(ns):
        e0, e1 = strip * EW, min(strip * EW + EW, nelx)
        assert e1 > e0
        sx0 = e0 * N
        so1 = nxg if e1 == nelx else e1 * N
        X0 = (sx0 - N) & ~3
        off = (sx0 - N) - X0
        assert 0 <= off <= 3 and X0 % 4 == 0
        cs, ce = max(X0, 0), min(X0 + BW, pitch)
        assert cs % 4 == 0 and ce % 4 == 0 and ce > cs      # 16-byte aligned bulk copies
        assert (cs - X0) % 4 == 0 and ((ce - cs) * 4) % 16 == 0
        copied = set(range(cs, ce))
        nseg = e1 - e0 + 1
        seg0 = 1 if e0 == 0 else 0
        assert nseg <= SEGS
        written = set()
        for sgi in range(seg0, nseg):        # phase A x-items read the segment's columns
            for b in range(NP):
                sm_col = off + sgi * N + b
                assert 0 <= sm_col < BW
                assert X0 + sm_col in copied
            written.add(sgi)
        assert so1 - sx0 <= THREADS
        for tid in range(THREADS):
            gx = sx0 + tid
            if gx >= so1:
                continue
            owner[gx] += 1
            sc = tid + N + off
            assert 0 <= sc < BW and X0 + sc == gx and gx in copied   # z-column and node reads
            er, ia = divmod(gx, N)
            s_r = er - e0 + 1
            need = [s_r] if ia else ([s_r - 1] if er >= 1 else []) + ([s_r] if er < nelx else [])
            assert need and all(x in written for x in need), (strip, gx)
    assert (owner == 1).all()


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
def test_strip_index_arithmetic(N):
    for nelx, nelz in ((1, 1), (7, 3), (30, 5), (100, 50), (131, 2), (200, 4)):
        audit(N, nelx, nelz)


def test_strip_receiver_lists_cover():
    rng = np.random.default_rng(0)
    for N, nelx, nelz in ((4, 100, 50), (3, 90, 20), (5, 47, 9), (1, 300, 3)):
        nxg = nelx * N + 1
        ns, EW = strips_of(nelx, N)
        for _ in range(100):
            ex, ez = rng.integers(nelx), rng.integers(nelz)
            bx = ex * N
            rec_strip = ex // EW
            e0 = rec_strip * EW
            sx0 = e0 * N
            X0 = (sx0 - N) & ~3
            # recording strip has the whole element in its copied columns
            assert bx - X0 >= 0 and bx + N - X0 < bw(N)
            assert bx + N <= min(X0 + bw(N), -(-nxg // 32) * 32) - 1
            # injection: every node owned by exactly one listed strip
            listed = []
            for s in range(ns):
                s0 = s * EW * N
                s1 = nxg if min((s + 1) * EW, nelx) == nelx else (s + 1) * EW * N
                if bx + N >= s0 and bx < s1:
                    listed.append((s0, s1))
            for i in range(N + 1):
                assert sum(s0 <= bx + i < s1 for s0, s1 in listed) == 1
