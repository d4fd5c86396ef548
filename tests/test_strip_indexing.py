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
    owner = np.zeros(nxg, dtype=int)
    for strip in range(ns):
        e0, e1 = strip * EW, min(strip * EW + EW, nelx)
        assert e1 > e0
        sx0 = e0 * N
        so1 = nxg if e1 == nelx else e1 * N
        NC = (e1 - e0) * N + N + 1
        assert NC <= THREADS
        X0 = (sx0 - N) & ~3
        off = (sx0 - N) - X0
        assert 0 <= off <= 3 and X0 % 4 == 0
        cs, ce = max(X0, 0), min(X0 + BW, pitch)
        assert cs % 4 == 0 and ce % 4 == 0 and ce > cs      # 16-byte aligned bulk copies
        assert (cs - X0) % 4 == 0 and ((ce - cs) * 4) % 16 == 0
        copied = set(range(cs, ce))
        qr_written, ql_written = set(), set()
        for tid in range(THREADS):
            gx = sx0 - N + tid
            valid = tid < NC and 0 <= gx < nxg
            if not valid:
                continue
            sc = tid + off
            assert 0 <= sc < BW
            er, ia = divmod(gx, N)
            if er < nelx and tid < NC - 1:
                for b in range(NP):
                    col = gx - ia + b
                    assert col in copied and 0 <= sc - ia + b < BW
                qr_written.add(tid)
            if ia == 0 and er >= 1 and tid >= N:
                for b in range(NP):
                    assert gx - N + b in copied
                ql_written.add(tid)
        for tid in range(THREADS):
            gx = sx0 - N + tid
            if not (tid < NC and 0 <= gx < nxg and sx0 <= gx < so1):
                continue
            owner[gx] += 1
            assert gx in copied
            er, ia = divmod(gx, N)
            cl = tid - ia
            if ia:
                need_r = [cl + p for p in range(N)]
                need_l = [cl + N]
            else:
                need_r, need_l = [], []
                if er >= 1:
                    need_r += [tid - N + p for p in range(N)]
                    need_l += [tid]
                if er < nelx:
                    need_r += [tid + p for p in range(N)]
                    need_l += [tid + N]
            assert all(c in qr_written for c in need_r), (strip, gx)
            assert all(c in ql_written for c in need_l), (strip, gx)
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
            # injection: every node owned by exactly one listed strip
            listed = []
            for s in range(ns):
                s0 = s * EW * N
                s1 = nxg if min((s + 1) * EW, nelx) == nelx else (s + 1) * EW * N
                if bx + N >= s0 and bx < s1:
                    listed.append((s0, s1))
            for i in range(N + 1):
                assert sum(s0 <= bx + i < s1 for s0, s1 in listed) == 1
