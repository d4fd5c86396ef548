"""CPU audit of the strip kernel's index arithmetic (mirrors strip_tick in
sem_kernels.cu): TMA copy ranges and alignment, shared-memory reads inside the copied
columns, the thread-to-x-item map (every (row, segment) item exactly once), 16-byte
aligned segment loads for N = 4, phase-B flux reads only where phase A wrote, exact
partition of the owned columns, shared-memory totals, and coverage of the per-band
receiver lists."""
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
        if N == 4:
            assert off == 0                  # segment starts on 4-float boundaries (float4)
        # x-items: thread tid -> (row tid // nseg, segment tid % nseg) for rows 0..N-1;
        # row N of the last band by threads tid < nseg
        items = []
        for tid in range(THREADS):
            xa, xsg = divmod(tid, nseg)
            if xa < N and xsg >= seg0:
                items.append((xa, xsg))
            if tid < nseg and tid >= seg0:
                items.append((N, tid))
        assert sorted(items) == [(a, g) for a in range(NP) for g in range(seg0, nseg)]
        written = set()
        for a, sgi in items:                 # phase A x-items read the segment's columns
            o = a * BW + off + sgi * N
            if N == 4:
                assert o % 4 == 0
            for b in range(NP):
                sm_col = off + sgi * N + b
                assert 0 <= sm_col < BW
                assert X0 + sm_col in copied
            assert (a * SEGS + sgi) * NP + N < NP * SEGS * NP   # exchange buffer bound
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


STAGES, STAGES_ADJ, INJ, HDR, NBUF = 3, 3, 256, 192, 2


def field_floats(N):
    """strip_field_floats: one staged field of a band, rounded to 32 floats (128 bytes)."""
    return ((N + 1) * bw(N) + 31) & ~31


def smem_bytes(N, adj):
    """strip_smem_floats(N, adj) * 4: header, ring slots, exchange buffers, injection.
    The float64 gradient is not staged (owner threads load their rows)."""
    NP, segs = N + 1, ew_max(N) + 1

    def stage(a):
        return (4 if a else 3) * field_floats(N)

    def xch(a):
        f = NBUF * (2 if a else 1) * NP * segs * NP + ((NP * THREADS + INJ) if a else 0)
        return (f + 31) & ~31

    fwd = STAGES * stage(False) + xch(False)
    adjf = STAGES_ADJ * stage(True) + xch(True)
    return 4 * (HDR + (max(fwd, adjf) if adj else fwd))


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
def test_strip_shared_memory_layout(N):
    # header: 64 floats of mbarriers (>= ring slots), D (NP^2 <= 64), beta (<= 16),
    # z-table rows [2][3][8] (NP <= 8); ring starts 128-byte aligned
    assert max(STAGES, STAGES_ADJ) * 2 <= 64 and (N + 1) ** 2 <= 64 and N + 1 <= 8
    assert 64 + 64 + 16 + 48 == HDR and (HDR * 4) % 128 == 0
    assert 3 * (N + 1) <= THREADS          # threads staging the z-table rows
    for adj in (False, True):
        assert smem_bytes(N, adj) + 1024 <= 227 * 1024
    if N <= 4:                             # four CTAs per SM on the 228 KB SM
        assert 4 * (smem_bytes(N, True) + 1024 + 1024) <= 228 * 1024


def test_field_offsets_fit_int32():
    # plans whose padded field reaches 2^31 floats are refused (kernels use int offsets)
    for N, nelx, nelz in ((4, 100, 50), (7, 2000, 2000), (4, 8000, 8000)):
        nxg, nzg = nelx * N + 1, nelz * N + 1
        ok = pitch_of(nxg) * nzg < (1 << 31) - 64
        if ok:
            assert (nzg - 1) * pitch_of(nxg) + nxg < 2 ** 31


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


def zchunk_of(total_strips, nelz_max, sms=148, forced=0, min_chunk=4):
    """strip_zchunk in sem_kernels.cu."""
    if forced > 0:
        return forced
    if total_strips >= 2 * sms:
        return nelz_max
    want = -(-4 * sms // total_strips)
    return max(min_chunk, -(-nelz_max // want))


def test_strip_zchunk_rule():
    assert zchunk_of(512, 50) == 50                  # 128 models of 100x50: full height
    assert zchunk_of(14, 200) == 5                   # one 400x200 mesh: 14 strips x 40 chunks
    assert zchunk_of(4, 50) == 4                     # small mesh: at least 4 rows per chunk
    assert zchunk_of(200, 50, forced=3) == 3


@pytest.mark.parametrize("nelz,zch", [(1, 1), (5, 1), (5, 2), (50, 4), (50, 50), (200, 5), (7, 3)])
def test_strip_chunks_partition_and_ring(nelz, zch):
    nzc = -(-nelz // zch)
    owner = np.zeros(nelz, dtype=int)
    for final_only in (False, True):
        for NST in (2, 3):
            owner[:] = 0
            for chunk in range(nzc):
                zb0, zb1 = chunk * zch, min(nelz, chunk * zch + zch)
                assert zb1 > zb0
                has_halo = zb0 > 0 and not final_only
                ezs = zb0 - (1 if has_halo else 0)
                nbands = zb1 - ezs
                assert ezs >= 0
                # ring: band rel uses slot rel % NST with parity (rel // NST) & 1; a slot is
                # refilled (band rel - 1 + NST at the barrier of band rel) only after the
                # band that used it (rel - 1) is done, and every band is issued once
                issued = list(range(min(NST, nbands)))
                for rel in range(nbands):
                    assert rel in issued
                    if final_only:
                        if rel + NST < nbands:
                            issued.append(rel + NST)
                    elif rel >= 1 and rel - 1 + NST < nbands:
                        issued.append(rel - 1 + NST)
                assert sorted(issued) == list(range(nbands))
                for rel in range(nbands):
                    ez = ezs + rel
                    if not (has_halo and rel == 0):
                        owner[ez] += 1
            assert (owner == 1).all()


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
def test_band_tensor_copies(N):
    """One tensor copy per staged field and band: box of bw(N) columns from X0 and N+1 rows
    from ez*N in the field's slot of the solve's workspace map, issued by lane 1 of warp f."""
    NP, NW, BW = N + 1, THREADS // 32, bw(N)
    assert BW <= 256 and NP <= 256 and (BW * 4) % 16 == 0      # box limits, 16-byte inner extent
    FB = field_floats(N)
    assert FB >= NP * BW and (FB * 4) % 128 == 0               # field blocks 128-byte aligned
    for adj in (False, True):
        nload = 4 if adj else 3
        assert nload <= NW                                     # one issuing warp per field
        issuers = [tid for tid in range(THREADS) if tid % 32 == 1 and tid // 32 < nload]
        assert [t // 32 for t in issuers] == list(range(nload))
        assert (nload * FB) % 32 == 0                          # ring slots stay aligned
    for nelx, nelz in ((100, 50), (400, 200), (7, 3), (40, 20)):
        nxg, nzg = nelx * N + 1, nelz * N + 1
        pitch = pitch_of(nxg)
        assert (pitch * 4) % 16 == 0                           # row stride of the map
        fstride = -(-(pitch * nzg) // 64) * 64                 # floats per field (256-byte multiple)
        assert (fstride * 4) % 16 == 0                         # slot stride of the map
        ns, EW = strips_of(nelx, N)
        for strip in range(ns):
            X0 = ((strip * EW) * N - N) & ~3
            assert X0 % 4 == 0 and -BW < X0 < pitch            # x * 4 bytes on a 16-byte boundary
        for ez in range(nelz):
            assert 0 <= ez * N and ez * N + N <= nzg - 1       # the band's rows are in the map
        # workspace slots: c2 | W W | V | ckpt (2 nseg) | ring (k+1) | L L | Mu, then the
        # float64 gradient; every staged field is slot (ptr - ws) / fstride < slots
        k, nt = 7, 50
        nseg = -(-nt // k)
        slots = 1 + 2 + 1 + 2 * nseg + (k + 1) + 2 + 1
        assert slots * fstride < 2 ** 40 and slots < 2 ** 32
