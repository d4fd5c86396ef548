"""CPU check of the per-solve time program of the tick kernel (decode, fwd_loc,
replay_loc in sem_kernels.cu): a symbolic run records which state b_t every buffer
slot holds and asserts that every tick reads the right states and that checkpoint and
ring slots stay in range."""
import pytest

A_NONE, A_FWD, A_FINAL, A_REPLAY, A_ADJ, A_SCALE = range(6)


def cdiv(a, b):  # C integer division/modulo for non-negative a
    assert a >= 0
    return a // b


def decode(nt, k, nseg, adj, shift, sig):
    if sig < 0:
        return A_NONE, 0, -1
    if sig < nt:
        return A_FWD, sig, -1
    sig -= nt
    if shift:
        if sig == 0:
            return A_FINAL, nt, -1
        sig -= 1
    if not adj:
        return A_NONE, 0, -1
    if sig == 0:
        return A_SCALE, 0, -1
    sig -= 1
    jl = nseg - 1
    len_last = nt - jl * k
    if sig < len_last:
        return A_ADJ, nt - 1 - sig, jl
    sig -= len_last
    if sig >= 2 * k * jl:
        return A_NONE, 0, -1
    j = jl - 1 - cdiv(sig, 2 * k)
    w = sig % (2 * k)
    if w < k:
        return A_REPLAY, j * k + w, j
    return A_ADJ, (j + 1) * k - 1 - (w - k), j


def fwd_b(nt, k, nseg, adj, t):
    if not adj:
        return ("W", t & 1)
    jl = nseg - 1
    if t >= jl * k:
        return ("ring", t - jl * k)
    if t % k == 0:
        return ("ckpt", 2 * (t // k))
    return ("W", t & 1)


def fwd_v(nt, k, nseg, adj, t):
    if not adj:
        return ("V", 0)
    jl = nseg - 1
    if t < jl * k and t % k == 0:
        return ("ckpt", 2 * (t // k) + 1)
    return ("V", 0)


def rep_b(k, j, t):
    return ("ckpt", 2 * j) if t == j * k else ("ring", t - j * k)


def rep_v(k, j, t):
    return ("ckpt", 2 * j + 1) if t == j * k else ("V", 0)


def simulate(nt, k, adj, shift):
    """Symbolic run: mem maps a slot to ('b', t) or ('v', t)."""
    nseg = -(-nt // k) if adj else 1
    mem = {}
    if adj:
        if nseg == 1:
            mem[("ring", 0)] = ("b", 0)
            mem[("V", 0)] = ("v", 0)
        else:
            mem[("ckpt", 0)], mem[("ckpt", 1)] = ("b", 0), ("v", 0)
    else:
        mem[("W", 0)], mem[("V", 0)] = ("b", 0), ("v", 0)
    lam = {nt & 1: nt}
    mu = nt
    prog = nt + (1 if shift else 0) + (1 + nt + k * (nseg - 1) if adj else 0)
    adj_seen = []

    def check(loc):
        kind, slot = loc
        if kind == "ring":
            assert 0 <= slot <= k
        if kind == "ckpt":
            assert 0 <= slot < 2 * nseg
        if kind == "W":
            assert slot in (0, 1)
        return loc

    for sig in range(prog + 3):
        act, t, seg = decode(nt, k, nseg, adj, shift, sig)
        if sig >= prog:
            assert act == A_NONE
            continue
        if act == A_FWD:
            rb, rv = check(fwd_b(nt, k, nseg, adj, t)), check(fwd_v(nt, k, nseg, adj, t))
            wb, wv = check(fwd_b(nt, k, nseg, adj, t + 1)), check(fwd_v(nt, k, nseg, adj, t + 1))
            assert mem[rb] == ("b", t) and mem[rv] == ("v", t)
            assert wb != rb  # b is read with a halo by other tiles: never in place
            mem[wb], mem[wv] = ("b", t + 1), ("v", t + 1)
        elif act == A_FINAL:
            assert mem[fwd_b(nt, k, nseg, adj, nt)] == ("b", nt)
        elif act == A_SCALE:
            assert not adj_seen
        elif act == A_REPLAY:
            rb, rv = check(rep_b(k, seg, t)), check(rep_v(k, seg, t))
            wb, wv = check(rep_b(k, seg, t + 1)), check(rep_v(k, seg, t + 1))
            assert mem[rb] == ("b", t) and mem[rv] == ("v", t)
            assert wb != rb
            mem[wb], mem[wv] = ("b", t + 1), ("v", t + 1)
        elif act == A_ADJ:
            slot = t + 1 - seg * k
            assert 1 <= slot <= k
            assert mem[("ring", slot)] == ("b", t + 1)
            assert lam[(t + 1) & 1] == t + 1 and mu == t + 1
            lam[t & 1] = t
            mu = t
            adj_seen.append(t)
        else:
            raise AssertionError(f"tick {sig} of {prog} decoded to nothing")
    if adj:
        assert adj_seen == list(range(nt - 1, -1, -1))


@pytest.mark.parametrize("nt", [1, 2, 3, 7, 10, 64, 101])
@pytest.mark.parametrize("k", [2, 3, 4, 5, 16, 1000])
def test_adjoint_program(nt, k):
    simulate(nt, min(k, nt) if nt >= 2 else 2, True, True)


@pytest.mark.parametrize("nt", [1, 2, 5, 33])
@pytest.mark.parametrize("shift", [False, True])
def test_forward_program(nt, shift):
    simulate(nt, 2, False, shift)
