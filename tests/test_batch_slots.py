"""CPU checks of the batch tiles' shared-memory slot permutations (zm_tile.cuh SwzX, chosen
per column length in zm_batch.cu's dispatch).

The batch kernel relies on three properties of each permutation: it is a permutation of
every aligned run of 16 slots (so a tile of 4096 elements stays in place); it is linear
over XOR, so a Stockham stage computes one slot per sub-transform and XORs in the
per-point offsets (f(a | c) = f(a) ^ f(c) for disjoint bit fields); and it leaves bits 0-1
to the row sweeps' k.  The last test restates the tile's shared accesses (the row sweeps,
every column stage's reads and writes, both frequency-side sweeps at P = 2) with the
kernel's thread mapping and checks that the 16 lanes of each half-warp hit 16 distinct
bank pairs (8-byte elements), the basis of the comment in zm_tile.cuh.
"""
import re
from pathlib import Path

import numpy as np
import pytest

SRC = Path(__file__).resolve().parents[1] / "stencilfft_b200" / "csrc" / "zm_batch.cu"
NT, EPT, TILE = 256, 16, 4096


def dispatch():
    txt = SRC.read_text()
    found = re.findall(r"case (\d+): ZM_BT\(\1, SwzX<(\d+), (\d+), (\d+), (\d+), (\d+)>\)", txt)
    return {int(m[0]): tuple(int(x) for x in m[1:]) for m in found}


def swz(params):
    a0, a1, b, c0, c1 = params

    def fld(i, s, t):
        return ((i >> s) & 3) << t if s else 0

    return lambda i: i ^ fld(i, a0, 0) ^ fld(i, a1, 0) ^ fld(i, b, 1) ^ fld(i, c0, 2) ^ fld(i, c1, 2)


def test_dispatch_lists_every_column_length():
    assert sorted(dispatch()) == list(range(4, 11))


@pytest.mark.parametrize("lm", range(4, 11))
def test_slot_permutation_properties(lm):
    f = swz(dispatch()[lm])
    i = np.arange(TILE, dtype=np.int64)
    fi = f(i)
    assert np.array_equal(np.sort(fi), i)                       # a permutation of the tile
    assert np.array_equal(fi >> 4, i >> 4)                      # inside each aligned run of 16
    assert np.array_equal(f(np.arange(4)), np.arange(4))        # f(k) = k for the row sweeps' k
    rng = np.random.default_rng(lm)
    a, c = rng.integers(0, TILE, 20000), rng.integers(0, TILE, 20000)
    assert np.array_equal(f(a ^ c), f(a) ^ f(c))                # linear over XOR


def sched(lm):
    rem = lm % 4
    return ([1 << rem] if rem else []) + [16] * (lm // 4)


def stage_accesses(lm):
    """(reads, writes) slot arrays [access, lane] of every column stage, thread mapping of
    stockham_stage_ct (COLM, VEC = 4, NT = 256), and the XOR-decomposed forms the kernel
    computes (base slot ^ per-point offset)."""
    m = 1 << lm
    logn = lm + 2
    ns = 1
    out = []
    tid = np.arange(NT, dtype=np.int64)
    for r_ in sched(lm):
        nr = m // r_
        lognr = nr.bit_length() - 1
        for u in range(EPT // r_):
            sig = tid + u * NT
            k2, rest = sig & 3, sig >> 2
            j, t = rest & (nr - 1), rest >> lognr
            bb = (t << logn) + k2
            k = j & (ns - 1)
            idxd = (j - k) * r_ + k
            for r in range(r_):
                out.append(("read", bb + (j + r * nr) * 4, bb + j * 4, r * nr * 4))
                out.append(("write", bb + (idxd + r * ns) * 4, bb + idxd * 4, r * ns * 4))
        ns *= r_
    return out


@pytest.mark.parametrize("lm", range(4, 11))
def test_stage_slots_decompose_over_xor(lm):
    f = swz(dispatch()[lm])
    for _, full, base, off in stage_accesses(lm):
        assert np.array_equal(f(full), f(base) ^ f(np.int64(off)))


def wavefronts(slots):
    """8-byte accesses of one warp: per half-warp, the most distinct slots on one bank pair."""
    tot = 0
    for h in (slots[:16], slots[16:]):
        pairs = {}
        for x in set(int(v) for v in h):
            pairs[x % 16] = pairs.get(x % 16, 0) + 1
        tot += max(pairs.values())
    return tot


def freq_accesses(lm, p, xpass):
    n = 4 << lm
    L = n // p
    logl, logn = L.bit_length() - 1, n.bit_length() - 1
    tl = TILE // n
    logt = tl.bit_length() - 1
    lvp = 2 - (p.bit_length() - 1)
    tid = np.arange(NT, dtype=np.int64)
    for i in range(EPT):
        e = tid + i * NT
        t = (e & (tl - 1)) if xpass else (e >> logn)
        cp = (e >> logt) if xpass else (e & (n - 1))
        ch, pos = cp >> logl, cp & (L - 1)
        yield (t << logn) + ((pos >> lvp) << 2) + (ch << lvp) + (pos & ((1 << lvp) - 1))


@pytest.mark.parametrize("lm", range(4, 11))
def test_tile_accesses_conflict_free(lm):
    f = swz(dispatch()[lm])
    acc = [a for _, a, _, _ in stage_accesses(lm)]
    tid = np.arange(NT, dtype=np.int64)
    acc += [(tid + q * NT) * 4 + k for q in range(EPT // 4) for k in range(4)]   # row sweeps
    acc += list(freq_accesses(lm, 2, True)) + list(freq_accesses(lm, 2, False))
    for a in acc:
        fa = f(a)
        for w in range(NT // 32):
            assert wavefronts(fa[32 * w:32 * w + 32]) == 2
