"""Parity pins that travel with the repository: the oracle and the library's own index
maps against fixtures recorded from the reference's host code (zmodel/utils.h index
maps, zmodel/utils.cu ramp fixture; tests/golden/make_golden.py), so they also run where
the reference sources are absent."""
import ctypes
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import oracle as O

GOLD = Path(__file__).resolve().parent / "golden"
MAPS = np.load(GOLD / "reference_index_maps.npz")
RAMP = json.loads((GOLD / "reference_ramp.json").read_text())


def _cfgs(prefix):
    out = []
    for k in MAPS.files:
        if k.startswith(prefix):
            dim = int(k.split("_")[1][0])
            n, b, p = (int(x[1:]) for x in k.split("_")[2:5])
            out.append((dim, n, b, p))
    return sorted(set(out))


@pytest.mark.parametrize("dim,n,b,p", _cfgs("real_"))
def test_oracle_maps_match_reference_fixture(dim, n, b, p):
    tag = f"{dim}d_N{n}_B{b}_P{p}"
    assert np.array_equal(O.real_layout_map(dim, n, b, p), MAPS["real_" + tag].astype(np.int64))
    assert np.array_equal(O.reciprocal_layout_map(dim, n, b, p), MAPS["reciprocal_" + tag].astype(np.int64))


@pytest.mark.parametrize("dim,n,b,p", _cfgs("real_"))
def test_library_host_maps_match_reference_fixture(dim, n, b, p):
    """The C ABI's zm_real_to_global / zm_reciprocal_to_global on a host-only plan."""
    from stencilfft_b200 import Plan
    pl = Plan(dim, n, b, p, dtype="c128", host_only=True)
    tag = f"{dim}d_N{n}_B{b}_P{p}"
    real, recip = MAPS["real_" + tag], MAPS["reciprocal_" + tag]
    L = n // p
    rng = np.random.default_rng(5)
    for e in rng.integers(0, n ** dim, 300):
        e = int(e)
        r, rem = divmod(e, L ** dim)
        if dim == 2:
            rid, cid = divmod(r, p)
            lr, lc = divmod(rem, L)
            gr, gc = pl.real_to_global(rid, cid, lr, lc)
            assert gr * n + gc == real[e]
            kr, kc = pl.reciprocal_to_global(rid, cid, lr, lc)
            assert kr * n + kc == recip[e]
        else:
            did, rc = divmod(r, p * p)
            rid, cid = divmod(rc, p)
            ld, rem2 = divmod(rem, L * L)
            lr, lc = divmod(rem2, L)
            gd, gr, gc = pl.real_to_global(rid, cid, lr, lc, did, ld)
            assert (gd * n + gr) * n + gc == real[e]
            kd, kr, kc = pl.reciprocal_to_global(rid, cid, lr, lc, did, ld)
            assert (kd * n + kr) * n + kc == recip[e]


@pytest.mark.parametrize("n,b,p", [(16384, 64, 4), (4096, 32, 4), (2048, 32, 2)])
def test_sampled_large_maps_match_reference_fixture(n, b, p):
    from stencilfft_b200 import Plan
    pl = Plan(2, n, b, p, dtype="c64", host_only=True)
    tag = f"N{n}_B{b}_P{p}"
    q = MAPS["sample_in_" + tag]
    for (a, c), rec, rea in zip(q, MAPS["sample_g2recip_" + tag], MAPS["sample_g2real_" + tag]):
        a, c = int(a), int(c)
        assert O.index_map("global_to_reciprocal", n, b, p, a, c) == tuple(int(v) for v in rec)
        assert O.index_map("global_to_real", n, b, p, a, c) == tuple(int(v) for v in rea)
        assert pl.global_to_reciprocal(a, c) == tuple(int(v) for v in rec)
        assert pl.global_to_real(a, c) == tuple(int(v) for v in rea)


@pytest.mark.parametrize("key", sorted(RAMP))
def test_oracle_ramp_matches_reference_fixture(key):
    dim = int(key[0])
    n, b, p = (int(x[1:]) for x in key.split("_")[1:4])
    ours = O.init_ramp(dim, n, b, p)
    assert hashlib.sha256(ours.tobytes()).hexdigest() == RAMP[key]["sha256"]
    assert np.array_equal(ours[:8], np.array([complex(*v) for v in RAMP[key]["first"]]))
