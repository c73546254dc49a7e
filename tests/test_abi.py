"""CPU tests of the C ABI boundary (no GPU needed): the library loads, exports every
symbol the public header declares, validates layouts like the reference, and its
host-side index maps agree with the oracle."""
import ctypes

import numpy as np
import pytest

import oracle as O
from stencilfft_b200 import abi


def test_library_exports_every_declared_symbol():
    L = abi.lib()
    declared = abi.declared_symbols()
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    # and the Python bindings cover every declared entry point
    assert set(declared) <= set(abi.SIGNATURES), set(declared) - set(abi.SIGNATURES)


def _create(dim, n, b, p, dtype=0, flags=abi.ZM_FLAG_HOST_ONLY):
    h = ctypes.c_void_p()
    rc = abi.lib().zm_plan_create(ctypes.byref(h), dim, n, b, p, dtype, flags)
    return rc, h


@pytest.mark.parametrize("dim,n,b,p,status", [
    (2, 64, 4, 2, abi.ZM_OK),
    (2, 64, 32, 2, abi.ZM_ERR_CONSTRAINT),   # VEC = 1 not divisible by P (B > N/P^2, run.sh:13)
    (2, 64, 3, 2, abi.ZM_ERR_CONSTRAINT),    # not a power of two
    (2, 96, 4, 2, abi.ZM_ERR_CONSTRAINT),
    (2, 64, 128, 2, abi.ZM_ERR_CONSTRAINT),  # B does not divide L
    (4, 64, 4, 2, abi.ZM_ERR_INVALID_ARG),
    (3, 16, 2, 2, abi.ZM_OK),
    (3, 16, 4, 4, abi.ZM_ERR_CONSTRAINT),
])
def test_plan_validation(dim, n, b, p, status):
    rc, h = _create(dim, n, b, p)
    assert rc == status, abi.lib().zm_last_error_string()
    if rc == abi.ZM_OK:
        info = abi.zm_plan_info()
        assert abi.lib().zm_plan_get_info(h, ctypes.byref(info)) == 0
        d = O.derived(dim, n, b, p)
        assert (info.local_dim, info.vec, info.vec_split, info.m) == (d["L"], d["VEC"], d["VP"], d["M"])
        assert info.total_elems == n ** dim
        assert abi.lib().zm_plan_destroy(h) == 0
    else:
        assert abi.lib().zm_last_error_string()


def test_unknown_dtype_and_flags_rejected():
    h = ctypes.c_void_p()
    assert abi.lib().zm_plan_create(ctypes.byref(h), 2, 64, 4, 2, 7, 0) == abi.ZM_ERR_INVALID_ARG
    assert abi.lib().zm_plan_create(ctypes.byref(h), 2, 64, 4, 2, 0, 0x80) == abi.ZM_ERR_INVALID_ARG
    assert abi.lib().zm_plan_create(None, 2, 64, 4, 2, 0, 0) == abi.ZM_ERR_INVALID_ARG


def test_host_only_plan_refuses_device_work():
    rc, h = _create(2, 64, 4, 2)
    assert rc == 0
    buf = ctypes.c_void_p(16)
    assert abi.lib().zm_fft_forward(h, buf, ctypes.c_void_p(1 << 20), None, None) == abi.ZM_ERR_UNSUPPORTED
    assert abi.lib().zm_laplace(h, buf, ctypes.c_void_p(1 << 20), 1.0, None) == abi.ZM_ERR_UNSUPPORTED
    abi.lib().zm_plan_destroy(h)


def test_null_plan_is_an_error_not_a_crash():
    assert abi.lib().zm_fft_forward(None, None, None, None, None) == abi.ZM_ERR_INVALID_ARG
    assert abi.lib().zm_plan_destroy(None) == abi.ZM_ERR_INVALID_ARG
    assert abi.lib().zm_status_string(abi.ZM_ERR_CONSTRAINT) == b"layout constraint violated"


@pytest.mark.parametrize("dim,n,b,p", [(2, 64, 4, 2), (2, 128, 8, 4), (2, 64, 1, 4), (3, 16, 2, 2),
                                       (3, 32, 2, 4)])
def test_index_maps_match_oracle(dim, n, b, p):
    rc, h = _create(dim, n, b, p)
    assert rc == 0
    L = abi.lib()
    o = [ctypes.c_int64() for _ in range(6)]
    ref_real = O.real_layout_map(dim, n, b, p)
    ref_recip = O.reciprocal_layout_map(dim, n, b, p)
    d = O.derived(dim, n, b, p)
    Ld = d["L"]
    rng = np.random.default_rng(0)
    for e in rng.integers(0, n ** dim, 300):
        e = int(e)
        r, loc = divmod(e, d["rank_elems"])
        if dim == 2:
            did, rid, cid = 0, r // p, r % p
            ld, lr, lc = 0, loc // Ld, loc % Ld
        else:
            did, rid, cid = r // (p * p), (r % (p * p)) // p, r % p
            ld, lr, lc = loc // (Ld * Ld), (loc // Ld) % Ld, loc % Ld
        assert L.zm_real_to_global(h, rid, cid, did, ld, lr, lc, *map(ctypes.byref, o[:3])) == 0
        gd, gr, gc = (v.value for v in o[:3])
        assert (gd * n + gr) * n + gc == ref_real[e] if dim == 3 else gr * n + gc == ref_real[e]
        assert L.zm_global_to_real(h, gd, gr, gc, *map(ctypes.byref, o)) == 0
        assert tuple(v.value for v in o) == (rid, cid, did, ld, lr, lc)
        assert L.zm_reciprocal_to_global(h, rid, cid, did, ld, lr, lc, *map(ctypes.byref, o[:3])) == 0
        kd, kr, kc = (v.value for v in o[:3])
        assert ((kd * n + kr) * n + kc if dim == 3 else kr * n + kc) == ref_recip[e]
        assert L.zm_global_to_reciprocal(h, kd, kr, kc, *map(ctypes.byref, o)) == 0
        assert tuple(v.value for v in o) == (rid, cid, did, ld, lr, lc)
    assert L.zm_real_to_global(h, p, 0, 0, 0, 0, 0, *map(ctypes.byref, o[:3])) == abi.ZM_ERR_INVALID_ARG
    L.zm_plan_destroy(h)
