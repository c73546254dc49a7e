"""zm_fft_inverse_static: the inverse transform for callers that cannot allocate device
memory (a plugin whose host owns every device allocation, a loop under a fixed memory
budget).  Its one-field intermediate lives in a scratch array built into the library
instead of a caller workspace.

Checked through the C ABI against zm_fft_inverse with a caller workspace, on two calls
in a row (the scratch keeps the first call's contents when the second starts), with
the input left intact.  Kept in a file collected last so a failure here comes after
every other test has run; it also passes alone in a fresh process, where its first call
performs the per-device set-up.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from helpers import rand_field, relerr, to_dev, to_host
from stencilfft_b200 import abi

pytestmark = pytest.mark.gpu

TOL = {"c128": 1e-12, "c64": 1e-6}


@pytest.mark.parametrize("dim,n,b,p,dt", [(2, 256, 16, 4, "c128"), (2, 1024, 32, 2, "c128"),
                                          (3, 32, 2, 4, "c64"), (2, 512, 16, 2, "c64")])
def test_static_inverse_matches_workspace_inverse(dim, n, b, p, dt):
    import torch
    from stencilfft_b200 import Plan
    L = abi.lib()
    pl = Plan(dim, n, b, p, dtype=dt)
    scale = complex(1.0 / n ** dim, 0.25 / n ** dim)
    for call in range(2):                      # two calls in a row share the scratch
        x = rand_field(dim, n, seed=100 + call)
        spec = O.forward_fft(O.natural_to_real_layout(x, b, p), dim, n, b, p)
        d_in = to_dev(spec, dt)
        keep = d_in.clone()
        ref_out, work = torch.empty_like(d_in), torch.empty_like(d_in)
        pl.inverse_fft(d_in, ref_out, scale=scale, work=work)        # existing entry point
        out = torch.empty_like(d_in)
        rc = L.zm_fft_inverse_static(pl.handle, ctypes.c_void_p(d_in.data_ptr()),
                                     ctypes.c_void_p(out.data_ptr()), scale.real, scale.imag,
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == abi.ZM_OK, L.zm_last_error_string()
        torch.cuda.synchronize()
        assert relerr(to_host(out), to_host(ref_out)) < TOL[dt]
        assert torch.equal(d_in, keep)          # input not used as scratch
        expect = O.inverse_fft(spec, dim, n, b, p, scale=scale)
        assert relerr(to_host(out), expect) < TOL[dt]


def test_static_inverse_rejects_fields_beyond_the_scratch():
    import torch
    from stencilfft_b200 import Plan
    L = abi.lib()
    pl = Plan(2, 2048, 32, 2, dtype="c128")      # 64 MiB > 16 MiB
    a = torch.empty(8, dtype=torch.complex128, device="cuda")
    rc = L.zm_fft_inverse_static(pl.handle, ctypes.c_void_p(a.data_ptr()),
                                 ctypes.c_void_p(a.data_ptr() + 64), 1.0, 0.0, None)
    assert rc == abi.ZM_ERR_WORKSPACE
    assert b"static scratch" in L.zm_last_error_string()
