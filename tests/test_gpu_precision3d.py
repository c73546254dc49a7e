"""3D precision form: N = 512 (512^3), P = 4 per axis, B = 32, field ~ N(0,1) from the
counter generator with seed 2.  The complex64 form (FP64-generated twiddles applied as
compensated hi/lo FP32 products) and the plain complex128 form run forward / inverse
fft3d and the 7-point laplace3d on the same GPU; their errors are measured against an
FP64 oracle (scipy's pocketfft on the natural-layout field, all host cores) and, for
the Laplacian, against the complex128 result.  Relative L2 and max-abs (relative to the
largest magnitude) are printed; the bars are the transform tolerances, 1e-6 for
complex64 and 1e-12 for complex128."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, B, P = 512, 32, 4


def _errs(a, ref):
    import torch
    d = (a.to(torch.complex128) - ref)
    rel = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(ref))
    mx = float(d.abs().max() / ref.abs().max())
    return rel, mx


def test_3d_precision_forms():
    import scipy.fft
    import torch
    from stencilfft_b200 import Plan, abi
    p64, p128 = Plan(3, N, B, P, dtype="c64"), Plan(3, N, B, P, dtype="c128")
    u = p128.empty()
    p128.fill(u, abi.ZM_FIELD_GAUSSIAN, 2)
    u64 = u.to(torch.complex64)

    # FP64 oracle spectrum in natural order, moved to the device for the comparisons
    nat = p128.empty()
    p128.real_to_natural(u, nat)
    X = scipy.fft.fftn(nat.cpu().numpy().reshape(N, N, N), workers=os.cpu_count())
    X = torch.from_numpy(np.ascontiguousarray(X).reshape(-1)).cuda()
    del nat

    res = {}
    for name, pl, src in (("c128", p128, u), ("c64", p64, u64)):
        spec, work, back, lap = pl.empty(), pl.empty(), pl.empty(), pl.empty()
        pl.forward_fft(src, spec, work=work)
        sn = pl.empty()
        pl.reciprocal_to_natural(spec, sn)
        res[name + "_fwd"] = _errs(sn, X)
        del sn
        pl.inverse_fft(spec, back, scale=1.0 / N ** 3, work=work)
        res[name + "_roundtrip"] = _errs(back, src.to(torch.complex128))
        pl.laplace(src, lap)
        res[name + "_lap"] = lap.to(torch.complex128) if name == "c128" else lap
        del spec, work, back
    res["c64_lap"] = _errs(res["c64_lap"], res.pop("c128_lap"))
    print("\n3D N=512 P=4 B=32 precision (rel-L2, max-abs/max):",
          {k: (f"{v[0]:.3e}", f"{v[1]:.3e}") for k, v in res.items()})
    assert res["c128_fwd"][0] < 1e-12
    assert res["c128_roundtrip"][0] < 1e-12
    assert res["c64_fwd"][0] < 1e-6
    assert res["c64_roundtrip"][0] < 1e-6
    assert res["c64_lap"][0] < 1e-6
