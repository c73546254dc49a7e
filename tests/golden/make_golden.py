"""Writes the golden fixtures of tests/test_golden.py from the reference's OWN host code.

The reference's zmodel/utils.h index maps and zmodel/utils.cu ramp fixture (init_host /
init_host_3d) are compiled unmodified per (N_DIM, B_DIM, P_DIM) by `make -C oracle
ref-host` (into oracle/_ref/, where the reference sources are available) and called
through oracle/ref_host_shim.cpp.  This script records their outputs so that the pins
travel with the repository:

  reference_index_maps.npz   whole-grid real_to_global / reciprocal_to_global tables
                             (global linear index held by each interleaved element) for
                             small 2D / 3D grids, and sampled global_to_real /
                             global_to_reciprocal answers for the large benchmark grids
  reference_ramp.json        SHA-256 of the whole-grid ramp fixture per config, plus
                             its first and last values

    python tests/golden/make_golden.py        (needs oracle/_ref from the reference)
"""
import ctypes
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
import oracle as O  # noqa: E402

MAPS_2D = [(16, 2, 2), (32, 4, 2), (64, 4, 2), (64, 2, 4), (64, 16, 2), (128, 8, 4)]
MAPS_3D = [(16, 2, 2), (32, 2, 4)]
SAMPLED = [(16384, 64, 4), (4096, 32, 4), (2048, 32, 2)]
RAMP = [(2, 64, 4, 2), (2, 64, 2, 4), (2, 256, 16, 4), (2, 1024, 32, 2), (3, 16, 2, 2), (3, 32, 2, 4)]


def main():
    arrays = {}
    for dim, cfgs in ((2, MAPS_2D), (3, MAPS_3D)):
        for n, b, p in cfgs:
            ref = O.ref_host_lib(n, b, p)
            if ref is None:
                sys.exit(f"reference host code for N={n} B={b} P={p} is not built (make -C oracle ref-host)")
            for kind in ("real", "reciprocal"):
                out = np.empty(n ** dim, dtype=np.int64)
                getattr(ref, f"zr_{kind}_layout_map")(dim, out.ctypes.data_as(ctypes.c_void_p))
                arrays[f"{kind}_{dim}d_N{n}_B{b}_P{p}"] = out.astype(np.int32)
    rng = np.random.default_rng(2024)
    ci = ctypes.c_int
    for n, b, p in SAMPLED:
        ref = O.ref_host_lib(n, b, p)
        if ref is None:
            sys.exit(f"reference host code for N={n} B={b} P={p} is not built")
        q = rng.integers(0, n, size=(256, 2))
        recip, real = [], []
        for a, c in q:
            out = [ci() for _ in range(4)]
            ref.zr_global_to_reciprocal(int(a), int(c), *[ctypes.byref(o) for o in out])
            recip.append([o.value for o in out])
            ref.zr_global_to_real(int(a), int(c), *[ctypes.byref(o) for o in out])
            real.append([o.value for o in out])
        arrays[f"sample_in_N{n}_B{b}_P{p}"] = q.astype(np.int32)
        arrays[f"sample_g2recip_N{n}_B{b}_P{p}"] = np.array(recip, dtype=np.int32)
        arrays[f"sample_g2real_N{n}_B{b}_P{p}"] = np.array(real, dtype=np.int32)
    np.savez_compressed(HERE / "reference_index_maps.npz", **arrays)

    ramp = {}
    for dim, n, b, p in RAMP:
        ref = O.ref_host_lib(n, b, p)
        d = O.derived(dim, n, b, p)
        per = d["rank_elems"]
        full = np.empty(n ** dim, dtype=np.complex128)
        for r in range(d["ranks"]):
            got = np.empty(per, dtype=np.complex128)
            ptr = got.ctypes.data_as(ctypes.c_void_p)
            if dim == 2:
                ref.zr_init_host(r // p, r % p, ptr)
            else:
                ref.zr_init_host_3d((r % (p * p)) // p, r % p, r // (p * p), ptr)
            full[r * per:(r + 1) * per] = got
        ramp[f"{dim}d_N{n}_B{b}_P{p}"] = {
            "sha256": hashlib.sha256(full.tobytes()).hexdigest(),
            "first": [[v.real, v.imag] for v in full[:8]],
            "last": [[v.real, v.imag] for v in full[-8:]],
        }
    (HERE / "reference_ramp.json").write_text(json.dumps(ramp, indent=1) + "\n")
    print("wrote", HERE / "reference_index_maps.npz", HERE / "reference_ramp.json")


if __name__ == "__main__":
    main()
