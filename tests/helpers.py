"""Shared helpers of the test suite."""
import numpy as np

TOL = {"c128": 1e-12, "c64": 1e-6}   # relative L2 bar of the transforms and stencils


def relerr(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def rand_field(dim: int, n: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    shape = (n,) * dim
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def to_dev(x: np.ndarray, dtype: str):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(x.astype(np.complex128 if dtype == "c128" else np.complex64)))
    return t.cuda()


def to_host(t) -> np.ndarray:
    return t.detach().cpu().numpy().astype(np.complex128)
