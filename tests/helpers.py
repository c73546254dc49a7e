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


def ramp_spectrum(dim: int, n: int) -> np.ndarray:
    """Closed-form DFT of the reference's init_host fixture, x = global linear index
    (row-major, last axis fastest), in natural order: per axis, the DFT of a constant
    (S = n at k = 0) and of a ramp 0..n-1 (T = n / (w^k - 1), n(n-1)/2 at k = 0)."""
    k = np.arange(n)
    w = np.exp(-2j * np.pi * k / n)
    S = np.where(k == 0, n, 0).astype(np.complex128)
    with np.errstate(divide="ignore", invalid="ignore"):
        T = np.where(k == 0, n * (n - 1) / 2, n / (w - 1))
    if dim == 2:
        return n * np.multiply.outer(T, S) + np.multiply.outer(S, T)
    return (n * n * np.einsum("i,j,k->ijk", T, S, S) + n * np.einsum("i,j,k->ijk", S, T, S)
            + np.einsum("i,j,k->ijk", S, S, T))
