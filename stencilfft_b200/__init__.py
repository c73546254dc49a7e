"""stencilfft_b200 -- B200-native interleaved block-cyclic FFT and stencils.

The product is ``lib/libzmodel_b200.so`` (CUDA, sm_100a) behind the C ABI declared in
``include/zmodel_b200.h``.  This package is the Python host side of that ABI:
``ctypes`` bindings (``abi``) and a ``Plan`` object mirroring the zmodel entry
points (``forward_fft``, ``inverse_fft``, ``laplace``, ``dx``, ``dy`` and the 3D
forms) over whole-grid device buffers, and a ``Batch`` of uneven-N 2D fields run by
one persistent launch per call.  PyTorch tensors are accepted for device
memory and streams only; no arithmetic is done in Python and there is no CPU
fallback -- calls fail loudly when the CUDA library is missing.
"""
from .abi import (ZM_C128, ZM_C64, ZM_FLAG_PERMUTE_ONLY, ZmError, lib, library_path,  # noqa: F401
                  launch_count)
from .batch import Batch  # noqa: F401
from .plan import Plan, autotune_b  # noqa: F401

__all__ = ["Plan", "Batch", "autotune_b", "ZmError", "ZM_C128", "ZM_C64", "ZM_FLAG_PERMUTE_ONLY", "lib", "library_path",
           "launch_count"]
