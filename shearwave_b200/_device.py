"""Device plumbing shared by the host-side API: torch owns every buffer.

Arrays arrive as numpy arrays or torch tensors.  They are moved to the current
CUDA device as contiguous tensors of the requested dtype; results go back to
numpy unless the caller asked for device tensors.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native

_NP = {torch.float32: np.float32, torch.float64: np.float64}
_TORCH = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64}


def require_cuda() -> torch.device:
    """The current CUDA device; raise if there is none (there is no CPU path)."""
    if not torch.cuda.is_available():
        raise RuntimeError(
            "shearwave_b200 runs on a CUDA device (sm_100a) only; none is available"
        )
    _native.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    _native.call("sw_set_device", dev.index)
    return dev


def stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


def dtype_code(t: torch.dtype) -> int:
    if t == torch.float32:
        return _native.SW_F32
    if t == torch.float64:
        return _native.SW_F64
    raise TypeError(f"unsupported dtype {t}")


def is_tensor(a) -> bool:
    return isinstance(a, torch.Tensor)


def to_device(a, dtype: torch.dtype, dev: torch.device) -> torch.Tensor:
    """Contiguous device tensor of ``dtype`` holding ``a`` (copied if needed)."""
    if isinstance(a, torch.Tensor):
        # page-locked host tensors copy asynchronously (stream-ordered before
        # the kernels that read them; the caller keeps the source alive)
        pinned = a.device.type == "cpu" and a.is_pinned()
        return a.to(device=dev, dtype=dtype, non_blocking=pinned).contiguous()
    arr = np.ascontiguousarray(np.asarray(a), dtype=_NP[dtype])
    return torch.from_numpy(arr).to(dev)


def ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def to_host(t: torch.Tensor, device_out: bool):
    return t if device_out else t.cpu().numpy()


def np_dtype(t: torch.dtype):
    return _NP[t]


def torch_dtype(d) -> torch.dtype:
    return _TORCH[np.dtype(d)]
