"""Device buffers and streams (torch is used for allocation only)."""

from __future__ import annotations

import numpy as np
import torch


def require_cuda(device=None) -> torch.device:
    """The CUDA device to run on; raises when there is none (no CPU fallback)."""
    if not torch.cuda.is_available():
        raise RuntimeError(
            "critmc_b200 samplers run on a CUDA GPU and none is available "
            "(there is no CPU fallback; the CPU oracle is test infrastructure)"
        )
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    if dev.type != "cuda":
        raise ValueError(f"device must be a CUDA device, got {dev}")
    return dev


def to_dev(a: np.ndarray, device: torch.device) -> torch.Tensor:
    """Copy a host array to the device, reinterpreting unsigned 32-bit as int32."""
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(a).to(device)


def to_host(t: torch.Tensor, dtype=None) -> np.ndarray:
    a = t.detach().cpu().numpy()
    if dtype is not None and a.dtype != dtype:
        a = a.view(dtype)
    return a


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if not t.is_contiguous():
        raise ValueError("device buffers passed to the C ABI must be contiguous")
    return t.data_ptr()


def stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def empty_bytes(n: int, device: torch.device) -> torch.Tensor:
    return torch.empty(max(16, int(n)), dtype=torch.uint8, device=device)
