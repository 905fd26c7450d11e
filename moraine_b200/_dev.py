"""Device plumbing of the drop-in functions.

The reference functions return arrays of the same kind as their input (numpy in, numpy
out; cupy in, cupy out). Here a torch CUDA tensor in gives torch CUDA tensors out, and a
numpy array (or torch CPU tensor) in is copied to the current CUDA device, processed
there, and copied back. Work runs on torch's current CUDA stream.
"""
from __future__ import annotations

import numpy as np
import torch

NUMPY, TORCH_CPU, TORCH_CUDA = "numpy", "torch_cpu", "torch_cuda"


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("moraine_b200 runs on a CUDA device only (none is visible); "
                           "there is no CPU fallback")
    return torch.device("cuda", torch.cuda.current_device())


def kind_of(x) -> str:
    if isinstance(x, torch.Tensor):
        return TORCH_CUDA if x.is_cuda else TORCH_CPU
    return NUMPY


def to_device(x, dtype: torch.dtype | None = None, device: torch.device | None = None) -> torch.Tensor:
    """Contiguous CUDA tensor view/copy of ``x`` with ``dtype`` (if given)."""
    dev = device or require_cuda()
    if isinstance(x, torch.Tensor):
        t = x
    else:
        a = np.asarray(x)
        if a.dtype == np.bool_:
            a = a.view(np.uint8)
        t = torch.from_numpy(np.ascontiguousarray(a))
    if t.dtype == torch.bool:
        t = t.view(torch.uint8)
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    if t.device != dev:
        t = t.to(dev, non_blocking=False)
    return t.contiguous()


def from_device(t: torch.Tensor, kind: str, as_bool: bool = False):
    if as_bool:
        t = t.view(torch.bool)
    if kind == TORCH_CUDA:
        return t
    if kind == TORCH_CPU:
        return t.cpu()
    return t.cpu().numpy()


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def workspace(nbytes: int, device: torch.device) -> torch.Tensor:
    return torch.empty(max(16, int(nbytes)), dtype=torch.uint8, device=device)


def pairs_tensor(image_pairs, device) -> torch.Tensor | None:
    if image_pairs is None:
        return None
    return to_device(image_pairs, torch.int32, device)
