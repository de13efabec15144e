"""Device context (mirrors python/cudolfinx/context.py:29-35).

The reference creates a PETSc CUDA device and retains the primary CUDA
context of device 0 (cpp/cudolfinx/common/CUDA.cpp:28-52).  Here one engine
context per device is created on first use; work is issued on torch's current
CUDA stream of that device.
"""
from __future__ import annotations

import torch

from . import _lib

_contexts: dict[int, "Context"] = {}


class Context:
    def __init__(self, device: int):
        self.device = device
        h = _lib.out_handle()
        _lib.check(_lib.lib.fe_context_create(device, h), "fe_context_create")
        self.handle = h.value

    def synchronize(self):
        """Wait for the device and raise if a kernel reported an error word."""
        _lib.check(_lib.lib.fe_context_synchronize(self.handle), "fe_context_synchronize")

    def stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    @property
    def torch_device(self):
        return torch.device("cuda", self.device)


def get_cuda_context(device: int | None = None) -> Context:
    """Return the engine context of ``device`` (default: torch's current device)."""
    if not torch.cuda.is_available():
        raise RuntimeError("cudolfinx_b200 needs a CUDA device (B200, sm_100a); none is visible")
    if device is None:
        device = torch.cuda.current_device()
    ctx = _contexts.get(device)
    if ctx is None:
        ctx = Context(device)
        _contexts[device] = ctx
    return ctx
