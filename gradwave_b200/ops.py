"""torch custom ops over the libgwb.so C ABI.

Each op takes the integer address of a library handle plus tensors, calls the
C entry point on torch's current CUDA stream and returns new tensors. They have
fake (meta) implementations so they trace under torch.compile / CUDA-graph
tooling without running.

    torch.ops.gwb.ham_apply(handle, c, prec) -> H c
"""

from __future__ import annotations

import torch

from . import _lib


@torch.library.custom_op("gwb::ham_apply", mutates_args=())
def ham_apply(handle: int, c: torch.Tensor, prec: int) -> torch.Tensor:
    _lib.require_cuda(c, "c")
    c = c.contiguous()
    out = torch.empty_like(c)
    nb = int(c.shape[1]) if c.dim() == 3 else 0
    _lib.call("gwb_ham_apply", handle, c.data_ptr(), out.data_ptr(), nb, _lib.io_dtype(c), int(prec),
              _lib.stream_ptr(c.device))
    return out


@ham_apply.register_fake
def _(handle, c, prec):
    return torch.empty_like(c)
