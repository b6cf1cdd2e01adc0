"""torch custom ops over the libgwb.so C ABI.

Each op takes the integer address of a library handle (where it needs one)
plus tensors, calls the C entry point on torch's current CUDA stream and
returns new tensors. They have fake (meta) implementations so they trace
under torch.compile / CUDA-graph tooling without running.

    torch.ops.gwb.ham_apply(handle, c, prec) -> H c
        gwb_ham_apply (gradwave core/batch.py:480-505)
    torch.ops.gwb.davidson_solve(handle, x0, t, mask, tol, max_iter, max_dim, mode, flags, params)
        -> (eigenvalues, eigenvectors, residual_norms, stats)
        gwb_davidson_solve (gradwave solvers/davidson.py:528-774); params is
        the learned preconditioner's weights or None for TPA; stats holds
        SOLVE_STATS (host float64)
    torch.ops.gwb.precond_apply(x, r, t, sel, eig, params, tpa_only) -> d
        the preconditioned, unit-normalised residuals of the selected bands:
        gwb_precond_teter (gradwave solvers/precond.py:20-39) when params is
        None, else gwb_precond_learned (TPA x exp(network), TPA for the bands
        flagged in tpa_only)
"""

from __future__ import annotations

import ctypes
from typing import Optional

import torch

from . import _lib

# stats of davidson_solve, in this order (float64)
SOLVE_STATS = ("n_iter", "hit_max_iter", "n_restart", "n_cert", "n_repair", "n_rollback", "n_apply_low",
               "n_apply_full", "max_residual", "apply_ms", "n_apply_calls", "n_tpa_fallback")
SOLVE_TIME_APPLIES = 1   # flags bit: CUDA-event totals of the H applies into the apply_ms stat
SOLVE_MODES = {"fp64": 0, "fp32exp": 1, "mixed": 2}


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


@torch.library.custom_op("gwb::davidson_solve", mutates_args=())
def davidson_solve(handle: int, x0: torch.Tensor, t: torch.Tensor, mask: torch.Tensor, tol: float, max_iter: int,
                   max_dim: int, mode: int, flags: int, params: Optional[torch.Tensor]
                   ) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]:
    """The whole block Davidson in one library call on a Hamiltonian handle.
    A status other than success raises (``GwbError``); a breakdown the library
    does not repair is GWB_ERR_BREAKDOWN."""
    _lib.require_cuda(x0, "x0")
    if x0.dtype != torch.complex128 or x0.dim() != 3:
        raise ValueError("x0 must be a (nk, nb, npw) complex128 tensor")
    nk, nb, npw = (int(s) for s in x0.shape)
    dev = x0.device
    p = _lib.DavidsonParams(nk, nb, npw, int(max_dim), int(max_iter), int(mode), 0 if params is None else 1,
                            int(flags), float(tol), float(t.max()))
    nbytes = ctypes.c_size_t()
    _lib.call("gwb_davidson_workspace_bytes", ctypes.byref(p), ctypes.byref(nbytes))
    ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=dev)
    x0c = x0.contiguous()
    tc = t.to(dev, torch.float64).contiguous()
    mk = mask.to(dev, torch.uint8).contiguous()
    eig = torch.empty(nk, nb, dtype=torch.float64, device=dev)
    vec = torch.empty(nk, nb, npw, dtype=torch.complex128, device=dev)
    rn = torch.empty(nk, nb, dtype=torch.float64, device=dev)
    st = _lib.DavidsonStats()
    pp = None if params is None else params.to(dev, torch.float32).contiguous()
    _lib.call("gwb_davidson_solve", handle, ctypes.byref(p), None if pp is None else pp.data_ptr(), x0c.data_ptr(),
              tc.data_ptr(), mk.data_ptr(), ws.data_ptr(), ws.numel(), eig.data_ptr(), vec.data_ptr(), rn.data_ptr(),
              ctypes.byref(st), _lib.stream_ptr(dev))
    stats = torch.tensor([float(getattr(st, k)) for k in SOLVE_STATS], dtype=torch.float64)
    return eig, vec, rn, stats


@davidson_solve.register_fake
def _(handle, x0, t, mask, tol, max_iter, max_dim, mode, flags, params):
    nk, nb, npw = x0.shape
    return (x0.new_empty((nk, nb), dtype=torch.float64), torch.empty_like(x0),
            x0.new_empty((nk, nb), dtype=torch.float64),
            torch.empty(len(SOLVE_STATS), dtype=torch.float64, device="cpu"))


@torch.library.custom_op("gwb::precond_apply", mutates_args=())
def precond_apply(x: torch.Tensor, r: torch.Tensor, t: torch.Tensor, sel: torch.Tensor, eig: torch.Tensor,
                  params: Optional[torch.Tensor], tpa_only: Optional[torch.Tensor]) -> torch.Tensor:
    """Rows d (nk, n_add, npw): for s < n_add the preconditioned residual of
    band sel[k, s] (x, r: (nk, nb, npw) complex128 Ritz vectors and
    residuals; t: (nk, npw) kinetic diagonal; eig: (nk, nb)), unit-normalised."""
    _lib.require_cuda(x, "x")
    nk, nb, npw = (int(s) for s in x.shape)
    n_add = int(sel.shape[1])
    dev = x.device
    x, r = x.contiguous(), r.contiguous()
    tc = t.to(dev, torch.float64).contiguous()
    sl = sel.to(dev, torch.int32).contiguous()
    d = torch.empty(nk, n_add, npw, dtype=torch.complex128, device=dev)
    s = _lib.stream_ptr(dev)
    if params is None:
        _lib.call("gwb_precond_teter", nk, nb, n_add, npw, x.data_ptr(), nb * npw, r.data_ptr(), nb * npw,
                  tc.data_ptr(), sl.data_ptr(), d.data_ptr(), n_add * npw, s)
        return d
    pp = params.to(dev, torch.float32).contiguous()
    ev = eig.to(dev, torch.float64).contiguous()
    fb = (torch.zeros(nk, nb, dtype=torch.uint8, device=dev) if tpa_only is None
          else tpa_only.to(dev, torch.uint8).contiguous())
    need = int(_lib.load().gwb_precond_learned_work_bytes(nk, n_add, npw))
    work = torch.empty(max(need, 8), dtype=torch.uint8, device=dev)
    _lib.call("gwb_precond_learned", pp.data_ptr(), nk, nb, n_add, npw, x.data_ptr(), nb * npw, r.data_ptr(),
              nb * npw, tc.data_ptr(), ev.data_ptr(), sl.data_ptr(), fb.data_ptr(), d.data_ptr(), n_add * npw,
              work.data_ptr(), work.numel(), s)
    return d


@precond_apply.register_fake
def _(x, r, t, sel, eig, params, tpa_only):
    return x.new_empty((x.shape[0], sel.shape[1], x.shape[2]))
