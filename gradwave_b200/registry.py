"""Block-eigensolver registry with the reference's contract
(gradwave ``solvers/registry.py:1-38,86-143,154-182``).

    solve(apply_H, X0, precond, mask, *, tol, nbands, **kw) -> EigResult

``apply_H`` (nk, nb, npw) -> (nk, nb, npw); ``X0`` the start block, padded 0;
``precond`` the kinetic diagonal T (nk, npw); ``mask`` (nk, npw) bool. The
result keeps the reference's field order, and ``diagnostics`` carries the
reference's keys (``solver``, ``max_dim_factor``, ``max_iter``,
``hit_max_iter``, ``n_apply_low``, ``n_apply_full``) plus this path's own.

Registered here: ``"davidson"`` (the B200 Davidson, float64 applies, TPA),
``"davidson_fp32exp"`` (the reference's float32-expansion mode) and
``"davidson_mixed"`` (float32 expansion applies with float64 certification and
the learned preconditioner when its weights are present). To
serve the reference's SCF loop, register the adapter into the reference's own
registry: ``gradwave.solvers.registry.register("davidson", davidson_adapter,
overwrite=True)``.
"""

from __future__ import annotations

from typing import Any, Callable, NamedTuple, Protocol

import torch


class EigResult(NamedTuple):
    eigenvalues: torch.Tensor      # (nk, nbands) ascending
    eigenvectors: torch.Tensor     # (nk, nbands, npw), padded slots zero
    n_iter: int
    residual_norms: torch.Tensor   # (nk, nbands)
    diagnostics: dict[str, Any]


class BlockEigensolver(Protocol):
    def __call__(self, apply_H: Callable[[torch.Tensor], torch.Tensor], X0: torch.Tensor, precond: torch.Tensor,
                 mask: torch.Tensor, *, tol: float, nbands: int, **kw: Any) -> EigResult: ...


_REGISTRY: dict[str, BlockEigensolver] = {}


def register(name: str, solver: BlockEigensolver, *, overwrite: bool = False) -> None:
    if name in _REGISTRY and not overwrite:
        raise ValueError(f"eigensolver {name!r} already registered; pass overwrite=True to replace")
    _REGISTRY[name] = solver


def get(name: str) -> BlockEigensolver:
    try:
        return _REGISTRY[name]
    except KeyError:
        raise ValueError(f"unknown eigensolver {name!r}; registered: {sorted(_REGISTRY)}") from None


def available() -> list[str]:
    return sorted(_REGISTRY)


def is_registered(name: str) -> bool:
    return name in _REGISTRY


def _adapter(mode: str, learned: bool = False):
    def davidson_adapter(apply_H, X0, precond, mask, *, tol, nbands=None, max_iter: int = 40,
                         max_dim_factor: int = 4, **kw) -> EigResult:
        from .davidson import davidson_batched
        pc = kw.pop("preconditioner", None)
        if pc is None:
            pc = "teter"
            if learned:
                from . import learned as lp
                if lp.available():
                    pc = lp.LearnedPreconditioner.load(device=X0.device)
        m = kw.pop("mode", mode)
        r = davidson_batched(apply_H, X0, precond, mask, tol=tol, max_iter=max_iter,
                             max_dim_factor=max_dim_factor, mode=m, precond=pc)
        diag = {"solver": "davidson", "max_dim_factor": max_dim_factor, "max_iter": max_iter,
                "hit_max_iter": r.n_iter >= max_iter, "n_apply_low": r.n_apply_low,
                "n_apply_full": r.n_apply_full, "mode": m,
                "preconditioner": "teter" if isinstance(pc, str) else "learned"}
        diag.update(r.info)
        return EigResult(r.eigenvalues, r.eigenvectors, r.n_iter, r.residual_norms, diag)

    davidson_adapter.__name__ = f"davidson_adapter_{mode}{'_learned' if learned else ''}"
    return davidson_adapter


davidson_adapter = _adapter("fp64")
davidson_fp32exp_adapter = _adapter("fp32exp")
davidson_mixed_adapter = _adapter("mixed", learned=True)

register("davidson", davidson_adapter)
register("davidson_fp32exp", davidson_fp32exp_adapter)
register("davidson_mixed", davidson_mixed_adapter)
