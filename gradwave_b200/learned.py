"""Learned Davidson preconditioner: training data, GPU training, inference.

A per-plane-wave network (4 -> 64 -> 64 -> 64 -> 1, SiLU, BF16 weights and
activations, FP32 accumulation; kernels in ``csrc/mlp.cu``) corrects the
Teter-Payne-Allan filter: K(G) = TPA(x) exp(o(u)) with the features u of
``gwb_precond_features`` (|k+G|^2 relative to the band's kinetic energy, the
band eigenvalue, the residual amplitude at G and the band's kinetic scale).
TPA stays the fallback and the yardstick: a band whose residual has not improved
on its best value by 10 % for three consecutive rounds reverts to TPA for the
rest of the solve.

Training data come from the Davidson solver itself. A cell is solved twice
with TPA: once to convergence (eigenvectors psi), then again while every round
keeps some of the selected bands whole: features at every plane wave, the
residual r = H x - eps x and the error e = x - P_psi x of the Ritz vector
against the converged eigenspace of its band cluster. Since r ~ (H - eps) e,
the ideal expansion direction is e; the network is trained to maximise, per
band, the alignment |<K r, e>|^2 / (|K r|^2 |e|^2) of the preconditioned
residual with the error (the expansion direction is scale free). The loss
gradient per plane wave comes from band sums; the network's backward pass,
forward pass and Adam are the project's own kernels.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _lib

DATA = Path(__file__).resolve().parent / "data"
WEIGHTS = DATA / "precond_mlp.npy"
HID, NIN = 64, 4


def nparam() -> int:
    return int(_lib.load().gwb_mlp_param_count())


def init_params(seed: int = 0) -> np.ndarray:
    """He initialisation with a zero output layer: the untrained network is
    exactly TPA."""
    rng = np.random.default_rng(seed)
    parts = [rng.standard_normal((HID, NIN)) * math.sqrt(2.0 / NIN), np.zeros(HID),
             rng.standard_normal((HID, HID)) * math.sqrt(2.0 / HID), np.zeros(HID),
             rng.standard_normal((HID, HID)) * math.sqrt(2.0 / HID), np.zeros(HID), np.zeros(HID), np.zeros(1)]
    return np.concatenate([p.reshape(-1) for p in parts]).astype(np.float32)


def _s(dev):
    return _lib.stream_ptr(dev)


def forward(params: torch.Tensor, feats: torch.Tensor) -> torch.Tensor:
    out = torch.empty(feats.shape[0], dtype=torch.float32, device=feats.device)
    _lib.call("gwb_mlp_forward", params.data_ptr(), int(feats.shape[0]), feats.contiguous().data_ptr(),
              out.data_ptr(), _s(feats.device))
    return out


def loss_grad(params: torch.Tensor, feats, target, weight):
    """(loss tensor (1,), grad tensor) of sum w (o - y)^2 on the GPU."""
    dev = feats.device
    grad = torch.zeros(params.numel(), dtype=torch.float32, device=dev)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    _lib.call("gwb_mlp_loss_grad", params.data_ptr(), int(feats.shape[0]), feats.contiguous().data_ptr(),
              target.contiguous().data_ptr(), weight.contiguous().data_ptr(), grad.data_ptr(), loss.data_ptr(),
              _s(dev))
    return loss, grad


@dataclass
class TrainResult:
    params: torch.Tensor
    train_loss: list
    val_loss: float
    val_loss_tpa: float


def train(feats: torch.Tensor, target: torch.Tensor, weight: torch.Tensor, *, steps: int = 3000,
          batch: int = 16384, lr: float = 2e-3, seed: int = 0, val_frac: float = 0.1) -> TrainResult:
    """Adam on the weighted MSE with the GPU kernels; the last val_frac of
    the (shuffled) samples is held out. val_loss_tpa is the loss of the
    untrained (= TPA) network on the same samples."""
    dev = feats.device
    g = torch.Generator(device="cpu").manual_seed(seed)
    perm = torch.randperm(feats.shape[0], generator=g).to(dev)
    feats, target, weight = feats[perm].contiguous(), target[perm].contiguous(), weight[perm].contiguous()
    nval = max(1, int(val_frac * feats.shape[0]))
    ft, yt, wt = feats[:-nval], target[:-nval], weight[:-nval]
    fv, yv, wv = feats[-nval:], target[-nval:], weight[-nval:]
    wv = wv / wv.sum()
    params = torch.from_numpy(init_params(seed)).to(dev)
    m = torch.zeros_like(params)
    v = torch.zeros_like(params)
    val_tpa = float(loss_grad(params, fv, yv, wv)[0].item())
    hist = []
    n = ft.shape[0]
    for step in range(1, steps + 1):
        idx = torch.randint(0, n, (min(batch, n),), generator=g).to(dev)
        wb = wt[idx]
        wb = wb / wb.sum()
        loss, grad = loss_grad(params, ft[idx], yt[idx], wb)
        lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * step / steps))
        _lib.call("gwb_mlp_adam", params.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(), step,
                  ctypes.c_float(lr_t), ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), _s(dev))
        if step % 100 == 0 or step == 1:
            hist.append((step, float(loss.item())))
    val = float(loss_grad(params, fv, yv, wv)[0].item())
    return TrainResult(params, hist, val, val_tpa)


class LearnedPreconditioner:
    """The network as a Davidson preconditioner (``precond=`` argument of
    ``davidson_batched``). Host-driver hook: ``apply_into(solver, n_add, eig)``."""

    stall_ratio = 0.9
    stall_patience = 3

    def __init__(self, params, device=None):
        p = torch.as_tensor(np.asarray(params, dtype=np.float32) if not torch.is_tensor(params) else params)
        dev = device or (p.device if p.is_cuda else torch.device("cuda", torch.cuda.current_device()))
        self.params = p.to(dev, torch.float32).contiguous()
        if self.params.numel() != nparam():
            raise ValueError(f"expected {nparam()} parameters, got {self.params.numel()}")

    @classmethod
    def load(cls, path: Path | str = WEIGHTS, device=None) -> "LearnedPreconditioner":
        return cls(np.load(path), device)

    def save(self, path: Path | str = WEIGHTS) -> None:
        np.save(path, self.params.cpu().numpy())

    def apply_into(self, solver, n_add: int, eig: torch.Tensor) -> None:
        ws, nk, nb, npw = solver.ws, solver.nk, solver.nb, solver.npw
        st = getattr(solver, "_lp_state", None)
        if st is None:
            st = (torch.full((nk, nb), float("inf"), dtype=torch.float64, device=solver.dev),
                  torch.zeros(nk, nb, dtype=torch.uint8, device=solver.dev),
                  torch.zeros(nk, nb, dtype=torch.uint8, device=solver.dev))
            solver._lp_state = st
        rn_best, count, tpa_only = st
        _lib.call("gwb_stall_update", ws.rn.data_ptr(), rn_best.data_ptr(), count.data_ptr(), tpa_only.data_ptr(),
                  nk * nb, self.stall_ratio, self.stall_patience, solver.stream)
        solver.n_tpa_fallback = int(0)  # read lazily by callers that want it
        eigc = eig.contiguous()
        solver._lp_eig = eigc
        work = getattr(solver, "_lp_work", None)
        if work is None:  # per solve: concurrent solves on other streams never share it
            work = _precond_work(solver.dev, nk, nb, npw)
            solver._lp_work = work
        _lib.call("gwb_precond_learned", self.params.data_ptr(), nk, nb, n_add, npw, ws.X.data_ptr(), nb * npw,
                  ws.R.data_ptr(), nb * npw, solver.t.data_ptr(), eigc.data_ptr(), ws.sel.data_ptr(),
                  tpa_only.data_ptr(), ws.D.data_ptr(), nb * npw, work.data_ptr(), work.numel(), solver.stream)


def _precond_work(dev, nk: int, n_rows: int, npw: int) -> torch.Tensor:
    """Scratch of gwb_precond_learned for up to n_rows selected rows per k."""
    need = int(_lib.load().gwb_precond_learned_work_bytes(nk, n_rows, npw))
    return torch.empty(max(need, 8), dtype=torch.uint8, device=dev)


# ---------------------------------------------------------------------------
# training data from the solver


def _tpa_from_u0(u0: torch.Tensor) -> torch.Tensor:
    x = torch.expm1(u0.double())
    x2 = x * x
    p = 27.0 + 18.0 * x + 12.0 * x2 + 8.0 * x2 * x
    return p / (p + 16.0 * x2 * x2)


class RowLogger:
    """Host-driver preconditioner hook that applies TPA and, every round,
    keeps up to ``rows_per_round`` of the selected bands whole: their network
    features at every plane wave, the residual r and the error e = x - P x of
    the Ritz vector against the converged eigenspace of its band cluster
    (``psi``/``eig_final`` from a first pass over the same cell)."""

    def __init__(self, psi: torch.Tensor, eig_final: torch.Tensor, rows_per_round: int = 48, seed: int = 0,
                 cluster_tol: float = 1e-3):
        self.psi = psi
        self.eig_final = eig_final
        self.rows_per_round = rows_per_round
        self.gen = torch.Generator(device="cpu").manual_seed(seed)
        self.cluster_tol = cluster_tol
        self.F, self.R, self.E, self.M = [], [], [], []

    def apply_into(self, solver, n_add: int, eig: torch.Tensor) -> None:
        ws, nk, nb, npw = solver.ws, solver.nk, solver.nb, solver.npw
        dev = solver.dev
        feats = torch.empty(nk, n_add, npw, NIN, dtype=torch.float32, device=dev)
        eigc = eig.contiguous()
        _lib.call("gwb_precond_features", nk, nb, n_add, npw, ws.X.data_ptr(), nb * npw, ws.R.data_ptr(),
                  nb * npw, solver.t.data_ptr(), eigc.data_ptr(), ws.sel.data_ptr(), feats.data_ptr(), solver.stream)
        sel = ws.sel.view(-1)[: nk * n_add].view(nk, n_add).long()
        x = torch.gather(ws.X, 1, sel[..., None].expand(nk, n_add, npw))
        r = torch.gather(ws.R, 1, sel[..., None].expand(nk, n_add, npw))
        eb = torch.gather(self.eig_final, 1, sel)
        cl = (self.eig_final[:, None, :] - eb[..., None]).abs() <= self.cluster_tol
        ov = torch.einsum("kcg,kag->kac", self.psi.conj(), x) * cl
        e = x - torch.einsum("kac,kcg->kag", ov, self.psi)
        mask = solver.mask[:, None, :].expand(nk, n_add, npw)
        pick = torch.randperm(nk * n_add, generator=self.gen)[: self.rows_per_round].to(dev)
        self.F.append(feats.reshape(-1, npw, NIN)[pick])
        self.R.append(r.reshape(-1, npw)[pick].to(torch.complex64))
        self.E.append(e.reshape(-1, npw)[pick].to(torch.complex64))
        self.M.append(mask.reshape(-1, npw)[pick])
        _lib.call("gwb_precond_teter", nk, nb, n_add, npw, ws.X.data_ptr(), nb * npw, ws.R.data_ptr(), nb * npw,
                  solver.t.data_ptr(), ws.sel.data_ptr(), ws.D.data_ptr(), nb * npw, solver.stream)

    def rows(self):
        return torch.cat(self.F), torch.cat(self.R), torch.cat(self.E), torch.cat(self.M)


def collect_rows(cell_specs, tol: float = 1e-8, rows_per_round: int = 48, max_iter: int = 200, device=None):
    """Logged rows (features, r, e, mask) from two-pass TPA solves of the
    given (name, seed) cells; rows of cells with different npw are padded."""
    from .cells import make_cell
    from .davidson import davidson_batched
    from .hamiltonian import BatchedHamiltonian
    dev = device or torch.device("cuda", 0)
    parts = []
    for name, seed in cell_specs:
        ci = make_cell(name, seed=seed)
        bk = ci.bk.to(dev)
        h = BatchedHamiltonian(bk, ci.shape, ci.v_eff_r, ci.p)
        x0 = ci.identity_start().to(dev)
        ref = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=tol, max_iter=max_iter)
        lg = RowLogger(ref.eigenvectors, ref.eigenvalues, rows_per_round=rows_per_round, seed=seed)
        davidson_batched(h.apply, x0, bk.t, bk.mask, tol=tol, max_iter=max_iter, precond=lg)
        parts.append(lg.rows())
    npw = max(p[0].shape[1] for p in parts)

    def pad(t, fill=0):
        if t.shape[1] == npw:
            return t
        shape = list(t.shape)
        shape[1] = npw - t.shape[1]
        return torch.cat([t, torch.full(shape, fill, dtype=t.dtype, device=t.device)], dim=1)
    return tuple(torch.cat([pad(p[i]) for p in parts]) for i in range(4))


def alignment_loss(params, F, R, E, M, dout: bool = False):
    """Mean over rows of 1 - |<K r, e>|^2 / (|K r|^2 |e|^2) with
    K = TPA exp(clamp(o, -3, 3)) on the mask; with dout also dL/do per sample."""
    nrow, npw = M.shape
    o = forward(params, F.reshape(-1, NIN)).view(nrow, npw).double()
    oc = o.clamp(-3.0, 3.0)
    K = _tpa_from_u0(F[..., 0]) * torch.exp(oc) * M
    r = R.to(torch.complex128)
    e = E.to(torch.complex128)
    a = r.conj() * e
    r2 = r.abs() ** 2
    A = (K * a).sum(-1)
    B = (K * K * r2).sum(-1).clamp_min(1e-300)
    C = (e.abs() ** 2).sum(-1).clamp_min(1e-300)
    L = 1.0 - A.abs() ** 2 / (B * C)
    if not dout:
        return float(L.mean())
    dK = -(2.0 * (A.conj()[:, None] * a).real * B[:, None] - (A.abs() ** 2)[:, None] * 2.0 * K * r2) \
        / (B * B * C)[:, None]
    do = dK * K * ((o > -3.0) & (o < 3.0)) / nrow
    return float(L.mean()), do.float().reshape(-1).contiguous()


def train_alignment(F, R, E, M, *, steps: int = 1500, batch_rows: int = 32, lr: float = 2e-3, seed: int = 0,
                    val_frac: float = 0.15) -> TrainResult:
    """Adam on the alignment loss with the project's forward/backward kernels;
    the last val_frac of the shuffled rows are held out. val_loss_tpa is the
    held-out loss of the untrained network (exactly TPA)."""
    dev = F.device
    g = torch.Generator(device="cpu").manual_seed(seed)
    perm = torch.randperm(F.shape[0], generator=g).to(dev)
    F, R, E, M = F[perm], R[perm], E[perm], M[perm]
    nval = max(1, int(val_frac * F.shape[0]))
    tr = slice(0, F.shape[0] - nval)
    va = slice(F.shape[0] - nval, F.shape[0])
    params = torch.from_numpy(init_params(seed)).to(dev)
    m = torch.zeros_like(params)
    v = torch.zeros_like(params)
    val_tpa = alignment_loss(params, F[va], R[va], E[va], M[va])
    hist = []
    ntr = F.shape[0] - nval
    for step in range(1, steps + 1):
        idx = torch.randint(0, ntr, (min(batch_rows, ntr),), generator=g).to(dev)
        Fb = F[idx].contiguous()
        loss, do = alignment_loss(params, Fb, R[idx], E[idx], M[idx], dout=True)
        grad = torch.zeros_like(params)
        _lib.call("gwb_mlp_backward", params.data_ptr(), int(do.numel()), Fb.reshape(-1, NIN).data_ptr(),
                  do.data_ptr(), grad.data_ptr(), _s(dev))
        lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * step / steps))
        _lib.call("gwb_mlp_adam", params.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(), step,
                  ctypes.c_float(lr_t), ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), _s(dev))
        if step % 100 == 0 or step == 1:
            hist.append((step, loss))
    val = alignment_loss(params, F[va], R[va], E[va], M[va])
    return TrainResult(params, hist, val, val_tpa)


def available() -> bool:
    """Whether trained weights are present in the package."""
    return WEIGHTS.exists()


def main(argv=None) -> int:
    """Train the preconditioner on the GPU from solver-logged pairs:

        python -m gradwave_b200.learned --cells si8_perturbed:1,si8_perturbed:2 --out precond_mlp.npy
    """
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", default="si8_perturbed:1,si8_perturbed:2,si8_perturbed:3")
    ap.add_argument("--rows-per-round", type=int, default=48)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch-rows", type=int, default=32)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=str(WEIGHTS))
    a = ap.parse_args(argv)
    specs = [(c.split(":")[0], int(c.split(":")[1])) for c in a.cells.split(",")]
    t0 = time.perf_counter()
    F, R, E, M = collect_rows(specs, rows_per_round=a.rows_per_round)
    t1 = time.perf_counter()
    res = train_alignment(F, R, E, M, steps=a.steps, batch_rows=a.batch_rows, lr=a.lr)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    np.save(a.out, res.params.cpu().numpy())
    print(json.dumps({"rows": int(F.shape[0]), "pairs": int(M.sum()), "collect_s": round(t1 - t0, 1),
                      "train_s": round(t2 - t1, 1), "val_loss": res.val_loss, "val_loss_tpa": res.val_loss_tpa,
                      "train_loss": res.train_loss[-5:], "out": a.out}), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
