"""Measured chunk and split choices of the Hamiltonian apply (the path's
autotuner).

Two choices of the apply are not fixed by the data and depend on the box, the
projector count and the GPU:

* the FFT scratch per band chunk (``w_budget``): the local term runs the
  bands in chunks whose plane scratch W should stay in the 126 MB L2; larger
  chunks mean fewer, larger launches;
* the number of CTAs the G-sliced projector contraction aims for
  (``nl_target``): more slices fill the SMs, more partial sums cost a
  reduction;
* the threads per block of the shared-memory FFT kernels of the 72^3 and
  96^3 boxes, per precision (``fft_threads``): a float64 96^3 plane fills an
  SM's shared memory, so its block's warps are all the latency hiding there is.

``tune(config)`` times whole-block applies of a workload (float32 and float64
arithmetic, CUDA events, several repetitions) over a grid of both values and
records every timing and the choice with the least summed time in
``data/tuning.json``, keyed by apply kind, box and projector count. Every
``BatchedHamiltonian`` and ``GammaHamiltonian`` looks its key up at
construction and sets the recorded choice on its handle
(``gwb_ham_set_tuning``); without an entry the built-in rules apply.

    python -m gradwave_b200.autotune --config si216_vacancy --out tuning.json
"""

from __future__ import annotations

import json
from pathlib import Path

from . import _lib

TUNING = Path(__file__).resolve().parent / "data" / "tuning.json"
_CACHE: dict | None = None


def key(kind: str, shape, nproj: int) -> str:
    n0, n1, n2 = (int(s) for s in shape)
    return f"{kind}:{n0}x{n1}x{n2}:p{int(nproj)}"


def _table() -> dict:
    global _CACHE
    if _CACHE is None:
        _CACHE = json.loads(TUNING.read_text()) if TUNING.exists() else {}
    return _CACHE


def lookup(kind: str, shape, nproj: int) -> dict | None:
    """The recorded choice for this apply kind, box and projector count."""
    return _table().get("entries", {}).get(key(kind, shape, nproj), {}).get("choice")


def apply_tuning(handle, kind: str, shape, nproj: int) -> dict | None:
    """Set the recorded choice (if any) on a libgwb handle; returns it.
    ``GWB_FFT_THREADS=fp32,fp64`` overrides the FFT block threads."""
    import os
    ch = lookup(kind, shape, nproj)
    if ch is not None:
        _lib.call("gwb_ham_set_tuning", handle, int(ch["w_budget_mb"]) << 20, int(ch["nl_target"]))
    nt = os.environ.get("GWB_FFT_THREADS")
    if nt:
        n32, n64 = (int(x) for x in nt.split(","))
        _lib.call("gwb_ham_set_fft_threads", handle, n32, n64)
    elif ch is not None and "fft_threads" in ch:
        _lib.call("gwb_ham_set_fft_threads", handle, int(ch["fft_threads"][0]), int(ch["fft_threads"][1]))
    return ch


def tune(config: str, budgets_mb=(16, 24, 32, 48, 64, 96, 128), targets=(148, 296, 592, 1184), steps: int = 5,
         warmup: int = 2, device=None) -> tuple[str, dict]:
    """Time the whole-block applies of ``config`` over the grid; returns
    (key, entry) with the table and the choice."""
    import torch
    from .cells import make_cell
    dev = device or torch.device("cuda", 0)
    ci = make_cell(config)
    gamma = ci.bk.nk == 1 and bool((abs(ci.kpoints) == 0).all())
    if gamma:
        from .gamma import GammaHamiltonian, build_gamma_basis
        gb = build_gamma_basis(ci.spheres[0], ci.shape)
        ham = GammaHamiltonian(gb, ci.v_eff_r, ci.p[0], ci.bk.dij_full, device=dev)
        g = torch.Generator().manual_seed(3)
        blk = torch.randn(ci.nbands, 2 * gb.nhalf - 1, dtype=torch.float64, generator=g).to(dev)

        def run(prec):
            ham.apply_phi(blk, prec=prec)
        handle, kind = ham._h, "gamma"
    else:
        from .hamiltonian import BatchedHamiltonian
        ham = BatchedHamiltonian(ci.bk.to(dev), ci.shape, ci.v_eff_r, ci.p)
        g = torch.Generator().manual_seed(3)
        blk = torch.randn(ci.bk.nk, ci.nbands, ci.bk.npw_max, dtype=torch.complex128, generator=g).to(dev)
        blk = blk * ham.mask[:, None, :]

        def run(prec):
            if prec == _lib.GWB_FP64:
                ham.apply(blk)
            else:
                ham.apply_fp32(blk)
        handle, kind = ham._h, "complex"
    nproj = int(ci.p.shape[1])

    def timed(prec) -> float:
        for _ in range(warmup):
            run(prec)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            run(prec)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    rows = []
    for mb in budgets_mb:
        for tg in targets:
            _lib.call("gwb_ham_set_tuning", handle, int(mb) << 20, int(tg))
            t32, t64 = timed(_lib.GWB_FP32), timed(_lib.GWB_FP64)
            rows.append({"w_budget_mb": mb, "nl_target": tg, "fp32_ms": round(t32, 4), "fp64_ms": round(t64, 4)})
    _lib.call("gwb_ham_set_tuning", handle, 0, 0)
    base = {"fp32_ms": round(timed(_lib.GWB_FP32), 4), "fp64_ms": round(timed(_lib.GWB_FP64), 4)}
    best = min(rows, key=lambda r: r["fp32_ms"] + r["fp64_ms"])
    _lib.call("gwb_ham_set_tuning", handle, int(best["w_budget_mb"]) << 20, int(best["nl_target"]))
    threads = []
    for nt in (256, 512, 1024):
        _lib.call("gwb_ham_set_fft_threads", handle, nt, nt)
        threads.append({"threads": nt, "fp32_ms": round(timed(_lib.GWB_FP32), 4),
                        "fp64_ms": round(timed(_lib.GWB_FP64), 4)})
    _lib.call("gwb_ham_set_fft_threads", handle, 0, 0)
    n32 = min(threads, key=lambda r: r["fp32_ms"])["threads"]
    n64 = min(threads, key=lambda r: r["fp64_ms"])["threads"]
    t32 = min(r["fp32_ms"] for r in threads)
    t64 = min(r["fp64_ms"] for r in threads)
    entry = {"config": config, "kind": kind, "bands": int(ci.nbands), "gpu": torch.cuda.get_device_name(dev),
             "timing": f"CUDA events, {steps} applies after {warmup}", "built_in_rule": base,
             "choice": {"w_budget_mb": best["w_budget_mb"], "nl_target": best["nl_target"],
                        "fft_threads": [n32, n64]},
             "gain": round((base["fp32_ms"] + base["fp64_ms"]) / (t32 + t64), 4),
             "table": rows, "fft_threads_table": threads}
    return key(kind, ci.shape, nproj), entry


def main(argv=None) -> int:
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", action="append", required=True)
    ap.add_argument("--out", default=str(TUNING))
    a = ap.parse_args(argv)
    out = Path(a.out)
    data = json.loads(out.read_text()) if out.exists() else {}
    data.setdefault("entries", {})
    for cfg in a.config:
        k, e = tune(cfg)
        data["entries"][k] = e
        print(json.dumps({"key": k, "choice": e["choice"], "gain": e["gain"], "built_in_rule": e["built_in_rule"]}),
              flush=True)
    out.write_text(json.dumps(data, indent=1) + "\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
