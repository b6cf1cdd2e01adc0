"""Per-round CPU times of the reference's own block Davidson, recorded as a
fixture for the benchmark's reference arm.

Runs gradwave's ``davidson_batched`` (``solvers/davidson.py:528-774``, float64,
CPU, the synchronous path) on a seeded cell from the identity start and
records, for every Rayleigh-Ritz round, its wall time, the largest residual
norm and the largest eigenvalue error against the cell's golden eigenvalues
(``<cell>.npz``, the same reference solve at tol 1e-10 eV). The run stops once
the eigenvalues are all within 1e-8 Ha of the golden ones (the benchmark's
unit of work: "one converged band solve, every eigenvalue within 1e-8 Ha of
the float64 oracle") and the largest residual is below ``--stop-tol``. The
rounds and their times go into ``reference_rounds.json`` beside this script;
``rounds`` and ``total_seconds`` count up to the first round that met the
eigenvalue criterion.

The reference is pure Python + torch but needs ``ase`` at package import; its
hot-path modules are imported through a namespace shim that bypasses the
package ``__init__``. Thread count: the reference's own default,
min(cores, 8) (gradwave ``_threads.py``), unless ``--threads`` is given.

Usage: python tests/golden/reference_rounds.py --ref <gradwave>/src [cells ...]
       (or set GWB_REFERENCE_SRC instead of --ref)
"""

from __future__ import annotations

import argparse
import json
import os
import platform
import sys
import time
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

HA = 27.211386245988
OUT = HERE / "reference_rounds.json"


class _Converged(Exception):
    pass


class _RoundLog(list):
    """``history_out`` of the reference's solver: every append is one
    finished Rayleigh-Ritz round (``(it, rn, eig)``); the time of each append
    and the eigenvalue error are recorded, and the solve is stopped once the
    error is within 1e-8 Ha."""

    def __init__(self, gold_eig: np.ndarray, t0: float, stop_tol: float):
        super().__init__()
        self.gold = gold_eig
        self.t_prev = t0
        self.stop_tol = stop_tol
        self.round_s: list[float] = []
        self.err_ev: list[float] = []
        self.rn_max: list[float] = []

    def append(self, item):
        now = time.perf_counter()
        self.round_s.append(now - self.t_prev)
        self.t_prev = now
        eig = item[2].numpy()
        err = float(np.abs(eig - self.gold).max())
        self.err_ev.append(err)
        self.rn_max.append(float(item[1].max()))
        if err <= 1e-8 * HA and self.rn_max[-1] <= self.stop_tol:
            raise _Converged()


def _cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or platform.machine()


def run(name: str, threads: int, max_iter: int, stop_tol: float) -> dict:
    from gradwave.core.batch import BatchedHamiltonian
    from gradwave.solvers.davidson import davidson_batched

    from gradwave_b200.cells import make_cell
    from make_golden import reference_setup

    torch.set_num_threads(threads)
    ci = make_cell(name, seed=0)
    grid, bk, p = reference_setup(ci)
    with np.load(HERE / f"{name}.npz") as z:
        gold = z["eigenvalues"]
    h = BatchedHamiltonian(bk, grid.shape, ci.v_eff_r, p)
    x0 = ci.identity_start()
    t0 = time.perf_counter()
    log = _RoundLog(gold, t0, stop_tol)
    converged = False
    try:
        davidson_batched(h.apply, x0, bk.t, bk.mask, tol=1e-10, max_iter=max_iter, history_out=log)
    except _Converged:
        converged = True
    ok = [i for i, e in enumerate(log.err_ev) if e <= 1e-8 * HA]
    n = ok[0] + 1 if ok else len(log.round_s)
    return {"cell": name, "threads": threads, "cpu": _cpu_model(), "cores": os.cpu_count(),
            "torch": torch.__version__, "converged_to_1e-8_ha": bool(ok),
            "rounds": n, "total_seconds": float(sum(log.round_s[:n])), "stop_tol_ev": stop_tol,
            "stopped": converged,
            "round_seconds": [round(s, 4) for s in log.round_s],
            "max_eig_err_ev": log.err_ev, "max_residual_ev": log.rn_max}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("cells", nargs="*", default=["si8_cubic", "si64_cubic", "si216_vacancy"])
    ap.add_argument("--ref", default=os.environ.get("GWB_REFERENCE_SRC"),
                    help="the reference's source directory (the one holding the gradwave package)")
    ap.add_argument("--threads", type=int, default=min(os.cpu_count() or 1, 8))
    ap.add_argument("--max-iter", type=int, default=200)
    ap.add_argument("--stop-tol", type=float, default=1e-7,
                    help="also run until the largest residual is below this (eV)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set GWB_REFERENCE_SRC")
    sys.path.insert(0, str(HERE))
    from make_golden import shim
    shim(args.ref)
    data = json.loads(OUT.read_text()) if OUT.exists() else {}
    for name in args.cells:
        rec = run(name, args.threads, args.max_iter, args.stop_tol)
        print(json.dumps({k: rec[k] for k in ("cell", "rounds", "total_seconds", "converged_to_1e-8_ha")}),
              flush=True)
        data[name] = rec
        OUT.write_text(json.dumps(data, indent=1) + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
