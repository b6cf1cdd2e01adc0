"""Benchmark: ms per converged band solve on one B200 (eigenvalues within
1e-8 Ha of the float64 reference).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME] [--impl ours|reference]

A step is one converged band solve of the workload (default ``si8_cubic``: the
8-atom cubic Si cell, 40 Ry, 10 irreducible k, 24 bands, 36^3 box) from the
identity start. Our arm reports:

* ``value``       device-timed ms per solve with the inputs resident in HBM
                  (CUDA events on the launching stream, max over ranks); the
                  solver is the product's fast mode (float32 expansion applies
                  with float64 certification, then float64 polish);
* ``e2e``         the same solve through the public API from pinned host
                  memory: H2D of the start block, solve, D2H of eigenvalues and
                  eigenvectors, all inside the timed region;
* ``plain_fp64``  the plain float64 TPA Davidson on the same GPU and kernels;
* ``roofline``    for the dominant kernel (the Hamiltonian apply), measured
                  live with CUDA events around its launches;
* ``cpu_baseline`` the float64 oracle (numpy restatement of the reference)
                  on the host cores, on a bounded sample of the same workload.

Between timed steps a 256 MiB buffer is written to flush L2 (126 MB).
Eigenvalue error is checked against the reference's own eigenvalues
(``tests/golden``) and reported; a solve outside 1e-8 Ha fails the run.

With N > 1 (torchrun) every rank solves its own k-shard of an N-fold k-set
(the si8 k-points on every rank: weak scaling, no collective inside the
solve; the eigenvalues are all-gathered once after the timed region) and
``value`` is the whole-job time per solve: the max over ranks of the step time
divided by N.

``--impl reference`` times the reference's CPU path (the float64 oracle port;
the reference itself is Python and does not travel) with all host threads on
a bounded k-point sample, scaled to the full workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

HA = 27.211386245988
EIG_TOL_EV = 1e-8 * HA
METRIC = "ms per converged band solve (eig err ≤1e-8 Ha): learned+mixed vs plain, 1 B200"
GOLDEN = {"si2_fcc": "si2_fcc", "si8_cubic": "si8_cubic", "si64_cubic": "si64_cubic",
          "si216_vacancy": "si216_vacancy"}


def _golden(name):
    p = ROOT / "tests" / "golden" / f"{GOLDEN.get(name, name)}.npz"
    if not p.exists():
        return None
    with np.load(p) as z:
        return {k: z[k] for k in z.files}


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _max_over_ranks(x: float, ws: int, dev) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args):
    """The reference's CPU path (float64 oracle port) on a bounded k sample."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    import torch
    from gradwave_b200.cells import make_cell
    from oracle.davidson import davidson_batched
    from oracle.ham import OracleHamiltonian
    threads = os.cpu_count() or 1
    os.environ.setdefault("GWB_ORACLE_THREADS", str(threads))
    torch.set_num_threads(threads)
    ci = make_cell(args.config)
    nk = ci.bk.nk
    ks = list(range(nk)) if nk <= 2 else [0, nk // 2]
    bk = ci.bk
    h = OracleHamiltonian(bk.mask.numpy()[ks], bk.flat_idx.numpy()[ks], bk.t.numpy()[ks], ci.shape,
                          ci.v_eff_r.numpy(), ci.p.numpy()[ks], bk.dij_full.numpy())
    x0 = ci.identity_start().numpy()[ks]

    def step():
        t0 = time.perf_counter()
        r = davidson_batched(h.apply, x0, bk.t.numpy()[ks], bk.mask.numpy()[ks], tol=args.tol, max_iter=300)
        return (time.perf_counter() - t0) * 1e3 * nk / len(ks), r

    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        ms, r = step()
        times.append(ms)
    v = statistics.mean(times)
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "ms", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(v, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128/f64", "data": "synthetic (seeded Si cells)",
            "config": {"workload": args.config, "nk": nk, "nbands": ci.nbands, "fft": list(ci.shape),
                       "tol_ev": args.tol, "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": round(v, 3), "unit": "ms", "cores": threads, "kind": "port", "cpu": _cpu_model(),
                             "sample": f"k-points {ks} of {nk} solved to tol {args.tol} eV, time scaled "
                                       f"by {nk}/{len(ks)}; float64 numpy/scipy restatement of the "
                                       "reference's davidson_batched + BatchedHamiltonian.apply"},
            "e2e": {"value": round(v, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "n_iter": int(r.n_iter)}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    from gradwave_b200 import _lib
    from gradwave_b200.cells import make_cell
    from gradwave_b200.davidson import davidson_batched
    from gradwave_b200.hamiltonian import BatchedHamiltonian

    ws, rank, local = _dist()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local if ws > 1 else 0)
    torch.cuda.set_device(dev)
    ci = make_cell(args.config)
    bk = ci.bk.to(dev)
    h = BatchedHamiltonian(bk, ci.shape, ci.v_eff_r, ci.p)
    gold = _golden(args.config)
    x0_host = ci.identity_start().pin_memory()
    x0_dev = x0_host.to(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    fast_mode, fast_pc = _solver_choice(args.solver, dev)

    def solve(x0, mode, pc="teter"):
        return davidson_batched(h.apply, x0, bk.t, bk.mask, tol=args.tol, max_iter=300, mode=mode, precond=pc)

    def check(res):
        if gold is None:
            return None
        err = float(np.abs(res.eigenvalues.cpu().numpy() - gold["eigenvalues"]).max())
        if err > EIG_TOL_EV:
            raise SystemExit(f"eigenvalue error {err:.3e} eV exceeds 1e-8 Ha")
        return err

    def timed(fn, steps, warmup, clocks=None):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(dev)
        ts = []
        out = None
        for _ in range(steps):
            flush.zero_()
            if ws > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            out = fn()
            e1.record()
            torch.cuda.synchronize(dev)
            ts.append(e0.elapsed_time(e1))
        return statistics.mean(ts), out

    # value: device-resident inputs; every H apply inside the timed native
    # solves is bracketed by CUDA events on the solve stream (GWB_TIME_APPLIES)
    n0 = _lib.launch_count()
    os.environ["GWB_TIME_APPLIES"] = "1"
    with ClockSampler(dev.index) as clk:
        for _ in range(args.warmup):
            solve(x0_dev, fast_mode, fast_pc)
        n1 = _lib.launch_count()
        ms_fast, res_fast = timed(lambda: solve(x0_dev, fast_mode, fast_pc), args.steps, 0)
        launches = (_lib.launch_count() - n1) // max(1, args.steps)
    os.environ["GWB_TIME_APPLIES"] = "0"
    err_fast = check(res_fast)
    # plain float64 TPA Davidson on the same GPU
    ms_plain, res_plain = timed(lambda: solve(x0_dev, "fp64"), max(1, args.steps // 2), 1)
    err_plain = check(res_plain)

    # e2e through the public API from pinned host memory
    def e2e():
        x0 = x0_host.to(dev, non_blocking=True)
        r = solve(x0, fast_mode, fast_pc)
        ev = r.eigenvalues.to("cpu", non_blocking=True)
        vec = r.eigenvectors.to("cpu", non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        return ev, vec
    ms_e2e, (ev, vec) = timed(e2e, args.steps, 1)

    ms_fast = _max_over_ranks(ms_fast, ws, dev)
    ms_e2e = _max_over_ranks(ms_e2e, ws, dev)
    ms_plain = _max_over_ranks(ms_plain, ws, dev)
    if ws > 1:
        # each rank's solve is the k-shard [rank*nk, (rank+1)*nk) of an N-fold
        # k-set (weak scaling); one all-gather, outside the timed region,
        # assembles the global eigenvalues in k order
        from gradwave_b200.sharding import gather_cat
        eig_all = gather_cat(res_fast.eigenvalues.contiguous(), ws)
        if tuple(eig_all.shape) != (ws * res_fast.eigenvalues.shape[0], res_fast.eigenvalues.shape[1]):
            raise RuntimeError(f"gathered eigenvalues have shape {tuple(eig_all.shape)}")

    # roofline of the H apply (the path's bandwidth kernel) from the last timed solve
    hbm_peak, peak_kind = _peaks()
    info = res_fast.info
    n_calls = int(info.get("n_apply_calls", 0))
    apply_ms = float(info.get("apply_ms", 0.0))
    units = res_fast.n_apply_low + res_fast.n_apply_full          # band*k applied
    nk = ci.bk.nk
    npw = ci.bk.npw.numpy().astype(np.float64)
    n_box = float(np.prod(ci.shape))
    nproj = int(ci.p.shape[1])
    mean_npw = float(npw.mean())
    # algorithmic bytes (per band*k: 16 npw + 32 N; per launch: 4 N for v(r)
    # and the projectors read twice, 16 nk nproj npw)
    bytes_per_unit = 16.0 * mean_npw + 32.0 * n_box
    per_launch = 4.0 * n_box + 16.0 * nk * nproj * mean_npw
    alg_bytes = units * bytes_per_unit + n_calls * per_launch
    achieved = alg_bytes / (apply_ms * 1e-3) / 1e9 if apply_ms > 0 else 0.0
    roof = {"kernel": "gwb_ham_apply (plane_inverse + pencil_vloc + plane_forward + becp + nl_add)",
            "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
            "frac": round(achieved / hbm_peak, 4), "peak_kind": peak_kind, "traffic": None,
            "launches": n_calls, "avg_launch_ms": round(apply_ms / max(1, n_calls), 4),
            "share_of_step": round(apply_ms / max(1e-9, ms_fast), 4),
            "bytes_per_unit": bytes_per_unit, "units_per_step": int(units)}
    summary = ROOT / "profiles" / f"gwb_ham_apply_{args.config}.md"
    if summary.exists():
        import re
        m = re.search(r"dram_bytes_per_band_k:\s*([0-9.eE+]+)", summary.read_text())
        if m and n_calls:
            roof["traffic"] = round(float(m.group(1)) * units / n_calls)

    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = _cpu_baseline(args, ci)
    largest = None
    if rank == 0 and ws == 1 and not args.no_largest:
        largest = _largest_config(dev)
    if ws > 1:
        torch.distributed.barrier()
    if rank == 0:
        n_vec = vec.numel() * vec.element_size()
        line = {"metric": METRIC, "value": round(ms_fast / ws, 3), "unit": "ms", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_fast, 3),
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "c128/f64 basis; f32 expansion applies, f64 certify; bf16 network",
                "data": "synthetic (seeded Si cells, analytic pseudopotential)",
                "config": {"workload": args.config, "nk": nk, "nbands": ci.nbands, "fft": list(ci.shape),
                           "npw": [int(n) for n in ci.bk.npw], "tol_ev": args.tol,
                           "l2": "flushed (256 MiB write) between timed steps", "parallelism": f"kshard{ws}" if ws > 1 else "single"},
                "eig_err_ev": err_fast, "eig_err_ha": None if err_fast is None else err_fast / HA,
                "solver": args.solver, "n_iter": res_fast.n_iter, "n_apply_low": res_fast.n_apply_low,
                "n_apply_full": res_fast.n_apply_full,
                "plain_fp64": {"value": round(ms_plain, 3), "unit": "ms", "n_iter": res_plain.n_iter,
                               "eig_err_ev": err_plain},
                "e2e": {"value": round(ms_e2e / ws, 3), "unit": "ms", "h2d_bytes_per_step": int(x0_host.numel() * 16),
                        "d2h_bytes_per_step": int(ev.numel() * 8 + n_vec)},
                "gpu_launches": int(launches), "roofline": roof, "clocks": clk.summary(),
                "eigh_note": "subspace eigensolver is latency bound (one CTA per k); see profiles/",
                "cpu_baseline": cpu}
        if largest is not None:
            line["largest_config"] = largest
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def _largest_config(dev, name: str = "si216_vacancy") -> dict:
    """The largest configuration (216 atoms, Gamma only, 480 bands) solved to
    1e-10 eV by the fastest form (Gamma real path, mixed schedule, locking of
    converged pairs, 32 buffer bands) and by the plain float64 complex TPA
    Davidson (the reference's algorithm) on this GPU: one untimed and one
    wall-timed solve each, CUDA-synchronised on both sides (the host driver
    runs on more than one stream), eigenvalue error against the reference's
    golden eigenvalues. A failure is reported in the result, not raised."""
    import torch
    from gradwave_b200.cells import make_cell
    from gradwave_b200.davidson import davidson_batched
    from gradwave_b200.gamma import GammaHamiltonian, build_gamma_basis, davidson_gamma, gamma_start
    from gradwave_b200.hamiltonian import BatchedHamiltonian
    out: dict = {"workload": name, "tol_ev": 1e-10, "timing": "wall, one warm-up solve, CUDA-synchronised"}
    try:
        ci = make_cell(name)
        gold = _golden(name)

        def wall(fn):
            fn()
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            r = fn()
            torch.cuda.synchronize(dev)
            return (time.perf_counter() - t0) * 1e3, r

        def err_ha(eig):
            if gold is None:
                return None
            return float(np.abs(np.asarray(eig).reshape(-1) - gold["eigenvalues"].reshape(-1)).max()) / HA

        gb = build_gamma_basis(ci.spheres[0], ci.shape)
        gh = GammaHamiltonian(gb, ci.v_eff_r, ci.p[0], ci.bk.dij_full, device=dev)
        x0g = gamma_start(gb, ci.nbands, dev)
        ms_g, rg = wall(lambda: davidson_gamma(gh, x0g, tol=1e-10, max_iter=300, mode="mixed", n_buffer=32))
        out["gamma_mixed"] = {"value": round(ms_g, 1), "unit": "ms", "n_iter": rg.n_iter,
                              "max_residual_ev": float(rg.residual_norms.max()),
                              "eig_err_ha": err_ha(rg.eigenvalues.cpu().numpy()),
                              "form": "Gamma real path, float32 expansion applies with float64 certification "
                                      "and polish, locking, 32 buffer bands, TPA"}
        del gh, rg
        torch.cuda.empty_cache()
        bk = ci.bk.to(dev)
        h = BatchedHamiltonian(bk, ci.shape, ci.v_eff_r, ci.p)
        x0 = ci.identity_start().to(dev)
        ms_p, rp = wall(lambda: davidson_batched(h.apply, x0, bk.t, bk.mask, tol=1e-10, max_iter=300, mode="fp64",
                                                 precond="teter"))
        out["plain_fp64"] = {"value": round(ms_p, 1), "unit": "ms", "n_iter": rp.n_iter,
                             "max_residual_ev": float(rp.residual_norms.max()),
                             "eig_err_ha": err_ha(rp.eigenvalues.cpu().numpy()),
                             "form": "complex float64 block Davidson, TPA"}
        out["speedup"] = round(ms_p / ms_g, 3)
        del h, bk, rp
        torch.cuda.empty_cache()
    except Exception as e:  # reported, so that the headline line still prints
        out["error"] = f"{type(e).__name__}: {e}"
    return out


def _cpu_model() -> str:
    """The host CPU's model name (``/proc/cpuinfo``), or the platform string."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or platform.machine()


def _cpu_baseline(args, ci):
    """Oracle (float64 numpy) on a bounded sample: two k-points of the workload."""
    import torch
    from oracle.davidson import davidson_batched
    from oracle.ham import OracleHamiltonian
    threads = os.cpu_count() or 1
    os.environ.setdefault("GWB_ORACLE_THREADS", str(threads))
    torch.set_num_threads(threads)
    bk = ci.bk
    nk = bk.nk
    ks = list(range(nk)) if nk <= 2 else [0, nk // 2]
    h = OracleHamiltonian(bk.mask.numpy()[ks], bk.flat_idx.numpy()[ks], bk.t.numpy()[ks], ci.shape,
                          ci.v_eff_r.numpy(), ci.p.numpy()[ks], bk.dij_full.numpy())
    t0 = time.perf_counter()
    davidson_batched(h.apply, ci.identity_start().numpy()[ks], bk.t.numpy()[ks], bk.mask.numpy()[ks],
                     tol=args.tol, max_iter=300)
    dt = (time.perf_counter() - t0) * 1e3 * nk / len(ks)
    return {"value": round(dt, 1), "unit": "ms", "cores": threads, "kind": "port", "cpu": _cpu_model(),
            "sample": f"k-points {ks} of {nk} solved to tol {args.tol} eV with the float64 oracle, "
                      f"time scaled by {nk}/{len(ks)}"}


def run_apply(args):
    """Apply-only loop (for profiling the Hamiltonian kernels under ncu): K
    applies of the full band block of the workload, float32 or float64."""
    import torch
    from gradwave_b200.cells import make_cell
    from gradwave_b200.hamiltonian import BatchedHamiltonian
    dev = torch.device("cuda", 0)
    ci = make_cell(args.config)
    h = BatchedHamiltonian(ci.bk.to(dev), ci.shape, ci.v_eff_r, ci.p)
    g = torch.Generator().manual_seed(1)
    c = torch.randn(ci.bk.nk, ci.nbands, ci.bk.npw_max, dtype=torch.complex128, generator=g)
    c = (c * ci.bk.mask[:, None, :]).to(dev)
    fn = h.apply_fp32 if args.prec == "fp32" else h.apply
    for _ in range(args.warmup):
        fn(c)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        fn(c)
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"mode": "apply", "config": args.config, "prec": args.prec, "nk": ci.bk.nk,
                      "nbands": ci.nbands, "ms_per_apply": e0.elapsed_time(e1) / args.steps}), flush=True)
    return 0


def run_once(args):
    """``--warmup`` untimed and one wall-timed solve of the workload (for ncu
    launch lists and the larger cells): rounds, applies, eigenvalue and band
    energy error against the reference's golden eigenvalues, and with
    GWB_PROFILE=1 the per-phase CUDA-event times of the host driver."""
    import torch
    from gradwave_b200.cells import make_cell
    from gradwave_b200.davidson import davidson_batched
    from gradwave_b200.hamiltonian import BatchedHamiltonian
    dev = torch.device("cuda", 0)
    ci = make_cell(args.config)
    bk = ci.bk.to(dev)
    h = BatchedHamiltonian(bk, ci.shape, ci.v_eff_r, ci.p)
    x0 = ci.identity_start().to(dev)
    mode, pc = _solver_choice(args.solver, dev)
    for _ in range(args.warmup):
        davidson_batched(h.apply, x0, bk.t, bk.mask, tol=args.tol, max_iter=300, mode=mode, precond=pc)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=args.tol, max_iter=300, mode=mode, precond=pc)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) * 1e3
    out = {"mode": "once", "config": args.config, "solver": args.solver, "n_iter": r.n_iter, "wall_ms": wall,
           "n_apply_low": r.n_apply_low, "n_apply_full": r.n_apply_full,
           "max_residual_ev": float(r.residual_norms.max())}
    for key in ("native", "k_groups", "tc_projection", "n_tc_fallback", "phase_ms"):
        if key in r.info:
            out[key] = r.info[key]
    gold = _golden(args.config)
    if gold is not None:
        eig = r.eigenvalues.cpu().numpy()
        err = float(np.abs(eig - gold["eigenvalues"]).max())
        nocc = ci.nocc()
        w = np.asarray(ci.kweights)
        be = 2.0 * float(np.sum(w[:, None] * (eig[:, :nocc] - gold["eigenvalues"][:, :nocc])))
        out.update({"eig_err_ha": err / HA, "band_energy_err_ha": abs(be) / HA, "within_1e-8_ha": err <= EIG_TOL_EV})
    print(json.dumps(out), flush=True)
    return 0


def run_tc(args):
    """The split-BF16 tensor-core products at one Davidson shape: nk batches of
    D (n x npw) against a basis V (m x npw): C = D V^H (A B^H, split-K) and
    D -= C V (A B), each ``--warmup`` untimed and ``--steps`` timed calls
    (CUDA events), next to cuBLAS ZGEMM on the same operands, with the error
    against the float64 product relative to sum_k |d||v|."""
    import torch
    from gradwave_b200.tc import OP_H, OP_N, PlaneSet, check_status, zgemm_tc
    dev = torch.device("cuda", 0)
    nk, n, m, npw = (int(v) for v in args.tc_shape.split(","))
    g = torch.Generator(device="cpu").manual_seed(0)
    D = torch.randn(nk, n, npw, dtype=torch.complex128, generator=g).to(dev)
    V = torch.randn(nk, m, npw, dtype=torch.complex128, generator=g).to(dev)
    pd, pv, pc = PlaneSet(nk, n, npw, dev), PlaneSet(nk, m, npw, dev), PlaneSet(nk, n, m, dev)
    C = torch.zeros(nk, n, m, dtype=torch.complex128, device=dev)
    D2 = D.clone()

    def ev(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / max(args.steps, 1)

    t_planes = ev(lambda: (pd.write(D, n), pv.write(V, m)))
    t_nh = ev(lambda: zgemm_tc(OP_H, n, m, npw, pd, pv, C, m, n * m))
    pc.write(C, n)
    t_nn = ev(lambda: zgemm_tc(OP_N, n, npw, m, pc, pv, D2, npw, n * npw, alpha=-1.0, beta=1.0))
    torch.cuda.synchronize()
    check_status(dev)
    ref = D @ V.conj().transpose(-1, -2)
    err = float(((C - ref).abs() / (D.abs() @ V.abs().transpose(-1, -2))).max())
    t_z_nh = ev(lambda: torch.matmul(D, V.conj().transpose(-1, -2), out=ref))
    t_z_nn = ev(lambda: torch.baddbmm(D, C, V, beta=1.0, alpha=-1.0))
    flop = 8.0 * nk * n * m * npw  # complex multiply-adds x 8
    print(json.dumps({"mode": "tc", "shape": {"nk": nk, "n": n, "m": m, "npw": npw}, "planes_ms": t_planes,
                      "a_bh_ms": t_nh, "a_b_ms": t_nn, "zgemm_a_bh_ms": t_z_nh, "zgemm_a_b_ms": t_z_nn,
                      "a_bh_tflops_equiv": flop / t_nh / 1e9, "a_b_tflops_equiv": flop / t_nn / 1e9,
                      "bf16_tflops_issued_a_bh": 3.0 * flop / t_nh / 1e9, "rel_err": err}), flush=True)
    return 0


def run_gamma(args):
    """The Gamma real path on a Gamma-only cell: ``--warmup`` untimed and one
    wall-timed ``davidson_gamma`` from the identity start on the lowest
    half-sphere slots, to ``--tol``; eigenvalue error against the reference's
    complex float64 golden eigenvalues."""
    import torch
    from gradwave_b200.cells import make_cell
    from gradwave_b200.gamma import GammaHamiltonian, build_gamma_basis, davidson_gamma, gamma_start
    dev = torch.device("cuda", 0)
    ci = make_cell(args.config)
    if ci.bk.nk != 1 or np.any(ci.kpoints != 0):
        raise SystemExit(f"{args.config} is not a Gamma-only cell")
    gb = build_gamma_basis(ci.spheres[0], ci.shape)
    gh = GammaHamiltonian(gb, ci.v_eff_r, ci.p[0], ci.bk.dij_full, device=dev)
    x0 = gamma_start(gb, ci.nbands, dev)
    mode = "mixed" if args.solver in ("mixed", "fp32exp", "learned-mixed") else "fp64"
    lock = {"auto": None, "on": True, "off": False}[args.lock]
    kw = dict(tol=args.tol, max_iter=300, mode=mode, max_dim_factor=args.max_dim_factor, lock=lock,
              n_buffer=args.n_buffer)
    for _ in range(args.warmup):
        davidson_gamma(gh, x0, **kw)
    torch.cuda.synchronize()
    n0 = gh.n_apply
    t0 = time.perf_counter()
    r = davidson_gamma(gh, x0, **kw)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) * 1e3
    out = {"mode": "gamma", "config": args.config, "solver": mode, "max_dim_factor": args.max_dim_factor,
           "lock": (mode == "mixed") if lock is None else lock, "n_buffer": args.n_buffer,
           "tol_ev": args.tol, "n_iter": r.n_iter,
           "wall_ms": wall,
           "band_applies": gh.n_apply - n0, "max_residual_ev": float(r.residual_norms.max()),
           "nhalf": gb.nhalf, "npw": gb.npw}
    if r.phase_ms:
        out["phase_ms"] = r.phase_ms
    gold = _golden(args.config)
    if gold is not None:
        err = float(np.abs(r.eigenvalues.cpu().numpy() - gold["eigenvalues"][0]).max())
        out.update({"eig_err_ha": err / HA, "within_1e-8_ha": err <= EIG_TOL_EV})
    print(json.dumps(out), flush=True)
    return 0


def _solver_choice(name, dev):
    """(mode, preconditioner) of a solver name: plain = float64 + TPA,
    fp32exp = the reference's float32-expansion mode + TPA, mixed = float32
    expansion with near-floor stall rule + TPA, learned-mixed = mixed with the
    learned preconditioner (TPA when no weights are present)."""
    from gradwave_b200 import learned
    if name == "plain":
        return "fp64", "teter"
    if name == "fp32exp":
        return "fp32exp", "teter"
    if name == "mixed":
        return "mixed", "teter"
    if name == "learned-mixed":
        pc = learned.LearnedPreconditioner.load(device=dev) if learned.available() else "teter"
        return "mixed", pc
    raise ValueError(f"unknown solver {name!r}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="si8_cubic")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-largest", action="store_true",
                    help="skip the largest configuration (si216 Gamma mixed vs plain float64) in the solve line")
    ap.add_argument("--tc-shape", default="4,160,640,37000", help="--mode tc: nk,n,m,npw")
    ap.add_argument("--max-dim-factor", type=int, default=4, help="--mode gamma: basis size / bands")
    ap.add_argument("--lock", default="auto", choices=["auto", "on", "off"],
                    help="--mode gamma: lock converged pairs (auto: on in the mixed mode)")
    ap.add_argument("--n-buffer", type=int, default=0, help="--mode gamma: buffer bands above the wanted ones")
    ap.add_argument("--mode", default="solve", choices=["solve", "apply", "once", "tc", "gamma"],
                    help="apply: only time Hamiltonian applies; once: a single solve (profiling)")
    ap.add_argument("--prec", default="fp32", choices=["fp32", "fp64"], help="arithmetic of --mode apply")
    ap.add_argument("--solver", default="learned-mixed", choices=["plain", "fp32exp", "mixed", "learned-mixed"],
                    help="solver of the timed value (the plain float64 solver is always timed beside it)")
    args = ap.parse_args()
    if args.mode == "apply":
        return run_apply(args)
    if args.mode == "tc":
        return run_tc(args)
    if args.mode == "gamma":
        return run_gamma(args)
    if args.mode == "once":
        return run_once(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
