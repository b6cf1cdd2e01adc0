"""Benchmark: ms per converged band solve on one B200 (eigenvalues within
1e-8 Ha of the float64 reference).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME] [--impl ours|reference]

A step is one converged band solve of the workload from the identity start,
to residual 1e-10 eV (every eigenvalue then lies within 1e-8 Ha of the float64
golden eigenvalues; the run checks it). The default workload is the largest
configuration, ``si216_vacancy``: the 216-atom Si supercell at 30 Ry, Gamma
only, 96^3 box, 80,797 plane waves, 480 bands, local potential perturbed by
seeded Gaussian vacancies. Our arm reports:

* ``value``       device-timed ms per solve with the inputs resident in HBM
                  (CUDA events on the launching stream, max over ranks) of the
                  product's fast form (``--solver``, default learned-mixed):
                  on a Gamma-only cell the real (half-sphere) path with the
                  learned preconditioner, float32 expansion applies, float64
                  certification and polish, locking and buffer bands; on a
                  multi-k cell the batched complex solver in its mixed mode
                  with the learned preconditioner;
* ``e2e``         the same solve through the public API from pinned host
                  memory: H2D of the start block, solve, D2H of eigenvalues and
                  eigenvectors, all inside the timed region;
* ``plain_fp64``  the plain float64 TPA block Davidson (the reference's
                  algorithm, complex, all steps float64) on the same GPU;
* ``roofline``    for the Hamiltonian apply (the path's bandwidth kernel),
                  measured live with CUDA events around its launches;
* ``cpu_baseline`` the float64 oracle (numpy restatement of the reference's
                  solver) on the host cores: a few Davidson rounds of the same
                  workload, at all host threads and at the reference's
                  default min(cores, 8);
* ``secondary``   the 8-atom, 10-k cell (si8_cubic) with the native one-call
                  solver, device-timed, next to its plain float64 solve.

Between timed steps a 256 MiB buffer is written to flush L2 (126 MB); the
si216 basis (2 GB) is larger than L2 anyway.

With N > 1 (torchrun): a multi-k workload is split into contiguous k-ranges
balanced by plane-wave count, one per rank (no collective inside the solve,
eigenvalues all-gathered after the timed region), and ``value`` is the max
over ranks of the time of the whole workload (strong scaling). A Gamma-only
workload has a single k-point and does not shard: every rank solves its own
replica, and ``value`` is the max over ranks divided by N (replicas, weak
scaling).

``--impl reference`` times the reference's algorithm on the host cores: the
float64 oracle port (the reference is Python and does not travel; its own
per-round times, recorded in ``tests/golden/reference_rounds.json``, are
reported beside). Each step is one Davidson round of the full workload's own
trajectory from the identity start; the trajectory restarts once every
eigenvalue is within 1e-8 Ha of the golden eigenvalues. ``ms_per_step`` is
the mean timed round; ``value`` is the measured time of one whole trajectory
(every round of one solve timed), or, when the run holds fewer rounds than
a solve, the mean round times the reference's own round count.
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
# buffer bands of the Gamma headline form (measured on si216: 16 gives the
# least time with the learned preconditioner)
GAMMA_BUFFERS = 16
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


def _is_gamma(ci) -> bool:
    return ci.bk.nk == 1 and bool(np.all(np.asarray(ci.kpoints) == 0))


def _reference_rounds(name: str) -> dict | None:
    """The reference's own solve of the cell, recorded in this repository by
    ``tests/golden/reference_rounds.py``: rounds to every eigenvalue within
    1e-8 Ha of the golden ones and their CPU times."""
    p = ROOT / "tests" / "golden" / "reference_rounds.json"
    if not p.exists():
        return None
    rec = json.loads(p.read_text()).get(name)
    if rec is None:
        return None
    return {"rounds": rec["rounds"], "seconds": round(rec["total_seconds"], 2), "threads": rec["threads"],
            "cpu": rec["cpu"], "converged": rec["converged_to_1e-8_ha"]}


class _OracleThreads:
    """Thread count of the oracle: numpy's BLAS pool and scipy.fft workers."""

    def __init__(self, n: int):
        self.n = n

    def __enter__(self):
        from threadpoolctl import threadpool_limits
        self.prev = os.environ.get("GWB_ORACLE_THREADS")
        os.environ["GWB_ORACLE_THREADS"] = str(self.n)
        self.lim = threadpool_limits(limits=self.n)
        return self

    def __exit__(self, *a):
        self.lim.restore_original_limits()
        if self.prev is None:
            os.environ.pop("GWB_ORACLE_THREADS", None)
        else:
            os.environ["GWB_ORACLE_THREADS"] = self.prev


def _oracle_round_times(ci, tol: float, gold_eig):
    """Endless stream of ``(ms, round, eig_err_ev, trajectory)``: the float64
    oracle's block Davidson (the reference's algorithm) on the full workload
    from the identity start, timed round by round (the first round includes
    the start block's orthonormalisation and apply). A trajectory ends once
    every eigenvalue is within 1e-8 Ha of ``gold_eig`` (or the solver stops)
    and the next one starts from the identity again."""
    from oracle.davidson import davidson_rounds
    from oracle.ham import from_cell
    h = from_cell(ci)
    x0 = ci.identity_start().numpy()
    t, mask = ci.bk.t.numpy(), ci.bk.mask.numpy()
    traj = 0
    while True:
        gen = davidson_rounds(h.apply, x0, t, mask, tol=tol, max_iter=300)
        while True:
            t0 = time.perf_counter()
            try:
                it, eig, _ = next(gen)
            except StopIteration:
                break
            ms = (time.perf_counter() - t0) * 1e3
            err = float(np.abs(eig - gold_eig).max()) if gold_eig is not None else float("nan")
            yield ms, it, err, traj
            if err <= EIG_TOL_EV:
                break
        traj += 1


REF_SRC = ROOT / "baseline" / "_ref" / "gradwave"


def _reference_import():
    """The reference package staged under ``baseline/_ref/gradwave`` (a copy
    of its ``src/gradwave``), imported through a namespace shim that skips
    its ``__init__`` (which needs the absent ``ase``); False when it is not
    staged."""
    import types
    if not REF_SRC.is_dir():
        return False
    if "gradwave" not in sys.modules:
        mod = types.ModuleType("gradwave")
        mod.__path__ = [str(REF_SRC)]
        sys.modules["gradwave"] = mod
    return True


def _reference_setup(name, dev):
    """The cell ``name`` built by the reference's own builders on ``dev``:
    (cell inputs, BatchedK, BatchedHamiltonian)."""
    import torch
    from gradwave.core.batch import BatchedHamiltonian, build_batched, projectors_b
    from gradwave.core.hamiltonian import build_projector_data
    from gradwave.grids import build_fft_grid, build_gsphere

    from gradwave_b200.cells import _SPEC, make_cell
    ci = make_cell(name)
    grid = build_fft_grid(ci.cell, ci.ecut, shape_override=ci.shape)
    sph = [build_gsphere(grid, ci.ecut, k) for k in ci.kpoints]
    sp = _SPEC["species"]["Si"]
    rc = float(sp["rc"])
    pds = []
    for s in sph:
        q = torch.sqrt(s.kpg2)
        tab = torch.stack([torch.exp(-0.5 * (q * rc) ** 2), q * rc * torch.exp(-0.5 * (q * rc) ** 2)])
        pds.append(build_projector_data(s, [0] * len(ci.positions), [tab], [[0, 1]],
                                        [torch.diag(torch.tensor(sp["D"], dtype=torch.float64))], grid.volume))
    bk = build_batched(sph, pds, device=dev)
    p = projectors_b(bk, torch.as_tensor(ci.positions).to(dev))
    h = BatchedHamiltonian(bk, grid.shape, torch.as_tensor(ci.v_eff_r).to(dev), p)
    return ci, bk, h


_REF_CPU_SETUP: dict = {}


class _RoundStamps(list):
    """``history_out`` of the reference's ``davidson_batched`` that also
    records the wall time of each append (one per round, after its
    Rayleigh-Ritz step)."""

    def __init__(self):
        super().__init__()
        self.times = []

    def append(self, item):
        self.times.append(time.perf_counter())
        super().append(item)


def _reference_own_rounds(name, tol, gold_eig, n_rounds, threads):
    """``n_rounds`` Davidson rounds of the reference's own ``davidson_batched``
    (complex float64, TPA, torch on the host cores with ``threads``
    threads) on the cell, from the identity start; a trajectory that reaches
    every eigenvalue within 1e-8 Ha of ``gold_eig`` ends and the next starts
    from the identity again. Returns [(ms, round, eig_err_ev, trajectory)]."""
    import torch
    from gradwave.solvers.davidson import davidson_batched
    old = torch.get_num_threads()
    torch.set_num_threads(threads)
    try:
        if name not in _REF_CPU_SETUP:  # built once per process
            _REF_CPU_SETUP[name] = _reference_setup(name, torch.device("cpu"))
        ci, bk, h = _REF_CPU_SETUP[name]
        x0 = ci.identity_start()
        out, traj = [], 0
        while len(out) < n_rounds:
            st = _RoundStamps()
            t0 = time.perf_counter()
            davidson_batched(h.apply, x0, bk.t, bk.mask, tol=tol, max_iter=n_rounds - len(out), history_out=st)
            prev = t0
            for (it, _, eig), t in zip(st, st.times):
                err = float(np.abs(eig.numpy() - gold_eig).max()) if gold_eig is not None else float("nan")
                out.append(((t - prev) * 1e3, int(it), err, traj))
                prev = t
                if err <= EIG_TOL_EV:
                    break
            traj += 1
        return out[:n_rounds]
    finally:
        torch.set_num_threads(old)


def run_reference(args):
    """The reference's own solver on the host cores (all host threads): one
    Davidson round of the full workload per step, from the reference package
    staged under ``baseline/_ref`` (``cpu_baseline.kind`` "reference"), or,
    when it is not staged, from its float64 port in ``oracle/`` ("port")."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    from gradwave_b200.cells import make_cell
    threads = os.cpu_count() or 1
    ci = make_cell(args.config)
    gold = _golden(args.config)
    gold_eig = None if gold is None else gold["eigenvalues"]
    ref = _reference_rounds(args.config)
    own = _reference_import()
    if own:
        rounds = _reference_own_rounds(args.config, args.tol, gold_eig, args.warmup + args.steps, threads)
    else:
        with _OracleThreads(threads):
            stream = _oracle_round_times(ci, args.tol, gold_eig)
            rounds = [next(stream) for _ in range(args.warmup + args.steps)]
    timed = [r[0] for r in rounds[args.warmup:]]
    ms_round = statistics.mean(timed)
    first = [r for r in rounds if r[3] == 0]
    complete = len(first) < len(rounds) or (first and first[-1][2] <= EIG_TOL_EV)
    if complete:
        value, kind = sum(r[0] for r in first), "measured: every round of one whole solve"
        n_rounds = len(first)
    else:
        n_rounds = ref["rounds"] if ref else first[-1][1]
        value, kind = ms_round * n_rounds, f"mean timed round x {n_rounds} rounds (the reference's own count)"
    sample = (f"{args.warmup + args.steps} consecutive Davidson rounds of the full {args.config} workload "
              f"(all {ci.bk.nk} k, {ci.nbands} bands, complex128) from the identity start; a solve ends when every "
              f"eigenvalue is within 1e-8 Ha of the golden eigenvalues; "
              + ("the reference's own davidson_batched + BatchedHamiltonian.apply (torch, CPU)" if own else
                 "float64 numpy/scipy restatement of the reference's davidson_batched + BatchedHamiltonian.apply"))
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": "ms", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_round, 1),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "c128/f64",
            "data": "synthetic (seeded Si cells, analytic pseudopotential)",
            "config": {"workload": args.config, "nk": ci.bk.nk, "nbands": ci.nbands, "fft": list(ci.shape),
                       "npw": [int(n) for n in ci.bk.npw], "tol_ev": args.tol, "l2": "n/a (CPU)",
                       "parallelism": "single"},
            "step": "one Davidson round", "value_kind": kind, "rounds_per_solve": n_rounds,
            "round_ms": [round(r[0], 1) for r in rounds], "round_eig_err_ev": [r[2] for r in rounds],
            "cpu_baseline": {"value": round(value, 1), "unit": "ms", "cores": threads,
                             "kind": "reference" if own else "port", "cpu": _cpu_model(), "sample": sample},
            "reference_own_solve": ref,
            "e2e": {"value": round(value, 1), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _cpu_baseline(args, ci, gold_eig) -> dict:
    """The float64 oracle on a bounded sample of the workload: its first
    ``n`` Davidson rounds, at all host threads and at the reference's default
    min(cores, 8) threads (gradwave ``_threads.py``). ``value`` is the mean
    round times the reference's own round count for this cell."""
    cores = os.cpu_count() or 1
    ref = _reference_rounds(args.config)
    n = 2
    out = {}
    own = _reference_import()
    for label, th in (("all", cores), ("default", min(cores, 8))):
        if own:
            ms = [r[0] for r in _reference_own_rounds(args.config, args.tol, gold_eig, n, th)]
        else:
            with _OracleThreads(th):
                stream = _oracle_round_times(ci, args.tol, gold_eig)
                ms = [next(stream)[0] for _ in range(n)]
        out[label] = (th, statistics.mean(ms))
    n_rounds = ref["rounds"] if ref else None
    per_round = out["all"][1]
    what = ("the reference's own davidson_batched (torch, CPU)" if own
            else "the float64 oracle (a restatement of the reference)")
    return {"value": None if n_rounds is None else round(per_round * n_rounds, 1), "unit": "ms",
            "cores": cores, "kind": "reference" if own else "port", "cpu": _cpu_model(),
            "sample": f"first {n} Davidson rounds of the full workload with {what}; value = mean "
                      f"round x {n_rounds} rounds (the reference's own count to 1e-8 Ha)",
            "ms_per_round": round(per_round, 1),
            "ms_per_round_default_threads": round(out["default"][1], 1),
            "default_threads": out["default"][0],
            "value_default_threads": None if n_rounds is None else round(out["default"][1] * n_rounds, 1),
            "reference_own_solve": ref}


def _timed(fn, steps, warmup, dev, flush, ws):
    """Mean CUDA-event ms of ``steps`` calls after ``warmup`` untimed ones;
    a barrier and a device synchronisation on both sides of every step and
    an L2 flush before it. Returns (mean ms, last output)."""
    import torch
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
        if ws > 1:
            torch.distributed.barrier()
        ts.append(e0.elapsed_time(e1))
    return statistics.mean(ts), out


def run_ours(args):
    import torch
    from gradwave_b200.cells import make_cell

    ws, rank, local = _dist()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local if ws > 1 else 0)
    torch.cuda.set_device(dev)
    ci = make_cell(args.config)
    gold = _golden(args.config)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    if _is_gamma(ci):
        line = _gamma_line(args, ci, gold, dev, flush, ws, rank)
    else:
        line = _kpoint_line(args, ci, gold, dev, flush, ws, rank)
    if rank == 0:
        if not args.no_cpu:
            line["cpu_baseline"] = _cpu_baseline(args, ci, None if gold is None else gold["eigenvalues"])
        if ws == 1 and not args.no_secondary and args.config != "si8_cubic":
            line["secondary"] = _secondary_si8(args, dev, flush)
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def _eig_err(eig, gold) -> float | None:
    if gold is None:
        return None
    err = float(np.abs(np.asarray(eig).reshape(-1) - gold["eigenvalues"].reshape(-1)).max())
    if err > EIG_TOL_EV:
        raise SystemExit(f"eigenvalue error {err:.3e} eV exceeds 1e-8 Ha")
    return err


def _apply_roofline(tm: dict, rows_per_band: float, npw: float, n_box: float, nproj: int, nk: int,
                    ms_step: float, kernel: str, traffic_key: str) -> dict:
    """HBM roofline of the Hamiltonian apply from CUDA-event totals ``tm``
    (calls, ms, bands): algorithmic bytes per complex row 16 npw + 32 N
    (float32 complex sphere row in and out, the dense box streamed once per
    3D FFT), per launch 4 N + 16 nk nproj npw (v(r) and the projectors read
    twice)."""
    hbm_peak, peak_kind = _peaks()
    rows = tm["bands"] * rows_per_band
    bytes_per_row = 16.0 * npw + 32.0 * n_box
    per_launch = 4.0 * n_box + 16.0 * nk * nproj * npw
    alg = rows * bytes_per_row + tm["calls"] * per_launch
    achieved = alg / (tm["ms"] * 1e-3) / 1e9 if tm["ms"] > 0 else 0.0
    roof = {"kernel": kernel, "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
            "frac": round(achieved / hbm_peak, 4), "peak_kind": peak_kind, "traffic": None,
            "launches": tm["calls"], "avg_launch_ms": round(tm["ms"] / max(1, tm["calls"]), 4),
            "share_of_step": round(tm["ms"] / max(1e-9, ms_step), 4),
            "bytes_per_row": bytes_per_row, "fixed_bytes_per_launch": per_launch,
            "alg_bytes_per_launch": round(alg / max(1, tm["calls"])), "rows_per_step": rows}
    # DRAM bytes per complex row of the float32 and float64 applies from the
    # committed ncu capture of the same apply kernels (one whole-block apply
    # of the workload; the figure per row is independent of the block size),
    # times this run's rows of each precision, per launch
    summary = ROOT / "profiles" / f"{traffic_key}.md"
    if summary.exists() and tm["calls"]:
        import re
        txt = summary.read_text()
        m32 = re.search(r"dram_bytes_per_row_fp32:\s*([0-9.eE+]+)", txt)
        m64 = re.search(r"dram_bytes_per_row_fp64:\s*([0-9.eE+]+)", txt)
        if m32 and m64:
            b = (float(m32.group(1)) * tm.get("bands_fp32", 0) + float(m64.group(1)) * tm.get("bands_fp64", 0))
            roof["traffic"] = round(b * rows_per_band / tm["calls"])
            roof["traffic_source"] = (f"profiles/{traffic_key}.md: ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                      "per complex row of each precision, times this run's rows")
    return roof


def _gamma_line(args, ci, gold, dev, flush, ws, rank) -> dict:
    """The Gamma-only workload: davidson_gamma mixed (fast form) against the
    plain complex float64 Davidson on the same GPU."""
    import torch
    from gradwave_b200 import _lib
    from gradwave_b200.davidson import davidson_batched
    from gradwave_b200.gamma import GammaHamiltonian, build_gamma_basis, davidson_gamma, gamma_start
    from gradwave_b200.hamiltonian import BatchedHamiltonian

    gb = build_gamma_basis(ci.spheres[0], ci.shape)
    gh = GammaHamiltonian(gb, ci.v_eff_r, ci.p[0], ci.bk.dij_full, device=dev)
    x0_host = gamma_start(gb, ci.nbands, "cpu").pin_memory()
    x0_dev = x0_host.to(dev)
    nbuf = GAMMA_BUFFERS if args.n_buffer is None else args.n_buffer
    mode, pc = _solver_choice(args.solver, dev)
    mode = "mixed" if mode in ("mixed", "fp32exp") else "fp64"

    def fast(x0):
        return davidson_gamma(gh, x0, tol=args.tol, max_iter=300, mode=mode, n_buffer=nbuf, precond=pc)

    with ClockSampler(dev.index) as clk:
        for _ in range(args.warmup):
            fast(x0_dev)
        torch.cuda.synchronize(dev)
        n1 = _lib.launch_count()
        gh.timing = []

        def step():
            gh.timing = []
            return fast(x0_dev)
        ms_fast, res = _timed(step, args.steps, 0, dev, flush, ws)
        launches = (_lib.launch_count() - n1) // max(1, args.steps)
    tm = gh.apply_times()
    gh.timing = None
    err_fast = _eig_err(res.eigenvalues.cpu().numpy(), gold)

    def e2e():
        x0 = x0_host.to(dev, non_blocking=True)
        r = fast(x0)
        ev = r.eigenvalues.to("cpu", non_blocking=True)
        vec = r.eigenvectors.to("cpu", non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        return ev, vec
    ms_e2e, (ev, vec) = _timed(e2e, args.steps, 1, dev, flush, ws)
    del gh
    torch.cuda.empty_cache()

    # the plain float64 TPA Davidson (complex, the reference's algorithm)
    bk = ci.bk.to(dev)
    h = BatchedHamiltonian(bk, ci.shape, ci.v_eff_r, ci.p)
    x0c = ci.identity_start().to(dev)
    ms_plain, res_p = _timed(lambda: davidson_batched(h.apply, x0c, bk.t, bk.mask, tol=args.tol, max_iter=300,
                                                      mode="fp64", precond="teter"),
                             max(2, args.steps // 5), 1, dev, flush, ws)
    err_plain = _eig_err(res_p.eigenvalues.cpu().numpy(), gold)
    n_iter_plain = res_p.n_iter
    del h, bk, res_p
    torch.cuda.empty_cache()

    ms_fast = _max_over_ranks(ms_fast, ws, dev)
    ms_e2e = _max_over_ranks(ms_e2e, ws, dev)
    ms_plain = _max_over_ranks(ms_plain, ws, dev)
    npw = float(gb.npw)
    roof = _apply_roofline(tm, 0.5, npw, float(np.prod(ci.shape)), int(ci.p.shape[1]), 1, ms_fast,
                           "gwb_gamma_apply (pack + plane_inverse + pencil_vloc + plane_forward + nonlocal + "
                           "unpack; two real bands per complex row)", f"gwb_gamma_apply_{args.config}")
    line = {"metric": METRIC, "value": round(ms_fast / ws, 3), "unit": "ms", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_fast, 3),
            "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64 basis and subspace; f32 expansion applies, f64 certify and polish; bf16x3 tensor-core "
                     "first projection",
            "data": "synthetic (seeded Si cells, analytic pseudopotential)",
            "config": {"workload": args.config, "nk": 1, "nbands": ci.nbands, "fft": list(ci.shape),
                       "npw": [int(gb.npw)], "nhalf": gb.nhalf, "tol_ev": args.tol,
                       "l2": "flushed (256 MiB write) between timed steps; basis 2 GB > L2",
                       "parallelism": f"replicas{ws}" if ws > 1 else "single"},
            "solver": f"gamma-{mode} (locking, {nbuf} buffer bands, "
                      f"{'TPA' if isinstance(pc, str) else 'learned preconditioner'})",
            "n_tpa_fallback": res.n_tpa_fallback,
            "eig_err_ev": err_fast, "eig_err_ha": None if err_fast is None else err_fast / HA,
            "n_iter": res.n_iter, "band_applies": {"fp32": tm["bands_fp32"], "fp64": tm["bands_fp64"]},
            "plain_fp64": {"value": round(ms_plain, 3), "unit": "ms", "n_iter": n_iter_plain,
                           "eig_err_ev": err_plain, "form": "complex float64 block Davidson, TPA"},
            "speedup_vs_plain_fp64": round(ms_plain / ms_fast, 3),
            "e2e": {"value": round(ms_e2e / ws, 3), "unit": "ms", "h2d_bytes_per_step": int(x0_host.numel() * 16),
                    "d2h_bytes_per_step": int(ev.numel() * 8 + vec.numel() * vec.element_size())},
            "gpu_launches": int(launches), "roofline": roof, "clocks": clk.summary()}
    return line


def _kpoint_line(args, ci, gold, dev, flush, ws, rank) -> dict:
    """A multi-k workload: the batched complex solver in the chosen mode
    (default learned + mixed) against the plain float64 solve. With N ranks
    each solves a contiguous k-range balanced by plane-wave count and the
    eigenvalues are all-gathered after the timed region."""
    import torch
    from gradwave_b200 import _lib
    from gradwave_b200.davidson import davidson_batched
    from gradwave_b200.hamiltonian import BatchedHamiltonian
    from gradwave_b200.sharding import gather_cat, shard_range_weighted, slice_batched

    nk_all = ci.bk.nk
    if ws > 1:
        k0, k1 = shard_range_weighted(ci.bk.npw.numpy().astype(float), rank, ws)
    else:
        k0, k1 = 0, nk_all
    bk = slice_batched(ci.bk, k0, k1).to(dev)
    h = BatchedHamiltonian(bk, ci.shape, ci.v_eff_r, ci.p[k0:k1])
    x0_host = ci.identity_start()[k0:k1].contiguous().pin_memory()
    x0_dev = x0_host.to(dev)
    fast_mode, fast_pc = _solver_choice(args.solver, dev)

    def solve(x0, mode, pc="teter"):
        return davidson_batched(h.apply, x0, bk.t, bk.mask, tol=args.tol, max_iter=300, mode=mode, precond=pc)

    os.environ["GWB_TIME_APPLIES"] = "1"
    with ClockSampler(dev.index) as clk:
        for _ in range(args.warmup):
            solve(x0_dev, fast_mode, fast_pc)
        torch.cuda.synchronize(dev)
        n1 = _lib.launch_count()
        ms_fast, res = _timed(lambda: solve(x0_dev, fast_mode, fast_pc), args.steps, 0, dev, flush, ws)
        launches = (_lib.launch_count() - n1) // max(1, args.steps)
    os.environ["GWB_TIME_APPLIES"] = "0"
    ms_plain, res_p = _timed(lambda: solve(x0_dev, "fp64"), max(2, args.steps // 4), 1, dev, flush, ws)

    def e2e():
        x0 = x0_host.to(dev, non_blocking=True)
        r = solve(x0, fast_mode, fast_pc)
        ev = r.eigenvalues.to("cpu", non_blocking=True)
        vec = r.eigenvectors.to("cpu", non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        return ev, vec
    ms_e2e, (ev, vec) = _timed(e2e, args.steps, 1, dev, flush, ws)

    ms_fast = _max_over_ranks(ms_fast, ws, dev)
    ms_e2e = _max_over_ranks(ms_e2e, ws, dev)
    ms_plain = _max_over_ranks(ms_plain, ws, dev)
    eig_fast, eig_plain = res.eigenvalues.contiguous(), res_p.eigenvalues.contiguous()
    if ws > 1:
        # one all-gather, outside the timed region, assembles the global
        # eigenvalues in k order for the check against the golden ones
        eig_fast = gather_cat(eig_fast, ws)
        eig_plain = gather_cat(eig_plain, ws)
    err_fast = _eig_err(eig_fast.cpu().numpy(), gold)
    err_plain = _eig_err(eig_plain.cpu().numpy(), gold)
    info = res.info
    tm = {"calls": int(info.get("n_apply_calls", 0)), "ms": float(info.get("apply_ms", 0.0)),
          "bands": int(res.n_apply_low + res.n_apply_full)}
    npw = float(bk.npw.float().mean())
    roof = _apply_roofline(tm, 1.0, npw, float(np.prod(ci.shape)), int(ci.p.shape[1]), k1 - k0, ms_fast,
                           "gwb_ham_apply (plane_inverse + pencil_vloc + plane_forward + becp + nl_add)",
                           f"gwb_ham_apply_{args.config}")
    return {"metric": METRIC, "value": round(ms_fast, 3), "unit": "ms", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_fast, 3),
            "higher_is_better": False, "scaling": "strong" if ws > 1 else "weak", "vs_baseline": None,
            "dtype": "c128/f64 basis; f32 expansion applies, f64 certify; bf16 network",
            "data": "synthetic (seeded Si cells, analytic pseudopotential)",
            "config": {"workload": args.config, "nk": nk_all, "nbands": ci.nbands, "fft": list(ci.shape),
                       "npw": [int(n) for n in ci.bk.npw], "tol_ev": args.tol,
                       "l2": "flushed (256 MiB write) between timed steps",
                       "parallelism": f"kshard{ws}" if ws > 1 else "single"},
            "eig_err_ev": err_fast, "eig_err_ha": None if err_fast is None else err_fast / HA,
            "solver": args.solver, "n_iter": res.n_iter, "n_apply_low": res.n_apply_low,
            "n_apply_full": res.n_apply_full,
            "plain_fp64": {"value": round(ms_plain, 3), "unit": "ms", "n_iter": res_p.n_iter,
                           "eig_err_ev": err_plain},
            "speedup_vs_plain_fp64": round(ms_plain / ms_fast, 3),
            "e2e": {"value": round(ms_e2e, 3), "unit": "ms", "h2d_bytes_per_step": int(x0_host.numel() * 16),
                    "d2h_bytes_per_step": int(ev.numel() * 8 + vec.numel() * vec.element_size())},
            "gpu_launches": int(launches), "roofline": roof, "clocks": clk.summary()}


def _secondary_si8(args, dev, flush) -> dict:
    """The 8-atom, 10-k cell with the native one-call solver (learned +
    mixed), device-timed over a few solves, next to its plain float64 solve."""
    import torch
    from gradwave_b200.cells import make_cell
    from gradwave_b200.davidson import davidson_batched
    from gradwave_b200.hamiltonian import BatchedHamiltonian
    out: dict = {"workload": "si8_cubic", "tol_ev": args.tol}
    try:
        ci = make_cell("si8_cubic")
        gold = _golden("si8_cubic")
        bk = ci.bk.to(dev)
        h = BatchedHamiltonian(bk, ci.shape, ci.v_eff_r, ci.p)
        x0 = ci.identity_start().to(dev)
        mode, pc = _solver_choice("learned-mixed", dev)
        ms, r = _timed(lambda: davidson_batched(h.apply, x0, bk.t, bk.mask, tol=args.tol, max_iter=300, mode=mode,
                                                precond=pc), 5, 3, dev, flush, 1)
        ms_p, rp = _timed(lambda: davidson_batched(h.apply, x0, bk.t, bk.mask, tol=args.tol, max_iter=300,
                                                   mode="fp64", precond="teter"), 3, 1, dev, flush, 1)
        out.update({"value": round(ms, 3), "unit": "ms", "n_iter": r.n_iter, "solver": "learned-mixed (native)",
                    "eig_err_ev": _eig_err(r.eigenvalues.cpu().numpy(), gold),
                    "plain_fp64": {"value": round(ms_p, 3), "n_iter": rp.n_iter,
                                   "eig_err_ev": _eig_err(rp.eigenvalues.cpu().numpy(), gold)},
                    "reference_own_solve": _reference_rounds("si8_cubic")})
        del h, bk
        torch.cuda.empty_cache()
    except (Exception, SystemExit) as e:  # reported, so that the headline line still prints
        out["error"] = f"{type(e).__name__}: {e}"
    return out


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


def run_apply_gamma(args):
    """Apply-only loop of the Gamma path (for profiling its kernels under
    ncu): K applies of the workload's whole embedded band block (nbands real
    rows, two per complex row of the apply kernels), float32 or float64."""
    import torch
    from gradwave_b200.cells import make_cell
    from gradwave_b200.gamma import GammaHamiltonian, build_gamma_basis
    dev = torch.device("cuda", 0)
    ci = make_cell(args.config)
    gb = build_gamma_basis(ci.spheres[0], ci.shape)
    gh = GammaHamiltonian(gb, ci.v_eff_r, ci.p[0], ci.bk.dij_full, device=dev)
    g = torch.Generator().manual_seed(1)
    phi = torch.randn(ci.nbands, 2 * gb.nhalf - 1, dtype=torch.float64, generator=g).to(dev)
    prec = 0 if args.prec == "fp32" else 1
    for _ in range(args.warmup):
        gh.apply_phi(phi, prec=prec)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        gh.apply_phi(phi, prec=prec)
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"mode": "apply_gamma", "config": args.config, "prec": args.prec, "bands": ci.nbands,
                      "complex_rows": (ci.nbands + 1) // 2, "ms_per_apply": e0.elapsed_time(e1) / args.steps}),
          flush=True)
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


def run_oz(args):
    """Float64 products on the int8 tensor cores next to cuBLAS DGEMM at the
    real Davidson shapes of the 216-atom Gamma cell: A B^T with K = 80,798
    (subspace / projection coefficients, Gram) and A B with K = the basis
    (Ritz vectors, projection update). ``--oz-scheme slices``: the Ozaki
    scheme's first form with ``--slices`` int8 slices; ``crt``: its second
    form with ``--moduli`` residues. ``--warmup`` untimed and ``--steps``
    timed calls each (CUDA events): the whole call (operands split on every
    call) and the product alone on split operands; error against the float64
    product relative to the operands' row maxima times sqrt(K) (``err``) and
    relative to |A||B| (``err_abs_prod``)."""
    import torch
    from gradwave_b200.oz import CrtMatmul, OzMatmul, check_status
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(0)
    npw = 80798
    decay = torch.exp(-torch.linspace(0.0, 8.0, npw, dtype=torch.float64))
    crt = args.oz_scheme == "crt"
    om = CrtMatmul(dev, n=args.moduli) if crt else OzMatmul(dev, s=args.slices)
    n_products = args.moduli if crt else args.slices * (args.slices + 1) // 2
    out = {"mode": "oz", "scheme": args.oz_scheme, "moduli" if crt else "slices": args.moduli if crt else args.slices,
           "int8_products": n_products, "shapes": {}}

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

    for name, (M, N, K, form) in {"nt_512x1920xnpw": (512, 1920, npw, "nt"),
                                  "nt_gram_512x512xnpw": (512, 512, npw, "nt"),
                                  "nn_512xnpwx1920": (512, npw, 1920, "nn")}.items():
        if form == "nt":
            a = (torch.randn(M, K, dtype=torch.float64, generator=g) * decay).to(dev)
            b = (torch.randn(N, K, dtype=torch.float64, generator=g) * decay).to(dev)
            c = torch.empty(M, N, dtype=torch.float64, device=dev)
            t_oz = ev(lambda: om.nt(a, b, c))
            sa, sb = om._set("nt_a", M, K), om._set("nt_b", N, K)
            t_prod = ev(lambda: om.gemm(M, N, K, sa, sb, c))
            ref = a @ b.T
            t_d = ev(lambda: torch.matmul(a, b.T, out=ref))
            sc = a.abs().amax(1)[:, None] * b.abs().amax(1)[None, :] * K ** 0.5
            sabs = a.abs() @ b.abs().T
        else:
            a = torch.randn(M, K, dtype=torch.float64, generator=g).to(dev)
            b = (torch.randn(K, N, dtype=torch.float64, generator=g) * decay[:N]).to(dev)
            c = torch.empty(M, N, dtype=torch.float64, device=dev)
            t_oz = ev(lambda: om.nn(a, b, c))
            sa, sb = om._set("nn_a", M, K), om._set("nn_b", N, K)
            t_prod = ev(lambda: om.gemm(M, N, K, sa, sb, c, b_scaled=False))
            ref = a @ b
            t_d = ev(lambda: torch.matmul(a, b, out=ref))
            sc = a.abs() @ b.abs().amax(1, keepdim=True) + 1e-300
            sabs = a.abs() @ b.abs()
        om.nt(a, b, c) if form == "nt" else om.nn(a, b, c)
        check_status(dev)
        flop = 2.0 * M * N * K
        d = (c - ref).abs()
        out["shapes"][name] = {"M": M, "N": N, "K": K, "oz_ms": round(t_oz, 4), "product_ms": round(t_prod, 4),
                               "dgemm_ms": round(t_d, 4), "speedup": round(t_d / t_oz, 3),
                               "speedup_product": round(t_d / t_prod, 3),
                               "oz_tflops_equiv": round(flop / t_oz / 1e9, 1),
                               "int8_tops_issued": round(flop * n_products / t_prod / 1e9, 1),
                               "err": float((d / sc).max()),
                               "err_abs_prod": float((d / (sabs + 1e-300)).max())}
        del a, b, c, ref, sabs, d
    print(json.dumps(out), flush=True)
    return 0


def run_eigh(args):
    """The subspace eigensolver on random symmetric matrices of the Davidson
    sizes (``--eigh-sizes``; diagonal -5..80 eV plus 0.05 noise, like the
    216-atom subspace matrices): ``gwb_sy_lowest`` (lowest 496) and its
    tridiagonalisation ``gwb_sytrd`` against ``torch.linalg.eigh``
    (cuSOLVER), ``--warmup`` untimed and ``--steps`` timed calls (CUDA
    events); with ``--eigh-trace`` the per-phase cycles of the
    tridiagonalisation (``gwb_sytrd_set_trace``)."""
    import torch
    from gradwave_b200 import _lib
    dev = torch.device("cuda", 0)
    lib = _lib.load()
    for m in (int(x) for x in args.eigh_sizes.split(",")):
        nev = min(m, 496)
        g = torch.Generator().manual_seed(m)
        a = torch.randn(m, m, dtype=torch.float64, generator=g)
        a = (0.5 * (a + a.T) * 0.05 + torch.diag(torch.linspace(-5, 80, m, dtype=torch.float64))).to(dev)
        A = torch.empty_like(a)
        w = torch.empty(nev, dtype=torch.float64, device=dev)
        ut = torch.empty(nev, m, dtype=torch.float64, device=dev)
        wk = torch.empty(int(lib.gwb_sy_lowest_work_bytes(m, nev)), dtype=torch.uint8, device=dev)
        d = torch.empty(m, dtype=torch.float64, device=dev)
        e = torch.empty(m, dtype=torch.float64, device=dev)
        tau = torch.empty(m, dtype=torch.float64, device=dev)
        wt = torch.empty(int(lib.gwb_sytrd_work_bytes(m)), dtype=torch.uint8, device=dev)
        st = torch.zeros(1, dtype=torch.int32, device=dev)
        s = _lib.stream_ptr(dev)

        def own():
            A.copy_(a)
            _lib.call("gwb_sy_lowest", m, nev, A.data_ptr(), m, w.data_ptr(), ut.data_ptr(), m, wk.data_ptr(),
                      wk.numel(), st.data_ptr(), s)

        def trd():
            A.copy_(a)
            _lib.call("gwb_sytrd", m, A.data_ptr(), m, d.data_ptr(), e.data_ptr(), tau.data_ptr(), wt.data_ptr(),
                      wt.numel(), st.data_ptr(), s)

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

        out = {"mode": "eigh", "m": m, "nev": nev, "own_ms": round(ev(own), 3), "sytrd_ms": round(ev(trd), 3),
               "torch_eigh_ms": round(ev(lambda: torch.linalg.eigh(a)), 3)}
        # the cooperative launch alone (no cluster part), for comparison
        _lib.call("gwb_sytrd_set_cluster", 0)
        out["sytrd_coop_only_ms"] = round(ev(trd), 3)
        _lib.call("gwb_sytrd_set_cluster", -1)
        own()
        ref = torch.linalg.eigvalsh(a)[:nev]
        out["eig_err_rel"] = float((w - ref).abs().max() / ref.abs().max())
        if args.eigh_trace:
            # the cooperative launch over all columns, then the default
            # split (its cluster part per cluster column)
            tr = torch.zeros(10, dtype=torch.int64, device=dev)
            _lib.call("gwb_sytrd_set_cluster", 0)
            _lib.call("gwb_sytrd_set_trace", tr.data_ptr())
            trd()
            torch.cuda.synchronize()
            _lib.call("gwb_sytrd_set_cluster", -1)
            tc = torch.zeros(10, dtype=torch.int64, device=dev)
            _lib.call("gwb_sytrd_set_trace", tc.data_ptr())
            trd()
            torch.cuda.synchronize()
            _lib.call("gwb_sytrd_set_trace", None)
            nc = int(lib.gwb_sytrd_cluster_rows(m))
            out["cluster_rows"] = nc
            if nc > 1:
                cn = ["column_and_reflector", "row_pass", "exchange", "cluster_barrier"]
                out["cluster_us_per_column"] = {k: round(v / 1.9e3 / (nc - 1), 3)
                                                for k, v in zip(cn, tc.cpu().tolist()[6:])}
            names = ["reflector", "row_products", "barrier_1", "w_and_next_column", "barrier_2", "trailing_update"]
            out["us_per_column"] = {n: round(c / 1.9e3 / (m - 1), 3) for n, c in zip(names, tr.cpu().tolist()[:6])}
        out["status"] = int(st.item())
        print(json.dumps(out), flush=True)
    return 0


def run_precond(args):
    """The learned preconditioner at the 216-atom Gamma shape (``--precond-rows``
    selected bands of 496, 40,399 half-sphere slots, random rows and
    network): ``gwb_precond_learned_gamma`` on the embedded real rows
    (tcgen05), and the complex-row ``gwb_precond_learned`` on the same rows as
    half-sphere rows with each inference kernel (tcgen05, mma.sync), the
    gather and repacking of the half rows included (the previous Gamma form).
    CUDA events over ``--steps`` calls after ``--warmup``."""
    import torch
    from gradwave_b200 import _lib, learned
    from gradwave_b200.gamma import _embed_rows, _half_rows
    dev = torch.device("cuda", 0)
    lib = _lib.load()
    nb, nhalf, n = 496, 40399, args.precond_rows
    nphi = 2 * nhalf - 1
    npad = nphi + 1
    g = torch.Generator(device="cpu").manual_seed(3)
    x = torch.randn(nb, npad, generator=g, dtype=torch.float64).to(dev)
    r = torch.randn(nb, npad, generator=g, dtype=torch.float64).to(dev)
    x[:, nphi:] = 0.0
    r[:, nphi:] = 0.0
    th = (torch.rand(nhalf, generator=g, dtype=torch.float64) * 60).to(dev)
    eig = torch.randn(nb, generator=g, dtype=torch.float64).to(dev)
    sel = torch.randperm(nb, generator=g)[:n].sort().values.to(torch.int32).to(dev)
    tpa = torch.zeros(nb, dtype=torch.uint8, device=dev)
    P = torch.from_numpy(learned.init_params(1)).to(dev)
    P[-65:] = 0.05 * torch.randn(65, generator=g, dtype=torch.float32).to(dev)
    d = torch.empty(n, npad, dtype=torch.float64, device=dev)
    wk = torch.empty(int(lib.gwb_precond_learned_gamma_work_bytes(n, nhalf)), dtype=torch.uint8, device=dev)
    s = _lib.stream_ptr(dev)

    def gamma_rows():
        _lib.call("gwb_precond_learned_gamma", P.data_ptr(), nb, n, nhalf, npad, x.data_ptr(), npad, r.data_ptr(),
                  npad, th.data_ptr(), eig.data_ptr(), sel.data_ptr(), tpa.data_ptr(), d.data_ptr(), npad,
                  wk.data_ptr(), wk.numel(), s)

    idx = torch.arange(n, dtype=torch.int32, device=dev).reshape(1, n)
    sl = sel.long()

    def half_rows():
        xs, rs = _half_rows(x[sl], nhalf), _half_rows(r[sl], nhalf)
        dd = torch.ops.gwb.precond_apply(xs[None], rs[None], th.reshape(1, -1), idx, eig[sl].reshape(1, n), P,
                                         tpa[sl].reshape(1, n))
        return _embed_rows(dd[0], npad)

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

    out = {"mode": "precond", "rows": n, "nhalf": nhalf, "gamma_rows_ms": round(ev(gamma_rows), 3)}
    ref = half_rows()
    gamma_rows()
    torch.cuda.synchronize()
    out["max_abs_diff_vs_half_rows"] = float((d - ref).abs().max())
    for name, kern in (("half_rows_tcgen05_ms", 1), ("half_rows_mma_sync_ms", 0)):
        _lib.call("gwb_precond_set_kernel", kern)
        out[name] = round(ev(half_rows), 3)
    _lib.call("gwb_precond_set_kernel", 1)
    out["plane_waves_per_s_gamma_rows"] = n * nhalf / (out["gamma_rows_ms"] * 1e-3)
    print(json.dumps(out), flush=True)
    return 0


def run_reference_gpu(args):
    """The reference's own float64 block Davidson on this GPU: its builders,
    ``BatchedHamiltonian`` (torch FFT + einsum nonlocal term) and
    ``davidson_batched`` (TPA, cuSOLVER subspace eigensolves above m = 256),
    all on cuda, imported from the reference package staged under
    ``baseline/_ref/gradwave`` (a copy of its ``src/gradwave``: the package
    cannot be pip-installed here, its build backend is missing from the
    wheelhouse) through a namespace shim that skips its ``__init__`` (which
    needs the absent ``ase``). One untimed solve of si2_fcc (cuFFT plans,
    library handles), then one wall-timed solve of each ``--ref-configs``
    cell from the identity start to ``--tol``, synchronised on both sides;
    eigenvalue error against the golden eigenvalues of the reference's
    converged CPU solve. This is the plain float64 TPA Davidson of the
    reference on the same B200, for comparison with the package's own."""
    import torch
    if not _reference_import():
        print(json.dumps({"mode": "reference_gpu", "unavailable": "the reference package is not staged under "
                          "baseline/_ref/gradwave"}), flush=True)
        return 0
    from gradwave.solvers.davidson import davidson_batched
    dev = torch.device("cuda", 0)

    def solve(name):
        ci, bk, h = _reference_setup(name, dev)
        x0 = ci.identity_start().to(dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=args.tol, max_iter=300)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, res

    solve("si2_fcc")
    for name in args.ref_configs.split(","):
        sec, res = solve(name)
        out = {"mode": "reference_gpu", "config": name, "tol_ev": args.tol, "ms": round(1e3 * sec, 1),
               "n_iter": int(res.n_iter), "form": "the reference's davidson_batched, complex float64, TPA, on cuda",
               "max_residual_ev": float(res.residual_norms.max())}
        try:
            out["eig_err_ev"] = _eig_err(res.eigenvalues.cpu().numpy(), _golden(name))
        except Exception as e:  # reported, so that the timing still prints
            out["eig_err_ev"] = f"{type(e).__name__}: {e}"
        print(json.dumps(out), flush=True)
        del res
        torch.cuda.empty_cache()
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
    _, pc = _solver_choice(args.solver, dev)
    kw = dict(tol=args.tol, max_iter=300, mode=mode, max_dim_factor=args.max_dim_factor, lock=lock,
              n_buffer=args.n_buffer or 0, precond=pc)
    for _ in range(args.warmup):
        davidson_gamma(gh, x0, **kw)
    torch.cuda.synchronize()
    n0 = gh.n_apply
    t0 = time.perf_counter()
    r = davidson_gamma(gh, x0, **kw)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) * 1e3
    out = {"mode": "gamma", "config": args.config, "solver": mode, "max_dim_factor": args.max_dim_factor,
           "lock": (mode == "mixed") if lock is None else lock, "n_buffer": args.n_buffer or 0,
           "tol_ev": args.tol, "n_iter": r.n_iter,
           "wall_ms": wall,
           "band_applies": gh.n_apply - n0, "max_residual_ev": float(r.residual_norms.max()),
           "nhalf": gb.nhalf, "npw": gb.npw, "precond": "teter" if isinstance(pc, str) else "learned",
           "n_tpa_fallback": r.n_tpa_fallback, "oz": os.environ.get("GWB_OZ", "0"), "rounds": r.info}
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
        w = os.environ.get("GWB_PRECOND_WEIGHTS")
        if w:
            return "mixed", learned.LearnedPreconditioner.load(w, device=dev)
        pc = learned.LearnedPreconditioner.load(device=dev) if learned.available() else "teter"
        return "mixed", pc
    raise ValueError(f"unknown solver {name!r}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="si216_vacancy")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the secondary si8_cubic solve in the line of another workload")
    ap.add_argument("--tc-shape", default="4,160,640,37000", help="--mode tc: nk,n,m,npw")
    ap.add_argument("--max-dim-factor", type=int, default=4, help="--mode gamma: basis size / bands")
    ap.add_argument("--lock", default="auto", choices=["auto", "on", "off"],
                    help="--mode gamma: lock converged pairs (auto: on in the mixed mode)")
    ap.add_argument("--n-buffer", type=int, default=None,
                    help="Gamma path: buffer bands above the wanted ones (default 32 in the bench line, 0 in --mode gamma)")
    ap.add_argument("--slices", type=int, default=8, help="--mode oz: int8 slices per float64 operand")
    ap.add_argument("--oz-scheme", default="slices", choices=["slices", "crt"], help="--mode oz: Ozaki scheme form")
    ap.add_argument("--moduli", type=int, default=18, help="--mode oz --oz-scheme crt: residues per operand")
    ap.add_argument("--eigh-sizes", default="993,1488,1984", help="--mode eigh: matrix sizes")
    ap.add_argument("--eigh-trace", action="store_true", help="--mode eigh: per-phase cycles of the tridiagonalisation")
    ap.add_argument("--ref-configs", default="si8_cubic,si216_vacancy",
                    help="--mode reference_gpu: cells for the reference's own solve on the GPU")
    ap.add_argument("--precond-rows", type=int, default=400, help="--mode precond: selected bands")
    ap.add_argument("--mode", default="solve", choices=["solve", "apply", "apply_gamma", "once", "tc", "gamma", "oz", "eigh",
                                                       "precond", "reference_gpu"],
                    help="apply: only time Hamiltonian applies; once: a single solve (profiling)")
    ap.add_argument("--prec", default="fp32", choices=["fp32", "fp64"], help="arithmetic of --mode apply")
    ap.add_argument("--solver", default="learned-mixed", choices=["plain", "fp32exp", "mixed", "learned-mixed"],
                    help="solver of the timed value (the plain float64 solver is always timed beside it)")
    args = ap.parse_args()
    if args.mode == "apply":
        return run_apply(args)
    if args.mode == "apply_gamma":
        return run_apply_gamma(args)
    if args.mode == "tc":
        return run_tc(args)
    if args.mode == "oz":
        return run_oz(args)
    if args.mode == "reference_gpu":
        return run_reference_gpu(args)
    if args.mode == "precond":
        return run_precond(args)
    if args.mode == "eigh":
        return run_eigh(args)
    if args.mode == "gamma":
        return run_gamma(args)
    if args.mode == "once":
        return run_once(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
