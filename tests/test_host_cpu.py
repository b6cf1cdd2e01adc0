"""CPU-side checks: the library loads and exports every entry point the
header declares, the registry contract, host set-up helpers and fail-loud
behaviour without a GPU."""

import re
from pathlib import Path

import numpy as np
import pytest
import torch

ROOT = Path(__file__).resolve().parents[1]


def test_library_exports_every_declared_symbol():
    from gradwave_b200 import _lib
    lib = _lib.load()
    header = (ROOT / "include" / "gwb.h").read_text()
    declared = set(re.findall(r"^\s*(?:int|int32_t|int64_t|const char\*|size_t|unsigned long long)\s+(gwb_\w+)\(", header, re.M))
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), f"libgwb.so does not export {name}"
    assert set(_lib.declared_symbols()) == declared
    assert lib.gwb_version().decode().startswith("gwb")


def test_registry_contract_without_gpu():
    from gradwave_b200 import registry
    assert {"davidson", "davidson_fp32exp", "davidson_mixed"} <= set(registry.available())
    with pytest.raises(ValueError):
        registry.register("davidson", registry.davidson_adapter)
    registry.register("davidson", registry.davidson_adapter, overwrite=True)
    with pytest.raises(ValueError, match="registered"):
        registry.get("lobpcg")


def test_product_path_fails_loudly_without_cuda():
    from gradwave_b200.cells import make_cell
    from gradwave_b200.davidson import davidson_batched
    from gradwave_b200.hamiltonian import BatchedHamiltonian
    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    ci = make_cell("si2_fcc")
    with pytest.raises(RuntimeError, match="CUDA"):
        BatchedHamiltonian(ci.bk, ci.shape, ci.v_eff_r, ci.p)
    with pytest.raises(RuntimeError, match="CPU fallback"):
        davidson_batched(lambda c: c, ci.identity_start(), ci.bk.t, ci.bk.mask)


def test_monkhorst_pack_and_ibz_weights():
    from gradwave_b200.basis import monkhorst_pack
    from gradwave_b200.cells import _ibz_oh
    k, w = monkhorst_pack((4, 4, 4))
    assert len(k) == 36 and abs(w.sum() - 1) < 1e-12
    k, w = _ibz_oh(4)
    assert len(k) == 10 and abs(w.sum() - 1) < 1e-12
    assert sorted(np.round(w * 64).astype(int).tolist()) == sorted([1, 6, 3, 12, 12, 3, 8, 12, 6, 1])


def test_fft_box_and_sphere_conventions():
    from gradwave_b200.basis import build_fft_grid, build_gsphere, good_fft_size
    assert [good_fft_size(n) for n in (23, 25, 41, 83, 107)] == [24, 25, 42, 84, 108]
    cell = np.diag([3.0, 3.5, 4.0])
    grid = build_fft_grid(cell, 200.0)
    sph = build_gsphere(grid, 200.0, (0.1, -0.2, 0.3))
    n0, n1, n2 = grid.shape
    m = sph.miller
    assert np.array_equal(sph.flat_idx, (m[:, 0] % n0) * n1 * n2 + (m[:, 1] % n1) * n2 + (m[:, 2] % n2))
    assert np.all(np.diff(np.round(sph.kpg2, 10)) >= 0)


def test_band_path_and_chunk_rule():
    """The k-path stand-in for ASE's bandpath: special points on the path at
    the labelled indices, segments sampled in proportion to their length,
    monotone coordinate; the reference's chunk rule (at most 24 k, fewer when
    dense boxes would pass 1.5 GB)."""
    from gradwave_b200.bands import chunk_size, k_path
    a = 5.43
    cell = 0.5 * a * np.array([[0.0, 1.0, 1.0], [1.0, 0.0, 1.0], [1.0, 1.0, 0.0]])
    pts = [("L", [0.5, 0.5, 0.5]), ("G", [0.0, 0.0, 0.0]), ("X", [0.5, 0.0, 0.5])]
    k, x, labels = k_path(cell, pts, 31)
    assert k.shape == (31, 3)
    assert [lab for _, lab in labels] == ["L", "G", "X"]
    for (i, _), (_, p) in zip(labels, pts):
        assert np.allclose(k[i], p)
    assert labels[0][0] == 0 and labels[-1][0] == 30
    assert np.all(np.diff(x) > 0)
    recip = 2 * np.pi * np.linalg.inv(cell).T
    seg = [np.linalg.norm((np.array(pts[i + 1][1]) - np.array(pts[i][1])) @ recip) for i in range(2)]
    n_seg = [labels[1][0] - labels[0][0], labels[2][0] - labels[1][0]]
    assert abs(n_seg[0] / n_seg[1] - seg[0] / seg[1]) < 0.2
    assert abs(x[-1] - sum(seg)) < 1e-12
    with pytest.raises(ValueError):
        k_path(cell, pts[:1], 10)
    assert chunk_size(8, 24 ** 3) == 24
    assert chunk_size(480, 96 ** 3) == 1
    assert chunk_size(160, 72 ** 3) == int(1.5e9 / (160 * 72 ** 3 * 16))


def test_bench_reference_arm_contract():
    """``bench.py --impl reference`` (the reference's CPU path, timed on the
    host cores) prints one JSON line with the contract's keys and says which
    ran (the staged reference or the port); on the 2-atom cell it runs in
    seconds."""
    import json
    import subprocess
    import sys
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--config", "si2_fcc",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["higher_is_better"] is False and line["value"] > 0
    # the reference's own solver when its package is staged under
    # baseline/_ref, else the float64 port
    staged = (ROOT / "baseline" / "_ref" / "gradwave").is_dir()
    assert line["cpu_baseline"]["kind"] == ("reference" if staged else "port")
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0


def test_autotune_records_and_lookup(tmp_path, monkeypatch):
    """The autotuner's table: keys by apply kind, box and projector count; a
    recorded choice is found, a missing one is None (built-in rules)."""
    import json
    from gradwave_b200 import autotune
    p = tmp_path / "tuning.json"
    k = autotune.key("gamma", (96, 96, 96), 864)
    assert k == "gamma:96x96x96:p864"
    p.write_text(json.dumps({"entries": {k: {"choice": {"w_budget_mb": 32, "nl_target": 296}}}}))
    monkeypatch.setattr(autotune, "TUNING", p)
    monkeypatch.setattr(autotune, "_CACHE", None)
    assert autotune.lookup("gamma", (96, 96, 96), 864) == {"w_budget_mb": 32, "nl_target": 296}
    assert autotune.lookup("complex", (96, 96, 96), 864) is None
    monkeypatch.setattr(autotune, "_CACHE", None)


def test_new_switches_and_gamma_preconditioner_refuse_bad_arguments():
    """The eigensolver and preconditioner switches accept only their
    documented values, and the Gamma preconditioner entry refuses bad sizes
    with GWB_ERR_ARG before it touches a device."""
    from gradwave_b200 import _lib
    for name, bad in (("gwb_sytrd_set_cluster", 5), ("gwb_sytrd_set_grid", 2), ("gwb_precond_set_kernel", 3)):
        with pytest.raises(_lib.GwbError) as ex:
            _lib.call(name, bad)
        assert ex.value.status == _lib.GWB_ERR_ARG
    # the defaults are accepted again (and restore the state)
    _lib.call("gwb_sytrd_set_cluster", -1)
    _lib.call("gwb_sytrd_set_grid", 0)
    _lib.call("gwb_precond_set_kernel", 1)
    lib = _lib.load()
    assert lib.gwb_precond_learned_gamma_work_bytes(0, 100) == 0
    nhalf = 100
    need = int(lib.gwb_precond_learned_gamma_work_bytes(4, nhalf))
    assert need == (4 * (2 + 1) + 1) * 8
    p = 1  # never dereferenced: the size checks come first
    # npad shorter than the embedding (2 nhalf - 1 coordinates)
    with pytest.raises(_lib.GwbError) as ex:
        _lib.call("gwb_precond_learned_gamma", p, 8, 4, nhalf, 2 * nhalf - 2, p, 2 * nhalf, p, 2 * nhalf, p, p, p,
                  None, p, 2 * nhalf, p, need, None)
    assert ex.value.status == _lib.GWB_ERR_ARG
    # more selected rows than bands
    with pytest.raises(_lib.GwbError) as ex:
        _lib.call("gwb_precond_learned_gamma", p, 3, 4, nhalf, 2 * nhalf, p, 2 * nhalf, p, 2 * nhalf, p, p, p,
                  None, p, 2 * nhalf, p, need, None)
    assert ex.value.status == _lib.GWB_ERR_ARG
    # a workspace smaller than asked for
    with pytest.raises(_lib.GwbError) as ex:
        _lib.call("gwb_precond_learned_gamma", p, 8, 4, nhalf, 2 * nhalf, p, 2 * nhalf, p, 2 * nhalf, p, p, p,
                  None, p, 2 * nhalf, p, need - 8, None)
    assert ex.value.status == _lib.GWB_ERR_ARG
