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
    declared = set(re.findall(r"^\s*(?:int|int64_t|const char\*|size_t|unsigned long long)\s+(gwb_\w+)\(", header, re.M))
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
