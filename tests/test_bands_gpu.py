"""The band-structure driver (gradwave ``postscf/bands.py:39-120``) on the
GPU: the 2-atom fcc cell at its frozen potential along L - Gamma - X.

Every path point is checked against the float64 oracle Davidson on the same
k-point tables (1e-9 eV); Gamma against the reference's own golden
eigenvalues of the cell; the chunking of the path (the reference's rule, or
chunks of 4) does not change the eigenvalues beyond the solver tolerance.
"""

import numpy as np
import pytest

from tests.conftest import load_golden

pytestmark = pytest.mark.gpu

PATH = [("L", [0.5, 0.5, 0.5]), ("G", [0.0, 0.0, 0.0]), ("X", [0.5, 0.0, 0.5])]


def test_band_structure_matches_oracle_and_reference(cuda_device):
    from gradwave_b200.bands import band_structure, bands_along_path
    from gradwave_b200.cells import at_kpoints, make_cell
    from oracle.davidson import davidson_batched as oracle_davidson
    from oracle.ham import from_cell
    ci = make_cell("si2_fcc")
    bs = bands_along_path(ci, PATH, npoints=9, diago_tol=1e-10, max_iter=200)
    assert bs.eigenvalues.shape == (9, ci.nbands)
    assert [lab for _, lab in bs.labels] == ["L", "G", "X"]
    cp = at_kpoints(ci, bs.kpts_frac)
    ref = oracle_davidson(from_cell(cp).apply, cp.identity_start().numpy(), cp.bk.t.numpy(), cp.bk.mask.numpy(),
                          tol=1e-10, max_iter=200).eigenvalues
    assert np.abs(bs.eigenvalues - ref).max() < 1e-9
    ig = bs.labels[1][0]
    g = load_golden("si2_fcc")
    assert np.abs(bs.eigenvalues[ig] - g["eigenvalues"][0]).max() < 1e-9
    assert bs.reference == pytest.approx(bs.eigenvalues[:, ci.nocc() - 1].max())
    small = band_structure(ci, bs.kpts_frac, diago_tol=1e-10, max_iter=200, chunk=4)
    assert len(small.n_iter) == 3
    assert np.abs(small.eigenvalues - bs.eigenvalues).max() < 1e-9
