"""Units of the band-solve path: eV for energies, Angstrom for lengths.

The values are the CODATA 2018 constants the reference uses
(gradwave ``constants.py:1-14``), so kinetic energies and potentials agree with
it to the last bit.
"""

HARTREE_EV = 27.211386245988
RY_EV = HARTREE_EV / 2.0
BOHR_ANG = 0.529177210903
# hbar^2 / 2 m_e in eV * A^2: T(G) = HBAR2_2M * |k+G|^2 with |k+G| in 1/A.
HBAR2_2M = RY_EV * BOHR_ANG ** 2
