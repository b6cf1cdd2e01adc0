"""Gated primitive-operation counters (the reference's ``core/opcount.py:1-46``).

A process-global tally of FFT passes (``fft``), subspace eigensolves (``eigh``)
and Hamiltonian applies (``hpsi``, band*k), bumped at the same chokepoints as
the reference. Off by default; pure side effect, never touches numerics.
"""

from __future__ import annotations

_STATE = {"on": False}
_COUNTS = {"fft": 0, "eigh": 0, "hpsi": 0}


def enable() -> None:
    _STATE["on"] = True


def disable() -> None:
    _STATE["on"] = False


def bump(key: str, n: int = 1) -> None:
    if _STATE["on"]:
        _COUNTS[key] += n


def snapshot() -> dict[str, int]:
    return dict(_COUNTS)


def since(prev: dict[str, int]) -> dict[str, int]:
    return {k: _COUNTS[k] - prev.get(k, 0) for k in _COUNTS}
