"""Host-side behaviour of the engine's Python layer with a stand-in for the
library handle (CPU): ``sweep`` raises on a failed point, as the reference's
solve does on a singular matrix and its pipeline on a non-finite charge
(solver.py:121-122), while ``charges`` hands back every point's status."""
import numpy as np
import pytest

from sawsim_b200 import _lib as L
from sawsim_b200.engine import FrequencySolver


class _Handle:
    """Answers ss_sweep with Q = omega and the given per-point statuses."""

    def __init__(self, statuses):
        self.statuses = statuses

    def __call__(self, name, *args):
        assert name == 'ss_sweep'
        n, om, _, _, Q, st, it = args
        for i in range(n):
            Q[2 * i], Q[2 * i + 1] = om[i], 0.0
            st[i] = self.statuses[i]
            it[i] = 1
        return L.SS_OK


def _engine(statuses):
    return FrequencySolver(_Handle(statuses), 12, 3, L.SS_Q9_ME1, [0], [1])


def test_sweep_returns_charges_when_every_point_is_ok():
    f = np.array([1.0e9, 1.5e9, 2.0e9])
    Q = _engine([0, 0, 0]).sweep(f)
    assert np.allclose(Q, 2 * np.pi * f)


def test_sweep_raises_on_a_failed_point():
    f = np.array([1.0e9, 1.5e9, 2.0e9])
    with pytest.raises(L.SawsimError) as e:
        _engine([0, L.SS_ESINGULAR, 0]).sweep(f)
    assert e.value.code == L.SS_ESINGULAR and '1 of 3 points' in str(e.value) and '1.500000000 GHz' in str(e.value)
    Q, st, _ = _engine([0, L.SS_ENOCONV, 0]).charges(2 * np.pi * f)
    assert list(st) == [0, L.SS_ENOCONV, 0] and Q.size == 3
