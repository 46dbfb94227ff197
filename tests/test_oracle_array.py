"""The oracle's CORRELATION_ARRAY reweighting against the reference's formula
(src/hawaii.c:2640-2664), written out here in numpy."""
import numpy as np

from oracle import oracle as O

HKT = 4.3597447222071e-18 / 1.380649e-23


def _reference_weight(ps, pesmin, T0, T, E):
    WTT = 1.0
    if ps == O.PS_BOUND and T < T0:
        WTT = np.exp(-pesmin * HKT / T0 / T * (T0 - T))
    w = np.exp(-E * HKT / T0 / T * (T0 - T)) / WTT
    if ps == O.PS_FREE_AND_METASTABLE and T > T0:
        w = 0.0
    return w


def test_array_weights_follow_reference_formula():
    Ts = [100.0, 250.0, 300.0, 350.0, 500.0]
    for ps in (O.PS_FREE_AND_METASTABLE, O.PS_BOUND):
        for E in (-2e-4, -1e-6, 0.0, 3e-5, 1e-3):
            w = O.array_weights(ps, -8.9e-4, 300.0, Ts, E)
            ref = [_reference_weight(ps, -8.9e-4, 300.0, T, E) for T in Ts]
            np.testing.assert_allclose(w, ref, rtol=1e-15, atol=0)
    # the base temperature itself always has weight 1
    assert O.array_weights(O.PS_BOUND, -8.9e-4, 300.0, [300.0], -1e-4)[0] == 1.0
