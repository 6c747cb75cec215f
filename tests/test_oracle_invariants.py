"""Velocity-gradient invariant spectra of the oracle (src/HIT_LES.cpp:1297-1319)
on an analytic field: the shear u = (sin y, 0, 0) has G = [[0, cos y, 0], 0, 0],
so Q_G = R_G = R_S = V^2 = 0 and Q_S = -cos^2(y)/4 = -1/8 - cos(2y)/8: its
spectrum is 1/64 at K=0 and 2 (1/16)^2 at K=2."""
import numpy as np

from gpu_util import make_args


def shear_state(N):
    K = N + 1
    U = np.zeros((3, K, K, N // 2 + 1), dtype=np.complex128)
    U[0, 1, 0, 0] = -0.5j          # ky = +1
    U[0, K - 1, 0, 0] = 0.5j       # ky = -1
    return U


def test_oracle_invariants_of_a_shear_layer():
    import oracle as O
    o = O.OracleHIT(make_args(16, nu=1e-2), k41_ranks=1)
    o.set_compact(shear_state(16))
    sp = o.Recalculate_Invariants_Distribution()
    assert np.max(np.abs(sp[[0, 2, 3, 4]])) < 1e-28
    expect = np.zeros(sp.shape[1])
    expect[0], expect[2] = 1 / 64, 2 / 256
    assert np.max(np.abs(sp[1] - expect)) < 1e-15
