"""Compensated single-precision form (SPNS_FP32_HILO) against the FP64 form.

The FP32 form keeps the state as a float hi + lo pair (about 48 significant
bits) and runs the transforms and products in float, with the reductions, the
CFL time step and the forcing normalisation in double.  Its bar is the energy
spectrum: E(K) within 1e-5 relative per shell after 100 steps of the 64^3
decaying DNS (nu=0.01, dt=1e-3, seeded k^4 exp(-2(k/4)^2) field), on the
shells that hold more than 1e-6 of the peak shell energy, and within 1e-7 of
the total energy on every shell.  The FP64 GPU form (itself pinned to the
oracle at 1e-12) is the reference.
"""
import numpy as np
import pytest

from gpu_util import make_args, rel_l2

pytestmark = pytest.mark.gpu

EK_SHELL_TOL = 1e-5


def _hit(args, precision, **opt):
    from spns_b200.hit import HIT
    return HIT(args, precision=precision, **opt)


def _spectra_close(e32, e64, tol=EK_SHELL_TOL):
    m = e64 > 1e-6 * e64.max()
    rel = np.abs(e32[m] - e64[m]) / e64[m]
    assert rel.max() < tol, f"max shell rel err {rel.max():.3e} at K={np.argmax(rel)}"
    assert np.max(np.abs(e32 - e64)) < 1e-7 * e64.sum()
    return float(rel.max())


def test_state_roundtrip_keeps_48_bits():
    from spns_b200.hit import SPNS_FP32_HILO
    from spns_b200.fields import seeded_spectral_field
    h = _hit(make_args(32, nu=1e-2), SPNS_FP32_HILO, fixed_dt=1e-3)
    U0 = seeded_spectral_field(32, 32, 32, kp=4.0, seed=3)
    h.set_compact(U0)
    U1 = h.get_compact()
    # |lo| <= ulp(hi)/2 and the split of lo itself loses at most 2^-24 of lo: ~2^-48 relative
    assert np.max(np.abs(U1 - U0)) <= 2.0 ** -46 * np.max(np.abs(U0))
    assert rel_l2(U1, U0) < 1e-14


def test_config1_fp32_vs_fp64_100_steps():
    """64^3 decaying DNS, nu=0.01, dt=1e-3, 100 steps: E(K) per shell within 1e-5."""
    from spns_b200.hit import SPNS_FP64, SPNS_FP32_HILO
    from spns_b200.fields import seeded_spectral_field
    args = make_args(64, nu=0.01)
    U0 = seeded_spectral_field(64, 64, 64, kp=4.0, seed=1)
    runs = {}
    for prec in (SPNS_FP64, SPNS_FP32_HILO):
        h = _hit(args, prec, fixed_dt=1e-3)
        h.set_compact(U0)
        h.Recalculate_Velocity_Antitransform()
        h.Recalculate_TimeStep()
        h.New_Fractional_Step_Method(100)
        runs[prec] = h
    e64 = runs[SPNS_FP64].Recalculate_Energy_Cascade()
    e32 = runs[SPNS_FP32_HILO].Recalculate_Energy_Cascade()
    err = _spectra_close(e32, e64)
    print(f"config1 FP32-hilo vs FP64 max shell rel err {err:.3e}, "
          f"state rel L2 {rel_l2(runs[SPNS_FP32_HILO].get_compact(), runs[SPNS_FP64].get_compact()):.3e}")
    assert abs(runs[SPNS_FP32_HILO].gettime() - runs[SPNS_FP64].gettime()) < 1e-12


@pytest.mark.parametrize("opts", [
    dict(),
    dict(self_adaptive=True),
    dict(rotating=(0.0, 0.0, 1.0), les=0.17),
], ids=["ab2", "kappa", "les-rotating"])
def test_k41_fp32_vs_fp64_cfl(opts):
    """K41 field, CFL time step (double) from float maxima, 20 steps."""
    from spns_b200.hit import SPNS_FP64, SPNS_FP32_HILO
    args = make_args(32, nu=3.283e-4, **opts)
    a = _hit(args, SPNS_FP64, k41_ranks=4)
    b = _hit(args, SPNS_FP32_HILO, k41_ranks=4)
    assert rel_l2(b.get_compact(), a.get_compact()) < 1e-14
    a.New_Fractional_Step_Method(20)
    b.New_Fractional_Step_Method(20)
    assert abs(b.gettime() - a.gettime()) <= 1e-5 * a.gettime()
    _spectra_close(b.Recalculate_Energy_Cascade(), a.Recalculate_Energy_Cascade())


def test_fp32_forcing_and_physical_field():
    """Forcing_Energy_Cascade scales hi and lo together; the physical field matches FP64 to float accuracy."""
    from spns_b200.hit import SPNS_FP64, SPNS_FP32_HILO
    args = make_args(32, nu=3.283e-4)
    a = _hit(args, SPNS_FP64, k41_ranks=1)
    b = _hit(args, SPNS_FP32_HILO, k41_ranks=1)
    lr = a.getlast_rad()
    target = np.zeros(lr + 1)
    target[1:] = 0.3 * np.arange(1, lr + 1, dtype=float) ** (-5.0 / 3.0)
    for h in (a, b):
        h.Forcing_Energy_Cascade(target, lr, False)
    ea, eb = a.Recalculate_Energy_Cascade(), b.Recalculate_Energy_Cascade()
    assert np.max(np.abs(eb[1:lr + 1] - ea[1:lr + 1]) / ea[1:lr + 1]) < 1e-13
    pa, pb = a.get_physical(), b.get_physical()
    assert rel_l2(pb, pa) < 1e-6
