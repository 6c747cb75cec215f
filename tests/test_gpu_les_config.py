"""Rotating LES on the non-cubic box of the LES configuration (Nx=Ny=128, Nz=256 with
Lz=2, i.e. FFT grid 192 x 192 x 384; C_s=0.17, Omega=(0,0,1), nu=1e-4, seeded k_p=3
field, u_rms=1, CFL time step), compensated FP32 form against the FP64 form over
2000 steps.

Stated tolerances (measured on B200 in brackets): E(K) per shell above 1e-6 of the
peak 2e-5 (6.7e-6), total energy 1e-6 (6.2e-8), mean and rms of the eddy viscosity
nu_t 1e-6 (2.2e-7), maximum of nu_t 5e-5 (4.2e-6); the two runs reach the same time
within 1e-7 relative.  The flow is chaotic, so the differences grow with the steps;
the bars hold at 2000 steps."""
import numpy as np
import pytest

from gpu_util import make_args

pytestmark = pytest.mark.gpu


def les_config_args():
    return make_args(128, nu=1e-4, Ns=(128, 128, 128), L=(1, 1, 2), les=0.17, rotating=(0.0, 0.0, 1.0))


def test_les_config_fp32_vs_fp64_2000_steps():
    from spns_b200.hit import HIT, SPNS_FP64, SPNS_FP32_HILO
    args = les_config_args()
    assert (args.Mx, args.My, args.Mz) == (192, 192, 384)
    runs = {}
    for prec in (SPNS_FP64, SPNS_FP32_HILO):
        h = HIT(args, precision=prec)
        h.seed_field(3, 3.0, 1.0)
        h.New_Fractional_Step_Method(2000)
        runs[prec] = h
    a, b = runs[SPNS_FP64], runs[SPNS_FP32_HILO]
    assert abs(b.gettime() - a.gettime()) <= 1e-7 * a.gettime()
    e64, e32 = a.Recalculate_Energy_Cascade(), b.Recalculate_Energy_Cascade()
    m = e64 > 1e-6 * e64.max()
    assert np.max(np.abs(e32[m] - e64[m]) / e64[m]) < 2e-5
    assert abs(e32.sum() - e64.sum()) < 1e-6 * e64.sum()
    n64, n32 = a.eddy_viscosity_stats(), b.eddy_viscosity_stats()
    rel = np.abs(n32 - n64) / n64
    assert rel[0] < 1e-6 and rel[1] < 1e-6 and rel[2] < 5e-5, rel
