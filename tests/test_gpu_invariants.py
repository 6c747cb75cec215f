"""Velocity-gradient invariant spectra on the GPU against the oracle.

Bar: per shell within 1e-10 relative on shells above 1e-10 of the peak (the
states themselves agree to 1e-12, the spectra are quadratic in fourth-order
products), FP32 within 1e-5; computing them leaves the run untouched (bit for bit against
a copy resumed from a checkpoint)."""
import numpy as np
import pytest

from gpu_util import make_args
from test_oracle_invariants import shear_state

pytestmark = pytest.mark.gpu


def _close(a, b, tol):
    for c in range(5):
        m = np.abs(b[c]) > 1e-10 * np.abs(b[c]).max()
        assert np.max(np.abs(a[c][m] - b[c][m]) / np.abs(b[c][m])) < tol, (c, np.max(np.abs(a[c][m] - b[c][m]) / np.abs(b[c][m])))


@pytest.mark.parametrize("opts,form", [(dict(), 0), (dict(), 2), (dict(les=0.17), 0), (dict(L=(1, 2, 1)), 0)],
                         ids=["rotational", "advective", "les", "noncubic"])
def test_invariant_spectra_match_the_oracle(opts, form):
    import oracle as O
    from spns_b200.hit import HIT
    args = make_args(32, nu=3.283e-4, **opts)
    gpu = HIT(args, k41_ranks=4, nonlinear_form=form)
    ref = O.OracleHIT(args, k41_ranks=4)
    for _ in range(5):
        gpu.New_Fractional_Step_Method()
        ref.New_Fractional_Step_Method()
    _close(gpu.Recalculate_Invariants_Distribution(), ref.Recalculate_Invariants_Distribution(), 1e-10)


def test_invariants_of_a_shear_layer_on_the_gpu():
    from spns_b200.hit import HIT
    h = HIT(make_args(32, nu=1e-2))
    h.set_compact(shear_state(32))
    sp = h.Recalculate_Invariants_Distribution()
    assert np.max(np.abs(sp[[0, 2, 3, 4]])) < 1e-28
    assert abs(sp[1][0] - 1 / 64) < 1e-15 and abs(sp[1][2] - 2 / 256) < 1e-15


def test_fp32_invariants_and_the_run_is_untouched(tmp_path):
    from spns_b200.hit import HIT, SPNS_FP64, SPNS_FP32_HILO
    args = make_args(32, nu=3.283e-4)
    a = HIT(args, k41_ranks=4, precision=SPNS_FP64)
    b = HIT(args, k41_ranks=4, precision=SPNS_FP32_HILO)
    for h in (a, b):
        h.New_Fractional_Step_Method(3)
    c = HIT(args, precision=SPNS_FP64)
    c.checkpoint_load(a.checkpoint_save())
    names = [str(tmp_path / f"inv{i}.dat") for i in range(5)]
    sa = a.Recalculate_Invariants_Distribution(names)
    _close(b.Recalculate_Invariants_Distribution(), sa, 1e-5)
    rows = np.loadtxt(names[1])
    assert rows.shape == (sa.shape[1], 2) and np.allclose(rows[:, 1], sa[1], rtol=1e-5, atol=0)
    a.New_Fractional_Step_Method(3)
    c.New_Fractional_Step_Method(3)
    assert np.array_equal(a.get_compact(), c.get_compact())


@pytest.mark.parametrize("N", [32, 48])
def test_eddy_viscosity_stats_match_the_oracle(N):
    import oracle as O
    from spns_b200.hit import HIT
    args = make_args(N, nu=3.283e-4, les=0.17)
    gpu = HIT(args, k41_ranks=4)
    ref = O.OracleHIT(args, k41_ranks=4)
    for _ in range(3):
        gpu.New_Fractional_Step_Method()
        ref.New_Fractional_Step_Method()
    g, r = gpu.eddy_viscosity_stats(), ref.eddy_viscosity_stats()
    assert np.all(r > 0)
    assert np.max(np.abs(g - r) / r) < 1e-11, (g, r)
    dns = HIT(make_args(N, nu=3.283e-4), k41_ranks=4)
    assert np.all(dns.eddy_viscosity_stats() == 0.0)


@pytest.mark.parametrize("box", [(512, 32, 32), (32, 512, 32), (32, 32, 512)], ids=["x768", "y768", "z768"])
def test_invariant_spectra_at_length_768(box):
    """The invariant passes (nine gradients through the inverse x and y passes, the
    invariants in the z pass, five forward transforms) are their own instantiations per
    FFT length: each axis in turn at the N=512 length, from a field with energy in every
    retained mode."""
    import oracle as O
    from gpu_util import broadband_field
    from spns_b200.hit import HIT
    args = make_args(0, nu=3.283e-4, Ns=box)
    U = broadband_field(*box, seed=5)
    gpu = HIT(args, k41_ranks=-1)
    ref = O.OracleHIT(args)
    for h in (gpu, ref):
        h.set_compact(U)
    _close(gpu.Recalculate_Invariants_Distribution(), ref.Recalculate_Invariants_Distribution(), 1e-10)
    gpu.close()
