"""Launch-shape autotuner (spns_autotune) and the alternate shapes it picks from.

Bars: every alternate shape (E = 6 values per thread) keeps the FP64 step within
1e-12 relative L2 of the oracle after 5 steps in each step form; tuning leaves
the state bit for bit as it found it; a tuned run stays within 1e-12 of an
untuned one (the shapes change only the radix plan, hence the rounding)."""
import numpy as np
import pytest

from gpu_util import make_args, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("opts,form", [(dict(), 0), (dict(), 2), (dict(les=0.17), 0),
                                       (dict(self_adaptive=True, rotating=(0.0, 0.0, 1.0)), 0)],
                         ids=["rotational", "advective", "les", "kappa-rotating"])
def test_alternate_shapes_match_the_oracle(opts, form):
    import oracle as O
    from spns_b200.hit import HIT
    args = make_args(32, nu=3.283e-4, **opts)
    gpu = HIT(args, k41_ranks=4, nonlinear_form=form)
    gpu.set_shapes([1, 1, 1, 1, 1])
    ref = O.OracleHIT(args, k41_ranks=4)
    for _ in range(5):
        gpu.New_Fractional_Step_Method()
        ref.New_Fractional_Step_Method()
    assert rel_l2(gpu.get_compact(), ref.get_compact()) < 1e-12
    assert abs(gpu.gettime() - ref.gettime()) <= 1e-13 * ref.gettime()


def test_fp32_alternate_shapes_track_fp64():
    from spns_b200.hit import HIT, SPNS_FP64, SPNS_FP32_HILO
    args = make_args(48, nu=1e-3, les=0.15)
    a, b = HIT(args, precision=SPNS_FP64, k41_ranks=4), HIT(args, precision=SPNS_FP32_HILO, k41_ranks=4)
    b.set_shapes([1, 1, 1, 1, 1])
    a.New_Fractional_Step_Method(10)
    b.New_Fractional_Step_Method(10)
    ea, eb = a.Recalculate_Energy_Cascade(), b.Recalculate_Energy_Cascade()
    m = ea > 1e-6 * ea.max()
    assert np.max(np.abs(eb[m] - ea[m]) / ea[m]) < 1e-5


@pytest.mark.parametrize("prec", [0, 1])
def test_tuning_leaves_the_run_unchanged(prec):
    from spns_b200.hit import HIT, autotune_forget
    autotune_forget()
    args = make_args(32, nu=2e-3, les=0.12, self_adaptive=True)
    a = HIT(args, precision=prec)
    a.seed_field(5, 3.0)
    a.New_Fractional_Step_Method(3)
    blob = a.checkpoint_save()
    U0, t0 = a.get_compact(), a.gettime()
    choice = a.autotune(steps=3)
    assert len(choice) == 5 and set(choice) <= {0, 1}
    assert np.array_equal(a.get_compact(), U0) and a.gettime() == t0
    b = HIT(args, precision=prec)                  # same box: takes the cached shapes
    b.checkpoint_load(blob)
    assert b.autotune(steps=3) == choice
    c = HIT(args, precision=prec)
    c.checkpoint_load(blob)
    c.set_shapes([0, 0, 0, 0, 0])
    for h in (a, b, c):
        h.New_Fractional_Step_Method(6)
    assert np.array_equal(a.get_compact(), b.get_compact())
    assert rel_l2(a.get_compact(), c.get_compact()) < (1e-12 if prec == 0 else 1e-6)
    autotune_forget()


def test_long_axes_have_no_alternate():
    from spns_b200.hit import HIT, SpnsError, autotune_forget
    autotune_forget()
    h = HIT(make_args(32, nu=1e-2, Ns=(32, 32, 256)))     # FFT lengths 48, 48, 384
    choice = h.autotune(steps=2)
    assert choice[2] == 0                                 # z pass at length 384: default only
    with pytest.raises(SpnsError):
        h.set_shapes([0, 0, 1, 0, 0])
    with pytest.raises(SpnsError):
        h.set_shapes([2, 0, 0, 0, 0])
    autotune_forget()
