"""GPU time step (FP64 plain form) against the CPU oracle on the same initial state.

Bar: spectral velocity field within 1e-12 relative L2 after 10 steps (the
FP64 drop-in tolerance); energy spectrum per shell within 1e-12 relative.
"""
import numpy as np
import pytest

from gpu_util import make_args, oracle_compact_to_true, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _pair(args, k41_ranks=4, form=0, **opt):
    import oracle as O
    from spns_b200.hit import HIT
    gpu = HIT(args, k41_ranks=k41_ranks, nonlinear_form=form, **opt)
    ref = O.OracleHIT(args, k41_ranks=k41_ranks, **opt)
    return gpu, ref


def _run(gpu, ref, nsteps, check_each=False):
    for i in range(nsteps):
        gpu.New_Fractional_Step_Method()
        ref.New_Fractional_Step_Method()
        if check_each:
            assert abs(gpu.getAt() - ref.getAt()) <= 1e-13 * ref.getAt()


def test_k41_initial_field_matches():
    gpu, ref = _pair(make_args(32, nu=3.283e-4))
    assert rel_l2(gpu.get_compact(), ref.get_compact()) < 1e-14
    assert abs(gpu.getAt() - ref.getAt()) <= 1e-14 * ref.getAt()
    assert abs(gpu.getEk_init() - ref.getEk_init()) <= 1e-13 * ref.getEk_init()


@pytest.mark.parametrize("form", [0, 2], ids=["rotational+edge", "advective"])
@pytest.mark.parametrize("opts", [
    dict(),
    dict(rotating=(1.5, -2.1, 3.0)),
    dict(self_adaptive=True),
    dict(conj=True),
])
def test_dns_10_steps_n32(opts, form):
    """K41 field: the +-N/2 modes fill during the steps, so both forms must be exact there."""
    gpu, ref = _pair(make_args(32, nu=3.283e-4, **opts), form=form)
    _run(gpu, ref, 10, check_each=True)
    assert rel_l2(gpu.get_compact(), ref.get_compact()) < TOL
    assert abs(gpu.gettime() - ref.gettime()) <= 1e-13 * ref.gettime()


def test_dns_constant_power_forcing():
    gpu, ref = _pair(make_args(32, nu=3.283e-4), eps_forcing=0.1)
    _run(gpu, ref, 10)
    assert rel_l2(gpu.get_compact(), ref.get_compact()) < TOL


def test_config1_seeded_n64_fixed_dt():
    """64^3 decaying DNS, nu=0.01, dt=1e-3, seeded k^4 exp(-2(k/4)^2) field, 10 steps."""
    from spns_b200.fields import seeded_spectral_field
    args = make_args(64, nu=0.01)
    gpu, ref = _pair(args, fixed_dt=1e-3)
    U0 = seeded_spectral_field(64, 64, 64, kp=4.0, seed=1)
    gpu.set_compact(U0)
    ref.set_compact(U0)
    for h in (gpu, ref):
        h.Recalculate_Velocity_Antitransform()
        h.Recalculate_TimeStep()
    _run(gpu, ref, 10)
    assert rel_l2(gpu.get_compact(), ref.get_compact()) < TOL
    eg, eo = gpu.Recalculate_Energy_Cascade(), ref.Recalculate_Energy_Cascade()
    m = eo > 1e-10 * eo.max()
    assert np.max(np.abs(eg[m] - eo[m]) / eo[m]) < 1e-11
    assert np.max(np.abs(eg - eo)) < 1e-14 * eo.sum()


def test_rotational_form_matches_when_edge_modes_are_empty():
    """omega x u differs from u.grad u by a gradient; with +-N/2 modes empty the projection removes it."""
    from spns_b200.fields import seeded_spectral_field
    args = make_args(64, nu=0.01)
    gpu, ref = _pair(args, fixed_dt=1e-3)
    from spns_b200.hit import HIT
    rot = HIT(args, k41_ranks=4, fixed_dt=1e-3, nonlinear_form=1)
    U0 = seeded_spectral_field(64, 64, 64, kp=4.0, seed=3)
    for h in (gpu, ref, rot):
        h.set_compact(U0)
        h.Recalculate_Velocity_Antitransform()
        h.Recalculate_TimeStep()
    for _ in range(10):
        for h in (gpu, ref, rot):
            h.New_Fractional_Step_Method()
    assert rel_l2(rot.get_compact(), ref.get_compact()) < TOL
    assert rel_l2(gpu.get_compact(), ref.get_compact()) < TOL


def test_unsupported_grid_is_reported():
    """Odd N gives M=(3N)/2 with no factor 3 (e.g. 46): outside the compiled FFT lengths."""
    from spns_b200.hit import HIT, SpnsError
    with pytest.raises(SpnsError) as ei:
        HIT(make_args(31, nu=3.283e-4), k41_ranks=4)
    assert ei.value.status == -2


def test_les_10_steps_n32():
    gpu, ref = _pair(make_args(32, nu=3.283e-4, les=0.16))
    _run(gpu, ref, 10, check_each=True)
    assert rel_l2(gpu.get_compact(), ref.get_compact()) < TOL


def test_les_rotating_noncubic():
    args = make_args(32, nu=3.283e-4, les=0.16, rotating=(1.5, -2.1, 3.0), L=(6, 3, 2))
    gpu, ref = _pair(args)
    _run(gpu, ref, 3)
    assert rel_l2(gpu.get_compact(), oracle_compact_to_true(ref.get_compact(), args)) < TOL


@pytest.mark.parametrize("form", [0, 2], ids=["rotational+edge", "advective"])
def test_noncubic_true_grid(form):
    """Length factors (6,3,2): GPU runs the 48^3 true grid, the oracle the expanded 288x144x96 one."""
    args = make_args(32, nu=3.283e-4, L=(6, 3, 2))
    gpu, ref = _pair(args, form=form)
    assert gpu.physical_shape[1:] == (48, 48, 48)
    assert rel_l2(gpu.get_compact(), oracle_compact_to_true(ref.get_compact(), args)) < 1e-14
    _run(gpu, ref, 3)
    assert rel_l2(gpu.get_compact(), oracle_compact_to_true(ref.get_compact(), args)) < TOL


def test_physical_velocity_and_parseval():
    gpu, ref = _pair(make_args(32, nu=3.283e-4))
    _run(gpu, ref, 2)
    ref.Recalculate_Velocity_Antitransform()
    pg, po = gpu.get_physical(), ref.get_physical()
    assert rel_l2(pg, po) < TOL
    ok, d1, _ = gpu.Check_PhysFour_Energy(1e-13)
    assert ok, d1


def test_nonfinite_state_is_reported():
    from spns_b200.hit import HIT, SpnsError
    gpu = HIT(make_args(32, nu=3.283e-4), k41_ranks=4)
    U = gpu.get_compact()
    U[0, 3, 3, 3] = np.nan
    gpu.set_compact(U)
    with pytest.raises(SpnsError) as ei:
        gpu.New_Fractional_Step_Method()
    assert ei.value.status == -5
