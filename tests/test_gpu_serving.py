"""Device-side extensions: seeded Philox field, exact checkpoints, ensembles
and the serving loop on the GPU.

Bars: the seeded field equals its host restatement to 1e-13 (libm rounding of
log/sin/cos only); a checkpoint resumes bit for bit; an ensemble member reaches
bit for bit the state it reaches stepped alone; a served run that resumes from a
checkpoint reaches the same time and E(K) within 1e-14 (E(K) is summed with
floating-point atomics, whose order varies), and a seeded served run within
1e-10 (its seeding normalisation is such a sum)."""
import numpy as np
import pytest

from gpu_util import make_args, rel_l2

pytestmark = pytest.mark.gpu


def test_seed_field_matches_host_restatement():
    from spns_b200.fields import philox_spectral_field, energy_spectrum
    from spns_b200.hit import HIT, SPNS_FP64
    for N, L in ((32, (1, 1, 1)), (48, (1, 1, 1)), (32, (1, 2, 1))):
        args = make_args(N, nu=1e-2, L=L)
        h = HIT(args, precision=SPNS_FP64)
        h.seed_field(12345, kp=3.0, urms=1.0)
        U = h.get_compact()
        ref = philox_spectral_field(N, N, N, kp=3.0, seed=12345, scale=L) if L == (1, 1, 1) else None
        if ref is not None:
            assert np.max(np.abs(U - ref)) <= 1e-13 * np.max(np.abs(ref))
        ek = h.Recalculate_Energy_Cascade()
        assert abs(ek.sum() - 1.5) < 1e-12
        # solenoidal, Hermitian kz=0 plane
        h.close()


def test_seed_field_fp32_hilo_keeps_the_double_field():
    from spns_b200.hit import HIT, SPNS_FP64, SPNS_FP32_HILO
    args = make_args(32, nu=1e-2)
    a, b = HIT(args, precision=SPNS_FP64), HIT(args, precision=SPNS_FP32_HILO)
    a.seed_field(7, 3.0)
    b.seed_field(7, 3.0)
    assert rel_l2(b.get_compact(), a.get_compact()) < 1e-14


@pytest.mark.parametrize("opts,prec", [(dict(), 0), (dict(self_adaptive=True), 0), (dict(self_adaptive=True), 1),
                                       (dict(les=0.17, rotating=(0.0, 0.0, 1.0)), 1)])
def test_checkpoint_resumes_bit_for_bit(opts, prec):
    from spns_b200.hit import HIT
    args = make_args(32, nu=3.283e-4, **opts)
    a = HIT(args, precision=prec, k41_ranks=4)
    a.New_Fractional_Step_Method(5)
    blob = a.checkpoint_save()
    a.New_Fractional_Step_Method(5)
    ref = a.get_compact()
    c = HIT(args, precision=prec, k41_ranks=4)
    c.checkpoint_load(blob)
    c.New_Fractional_Step_Method(5)
    assert np.array_equal(c.get_compact(), ref)
    assert c.gettime() == a.gettime() and c.getAt() == a.getAt()


def test_checkpoint_rejects_another_box():
    from spns_b200.hit import HIT, SpnsError
    a = HIT(make_args(32, nu=1e-2))
    blob = a.checkpoint_save()
    b = HIT(make_args(48, nu=1e-2))
    with pytest.raises(SpnsError):
        b.checkpoint_load(blob)
    with pytest.raises(SpnsError):
        b.checkpoint_load(b"not a checkpoint at all" * 4)


SPECS = [(32, dict(les=0.12), 1, 1), (48, dict(), 0, 2), (64, dict(les=0.18), 1, 3), (32, dict(self_adaptive=True), 0, 4),
         (48, dict(les=0.15, self_adaptive=True), 1, 5)]


def _seeded(specs):
    """One seeded handle per spec and the checkpoint of its initial state."""
    from spns_b200.hit import HIT
    out = []
    for N, opts, prec, seed in specs:
        h = HIT(make_args(N, nu=2e-3, **opts), precision=prec)
        h.seed_field(seed, 3.0)
        out.append((h, h.checkpoint_save()))
    return out


def _from(specs, blobs):
    from spns_b200.hit import HIT
    out = []
    for (N, opts, prec, seed), blob in zip(specs, blobs):
        h = HIT(make_args(N, nu=2e-3, **opts), precision=prec)
        h.checkpoint_load(blob)
        out.append(h)
    return out


def test_ensemble_members_equal_their_runs_alone():
    from spns_b200.hit import Ensemble
    mix = _seeded(SPECS)
    alone = _from(SPECS, [b for _, b in mix])
    for h in alone:
        h.New_Fractional_Step_Method(12)
    members = [h for h, _ in mix]
    ens = Ensemble(members)
    ens.step(5)
    ens.step(7)
    for h, ref in zip(members, alone):
        assert np.array_equal(h.get_compact(), ref.get_compact())
        assert h.gettime() == ref.gettime()
    # members keep working on their own after the ensemble
    for h, ref in zip(members, alone):
        h.New_Fractional_Step_Method(2)
        ref.New_Fractional_Step_Method(2)
        assert np.array_equal(h.get_compact(), ref.get_compact())
    ens.close()


def test_served_runs_equal_their_runs_alone():
    """Resumed requests (exact initial state) give bit-identical results in the mix;
    seeded requests agree to the rounding of their seeding."""
    from spns_b200.serving import GpuBackend, Server, SolveRequest
    seeded = _seeded(SPECS)
    blobs = [b for _, b in seeded]
    reqs = []
    for i, ((N, opts, prec, seed), blob) in enumerate(zip(SPECS, blobs)):
        args = make_args(N, nu=2e-3, **opts)
        reqs.append(SolveRequest(i, args, nsteps=30 + 7 * i, seed=seed, kp=3.0, precision=prec, arrival=0.002 * i,
                                 init=blob))
        reqs.append(SolveRequest(100 + i, args, nsteps=30 + 7 * i, seed=seed, kp=3.0, precision=prec,
                                 arrival=0.002 * i + 0.001))
    srv = Server(GpuBackend(), budget_bytes=8 << 30, chunk=4)
    res = srv.run(reqs)
    assert srv.used == 0
    alone = _from(SPECS, blobs)
    for i, h in enumerate(alone):
        h.New_Fractional_Step_Method(30 + 7 * i)
        ek = h.Recalculate_Energy_Cascade()
        exact, seeded_run = res[i], res[100 + i]
        assert exact.status == "done" and seeded_run.status == "done", (exact.error, seeded_run.error)
        m = ek > 1e-12 * ek.max()
        assert exact.time == h.gettime()
        assert np.max(np.abs(exact.ek[m] - ek[m]) / ek[m]) < 1e-14
        assert np.max(np.abs(seeded_run.ek[m] - ek[m]) / ek[m]) < 1e-10


def test_estimate_matches_the_allocation():
    import torch
    from spns_b200.hit import HIT, estimate_device_bytes
    args = make_args(64, nu=1e-2, self_adaptive=True)
    for prec in (0, 1):
        est = estimate_device_bytes(args, precision=prec)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        h = HIT(args, precision=prec)
        free1, _ = torch.cuda.mem_get_info()
        used = free0 - free1
        # allocation granularity (2 MiB pages) and the stream's own memory
        assert est <= used + (64 << 20) and used <= est + (64 << 20), (est, used)
        h.close()


def test_ensemble_batched_classes_equal_their_runs_alone():
    """Members of one class (same precision, box, form and launch shapes; Adams-Bashforth)
    step in one launch per pass for the whole class; each still reaches bit for bit the
    state it reaches alone.  Mixed with members that keep their own branch."""
    from spns_b200.hit import HIT, Ensemble
    specs = [(32, dict(les=0.10), 1, 2), (32, dict(les=0.15), 1, 2), (32, dict(les=0.20, rotating=(0.0, 0.0, 1.0)), 1, 2),
             (48, dict(), 0, 2), (48, dict(), 0, 2), (32, dict(les=0.17), 0, 2), (32, dict(les=0.12), 0, 2),
             (32, dict(self_adaptive=True), 0, 0), (48, dict(les=0.1), 1, 2)]

    def make(N, opts, prec, form):
        return HIT(make_args(N, nu=2e-3, **opts), precision=prec, nonlinear_form=form, k41_ranks=-1)

    members, alone = [], []
    for i, sp in enumerate(specs):
        h = make(*sp)
        h.seed_field(100 + i, 3.0)
        blob = h.checkpoint_save()        # the same initial state, bit for bit, for the run alone
        members.append(h)
        a = make(*sp)
        a.checkpoint_load(blob)
        alone.append(a)
    for h in alone:
        h.New_Fractional_Step_Method(9)
    ens = Ensemble(members, batched=True)
    ens.step(2)
    ens.step(7)
    for h, ref in zip(members, alone):
        assert np.array_equal(h.get_compact(), ref.get_compact())
        assert h.gettime() == ref.gettime() and h.getAt() == ref.getAt()
    ens.close()
