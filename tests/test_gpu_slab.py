"""Slab decomposition (spns_slab_*, spns_b200.slab) against the one-GPU step.

G ranks are emulated by one process on one GPU (LocalTransport: the all-to-alls
are device-to-device copies; no kernel waits on another).  Every rank runs the
slab kernels on its own ky rows and x planes, so the pack/unpack reorders, the
slab geometry of the passes, the wavenumbers of a rank's rows and the reductions
over ranks (CFL maxima, forced-shell energy) are all exercised.  The one-GPU
handle runs the same arithmetic (advective form, or LES) on the whole box.

Bar: relative L2 of the spectral state <= 1e-12 after 10 steps, dt equal to
1e-13 at every step (the reductions over ranks sum in another order than one
block does, so agreement is to rounding, not bit for bit).  The compensated FP32
form on slabs against FP32 on one GPU: 1e-6.  What runs on several GPUs in
separate processes (TorchTransport over NCCL) is not tested here: this run has
one GPU.
"""
import numpy as np
import pytest

from gpu_util import broadband_field, make_args, rel_l2

pytestmark = pytest.mark.gpu

CASES = {
    "ab2-2ranks": ((32, 32, 32), dict(), dict(), 2),
    "ab2-3ranks": ((32, 32, 32), dict(), dict(), 3),
    "kappa-eps-4ranks": ((32, 32, 32), dict(self_adaptive=True), dict(eps_forcing=0.1), 4),
    "les-rotating-2ranks": ((32, 32, 32), dict(les=0.17, rotating=(0.0, 0.0, 1.0)), dict(), 2),
    "n64-kappa-eps-4ranks": ((64, 64, 64), dict(self_adaptive=True), dict(eps_forcing=0.1), 4),
    "z768-2ranks": ((32, 32, 512), dict(self_adaptive=True), dict(eps_forcing=0.1), 2),
    "y768-3ranks": ((32, 512, 32), dict(), dict(), 3),
}


def _pair(box, aopt, hopt, G, precision=0):
    from spns_b200.hit import HIT
    from spns_b200.slab import LocalTransport, SlabHIT
    args = make_args(0, nu=3.283e-4, Ns=box, **aopt)
    one = HIT(args, nonlinear_form=2, precision=precision, **hopt)
    slab = SlabHIT(args, G, LocalTransport(), precision=precision, **hopt)
    U0 = broadband_field(*box, seed=11)
    one.set_compact(U0)
    slab.set_compact(U0)
    for h in (one, slab):
        h.Recalculate_Velocity_Antitransform()
        h.Recalculate_TimeStep()
    return one, slab


@pytest.mark.parametrize("name", list(CASES))
def test_slab_step_equals_one_gpu_step(name):
    box, aopt, hopt, G = CASES[name]
    one, slab = _pair(box, aopt, hopt, G)
    assert abs(slab.getAt() - one.getAt()) <= 1e-13 * one.getAt()
    for i in range(10):
        one.New_Fractional_Step_Method()
        slab.New_Fractional_Step_Method()
        assert abs(slab.getAt() - one.getAt()) <= 1e-13 * one.getAt(), f"dt differs at step {i + 1}"
    err = rel_l2(slab.get_compact(), one.get_compact())
    e1, es = one.Recalculate_Energy_Cascade(), slab.Recalculate_Energy_Cascade_rows()
    m = e1 > 1e-10 * e1.max()
    print(f"{name}: state rel L2 {err:.3e}, E(K) max shell rel {np.max(np.abs(es[m] - e1[m]) / e1[m]):.3e}")
    assert err < 1e-12
    assert np.max(np.abs(es[m] - e1[m]) / e1[m]) < 1e-11
    assert abs(slab.gettime() - one.gettime()) <= 1e-13 * one.gettime()
    slab.close()
    one.close()


def test_slab_fp32_form():
    from spns_b200.hit import SPNS_FP32_HILO
    one, slab = _pair((32, 32, 32), dict(self_adaptive=True), dict(eps_forcing=0.1), 2, precision=SPNS_FP32_HILO)
    one.New_Fractional_Step_Method(10)
    slab.New_Fractional_Step_Method(10)
    assert rel_l2(slab.get_compact(), one.get_compact()) < 1e-6
    slab.close()
    one.close()


def test_slab_rejects_what_it_cannot_do():
    from spns_b200.hit import SpnsError
    from spns_b200.slab import SlabRank
    with pytest.raises(SpnsError):
        SlabRank(make_args(32, conj=True), 2, 0)
    with pytest.raises(SpnsError):
        SlabRank(make_args(32), 40, 0)        # 33 ky rows cannot give 40 ranks a row each


def test_torch_transport_one_rank_over_nccl():
    """The multi-process transport (torch.distributed over NCCL) with one rank: the slab
    phases, the all-to-all calls on the rank's stream and the reductions run through NCCL
    on the GPU, and the step equals the one-GPU step."""
    import os
    import socket
    import torch
    import torch.distributed as dist
    from spns_b200.hit import HIT
    from spns_b200.slab import SlabHIT, TorchTransport
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        box = (32, 32, 32)
        args = make_args(0, nu=3.283e-4, Ns=box, self_adaptive=True)
        one = HIT(args, nonlinear_form=2, eps_forcing=0.1)
        slab = SlabHIT(args, 1, TorchTransport(), ranks=[0], eps_forcing=0.1)
        U0 = broadband_field(*box, seed=4)
        for h in (one, slab):
            h.set_compact(U0)
            h.Recalculate_Velocity_Antitransform()
            h.Recalculate_TimeStep()
        one.New_Fractional_Step_Method(10)
        slab.New_Fractional_Step_Method(10)
        torch.cuda.synchronize()
        assert rel_l2(slab.get_compact(), one.get_compact()) < 1e-12
        assert abs(slab.getAt() - one.getAt()) <= 1e-13 * one.getAt()
        slab.close()
        one.close()
    finally:
        dist.destroy_process_group()
