"""Shell sums of the state at the sizes the configurations query (E(K) after every step
in the benchmark's end-to-end loop), against a host computation of the same sums.

E(K) = sum over retained modes with round(|k|) = K of |u|^2 / 2, modes with kz > 0
counted twice (src/HIT_LES.cpp:1137-1214, 1261-1266); Omega(K) the same with 2 |k|^2
(the enstrophy integrand of :998-1002), whose total is Recalculate_Enstrophy.  The
boxes put up to 0.5 M rows of Kz = 17 .. 513 modes through the kernel (one warp per
run of rows, runs of equal K within a row), including a non-cubic box and the FP32
form's hi + lo state.
"""
import numpy as np
import pytest

from gpu_util import broadband_field, make_args

pytestmark = pytest.mark.gpu


def _actual(n, f):
    return n // f if n % 2 == 0 else (n - 1) // f + 1


def _host_sums(U, args):
    """E(K), Omega(K) of a compact state [3][Ky][Kx][Kz] of the true grid."""
    sx, sy, sz = args.Lx, args.Ly, args.Lz
    _, Ky, Kx, Kz = U.shape
    hx, hy = (Kx - 1) // 2, (Ky - 1) // 2
    m1 = np.where(np.arange(Kx) <= hx, np.arange(Kx), np.arange(Kx) - Kx) * sx
    m2 = np.where(np.arange(Ky) <= hy, np.arange(Ky), np.arange(Ky) - Ky) * sy
    m3 = np.arange(Kz) * sz
    k2 = (m2[:, None, None] ** 2 + m1[None, :, None] ** 2 + m3[None, None, :] ** 2).astype(np.float64)
    K = np.rint(np.sqrt(k2)).astype(np.int64)
    w = np.where(m3 > 0, 2.0, 1.0)[None, None, :]
    e = 0.5 * w * np.sum(np.abs(U) ** 2, axis=0)
    # last_rad_max of the reference (src/HIT_LES.h:49), on the expanded N
    kmax = int(np.ceil(np.sqrt((args.Nx // 2) ** 2 + (args.Ny // 2) ** 2 + (args.Nz // 2) ** 2)))
    sel = K <= kmax
    ek = np.bincount(K[sel], weights=e[sel], minlength=kmax + 1)
    om = np.bincount(K[sel], weights=(2.0 * k2 * e)[sel], minlength=kmax + 1)
    return ek, om


@pytest.mark.parametrize("shape,L", [((256, 256, 256), (1, 1, 1)), ((128, 64, 1024), (1, 1, 1)),
                                     ((1024, 512, 32), (1, 1, 1)), ((96, 48, 32), (2, 1, 1))])
def test_shell_sums_match_the_host(shape, L):
    from spns_b200.hit import HIT
    args = make_args(0, Ns=shape, L=L)
    true = tuple(_actual(n, f) for n, f in zip((args.Nx, args.Ny, args.Nz), L))
    h = HIT(args, k41_ranks=-1)
    U = broadband_field(*true, seed=sum(shape))
    h.set_compact(U)
    ek = h.Recalculate_Energy_Cascade()
    om_tot = h.Recalculate_Enstrophy()
    h.close()
    ek_ref, om_ref = _host_sums(U, args)
    assert ek.shape == ek_ref.shape
    m = ek_ref > 1e-12 * ek_ref.max()
    assert np.max(np.abs(ek[m] - ek_ref[m]) / ek_ref[m]) < 1e-12
    assert np.max(np.abs(ek - ek_ref)) <= 1e-14 * ek_ref.sum()
    assert abs(om_tot - om_ref[1:].sum()) <= 1e-12 * om_ref[1:].sum()


def test_shell_sums_of_the_compensated_fp32_state():
    """The FP32 form's state is a float hi + lo pair (about 48 bits); its shell sums are
    formed in double from hi + lo."""
    from spns_b200.hit import HIT, SPNS_FP32_HILO
    shape = (256, 128, 512)
    args = make_args(0, Ns=shape)
    h = HIT(args, k41_ranks=-1, precision=SPNS_FP32_HILO)
    U = broadband_field(*shape, seed=11)
    h.set_compact(U)
    ek = h.Recalculate_Energy_Cascade()
    h.close()
    ek_ref, _ = _host_sums(U, args)
    m = ek_ref > 1e-12 * ek_ref.max()
    assert np.max(np.abs(ek[m] - ek_ref[m]) / ek_ref[m]) < 1e-10
