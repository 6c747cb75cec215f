"""The allocation-free energy spectrum entry point against the handle-based one.

spns_energy_cascade_noalloc_f64 serves callers that cannot allocate device
memory at the time they need E(K): host frameworks whose caching pool holds the
device's free memory, and loops that must not stall other streams with the
synchronisation an allocation can cause.  Its working bins live in a fixed
array compiled into libspns.  It must give the same spectrum as spns_recalculate_energy_cascade
(the handle's cudaMalloc'd bins) on the same state, call after call, since the
shared array keeps the previous call's contents.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(L, h, nbins):
    u, v, w = C.c_void_p(), C.c_void_p(), C.c_void_p()
    assert L.spns_device_state(h._h, C.byref(u), C.byref(v), C.byref(w)) == 0
    _, Ky, Kx, Kz = h.spectral_shape
    Ek = np.zeros(nbins)
    tot = C.c_double()
    st = L.spns_energy_cascade_noalloc_f64(u, Kx, Ky, Kz, h.args.Lx, h.args.Ly, h.args.Lz,
                                           Ek.ctypes.data_as(C.POINTER(C.c_double)), nbins, C.byref(tot), None)
    assert st == 0, L.spns_last_error(None)
    return Ek, tot.value


@pytest.mark.parametrize("L_factors", [(1, 1, 1), (6, 3, 2)])
def test_noalloc_spectrum_matches_handle_spectrum(L_factors):
    from gpu_util import make_args
    from spns_b200.hit import HIT, lib
    L = lib()
    h = HIT(make_args(32, nu=3.283e-4, L=L_factors), k41_ranks=4)
    nbins = h.getlast_rad_max() + 1
    for _ in range(2):  # two calls in a row, the state changing in between
        h.New_Fractional_Step_Method()
        ref = h.Recalculate_Energy_Cascade()
        got, tot = _noalloc(L, h, nbins)
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-14 * ref.sum())
        assert abs(tot - h.getEk_Tot()) <= 1e-12 * h.getEk_Tot()
    h.close()


def test_noalloc_rejects_too_many_bins():
    from gpu_util import make_args
    from spns_b200.hit import HIT, lib
    L = lib()
    h = HIT(make_args(32, nu=3.283e-4), k41_ranks=4)
    u = C.c_void_p()
    L.spns_device_state(h._h, C.byref(u), None, None)
    Ek = np.zeros(4096)
    st = L.spns_energy_cascade_noalloc_f64(u, 33, 33, 17, 1, 1, 1, Ek.ctypes.data_as(C.POINTER(C.c_double)), 4096,
                                           None, None)
    assert st == -2
    assert b"exceeds" in L.spns_last_error(None)
    h.close()
