"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this
module, as the checker.  ``OracleHIT`` exposes the reference ``HIT`` method names
(src/HIT_LES.h:90-201) over the C restatement in spns_oracle.c.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libspns_oracle.so")
_lib = None


class OrcArgs(C.Structure):
    _fields_ = [
        ("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int),
        ("Mx", C.c_int), ("My", C.c_int), ("Mz", C.c_int),
        ("nu", C.c_double), ("C_Smag", C.c_double), ("C_At", C.c_double),
        ("Lx", C.c_int), ("Ly", C.c_int), ("Lz", C.c_int),
        ("omega_x", C.c_double), ("omega_y", C.c_double), ("omega_z", C.c_double),
        ("Nx_file", C.c_int), ("Ny_file", C.c_int), ("Nz_file", C.c_int),
        ("isReLambda", C.c_int), ("isInitialFieldFromFile", C.c_int), ("isNotCubic", C.c_int),
        ("isRotating", C.c_int), ("isLES", C.c_int),
        ("isComplexConjugateCorrected", C.c_int), ("isSelfAdaptive", C.c_int),
        ("k41_ranks", C.c_int), ("nthreads", C.c_int),
        ("fixed_dt", C.c_double), ("eps_forcing", C.c_double),
        ("eps_kmin", C.c_int), ("eps_kmax", C.c_int),
    ]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, dp, i, d = C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_double
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(OrcArgs), dp]
        for name in ("orc_destroy", "orc_step", "orc_recalculate_timestep", "orc_velocity_antitransform",
                     "orc_complex_conjugate_correction"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = None
        L.orc_forcing_energy_cascade.argtypes = [vp, dp, i, i]
        L.orc_forcing_reynolds_lambda.argtypes = [vp, d]
        for name in ("orc_recalculate_reynolds_lambda", "orc_recalculate_energy", "orc_recalculate_enstrophy"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = d
        L.orc_recalculate_energy_cascade.argtypes = [vp, dp]
        L.orc_invariant_spectra.argtypes = [vp, dp]
        L.orc_eddy_viscosity_stats.argtypes = [vp, dp]
        L.orc_recalculate_energy_cascade.restype = d
        L.orc_check_physfour_energy.argtypes = [vp, d, dp, dp]
        L.orc_check_physfour_energy.restype = i
        L.orc_get_scalars.argtypes = [vp, dp]
        L.orc_set_nu.argtypes = [vp, d]
        L.orc_compact_size.argtypes = [vp]
        L.orc_compact_size.restype = C.c_long
        L.orc_get_compact.argtypes = [vp, dp]
        L.orc_set_compact.argtypes = [vp, dp]
        L.orc_get_physical.argtypes = [vp, dp]
        L.orc_fft1d.argtypes = [i, dp, i]
        L.orc_rfft3d.argtypes = [i, i, i, dp, dp]
        L.orc_irfft3d.argtypes = [i, i, i, dp, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class OracleHIT:
    """CPU restatement of the reference ``HIT`` class (one MPI rank)."""

    def __init__(self, args, file_uvw=None, k41_ranks=1, nthreads=None, fixed_dt=0.0, eps_forcing=0.0,
                 eps_kmin=1, eps_kmax=2):
        L = lib()
        a = OrcArgs()
        for f in ("Nx", "Ny", "Nz", "Mx", "My", "Mz", "Lx", "Ly", "Lz", "Nx_file", "Ny_file", "Nz_file"):
            setattr(a, f, int(getattr(args, f)))
        for f in ("nu", "C_Smag", "C_At", "omega_x", "omega_y", "omega_z"):
            setattr(a, f, float(getattr(args, f)))
        a.isReLambda = int(args.isReLambda)
        a.isInitialFieldFromFile = int(args.is_file_init)
        a.isNotCubic = int(args.isNotCubic)
        a.isRotating = int(args.isRotating)
        a.isLES = int(args.isLES)
        a.isComplexConjugateCorrected = int(args.isComplexConjugateCorrected)
        a.isSelfAdaptive = int(args.isSelfAdaptive)
        a.k41_ranks = int(k41_ranks)
        a.nthreads = int(nthreads or os.cpu_count() or 1)
        a.fixed_dt = float(fixed_dt)
        a.eps_forcing = float(eps_forcing)
        a.eps_kmin, a.eps_kmax = int(eps_kmin), int(eps_kmax)
        self.args = args
        fp = None
        if args.is_file_init:
            self._file = np.ascontiguousarray(file_uvw, dtype=np.float64)
            fp = _dp(self._file)
        self._h = L.orc_create(C.byref(a), fp)
        self._L = L

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.orc_destroy(self._h)
            self._h = None

    # --- HIT interface (src/HIT_LES.h) ---
    def New_Fractional_Step_Method(self):
        self._L.orc_step(self._h)

    def Recalculate_TimeStep(self):
        self._L.orc_recalculate_timestep(self._h)

    def Forcing_Energy_Cascade(self, Ek, last_input_rad, nullify):
        e = np.ascontiguousarray(Ek, dtype=np.float64)
        self._L.orc_forcing_energy_cascade(self._h, _dp(e), int(last_input_rad), int(bool(nullify)))

    def Forcing_Reynolds_Lambda(self, relambda):
        self._L.orc_forcing_reynolds_lambda(self._h, float(relambda))

    def Recalculate_Reynolds_Lambda(self):
        return self._L.orc_recalculate_reynolds_lambda(self._h)

    def Recalculate_Energy(self):
        return self._L.orc_recalculate_energy(self._h)

    def Recalculate_Enstrophy(self):
        return self._L.orc_recalculate_enstrophy(self._h)

    def Recalculate_Invariants_Distribution(self):
        """Spectra [5][last_rad_max+1] of Q_G, Q_S, R_G, R_S, V^2 (src/HIT_LES.cpp:1297-1319)."""
        s = self._scalars()
        out = np.zeros((5, int(s[12]) + 1))
        self._L.orc_invariant_spectra(self._h, _dp(out))
        return out

    def eddy_viscosity_stats(self):
        """Mean, rms and maximum of nu_t over the grid (src/HIT_LES.cpp:130-142)."""
        out = np.zeros(3)
        self._L.orc_eddy_viscosity_stats(self._h, _dp(out))
        return out

    def Recalculate_Energy_Cascade(self):
        s = self._scalars()
        out = np.zeros(int(s[12]) + 1)
        self._L.orc_recalculate_energy_cascade(self._h, _dp(out))
        return out

    def Recalculate_Velocity_Antitransform(self):
        self._L.orc_velocity_antitransform(self._h)

    def Complex_Conjugate_Correction(self):
        self._L.orc_complex_conjugate_correction(self._h)

    def Check_PhysFour_Energy(self, atol=1e-13):
        d1, d2 = C.c_double(), C.c_double()
        bad = self._L.orc_check_physfour_energy(self._h, float(atol), C.byref(d1), C.byref(d2))
        return bad == 0, d1.value, d2.value

    def _scalars(self):
        s = np.zeros(14)
        self._L.orc_get_scalars(self._h, _dp(s))
        return s

    def gettime(self): return float(self._scalars()[0])
    def getAt(self): return float(self._scalars()[1])
    def getnu(self): return float(self._scalars()[2])
    def getEk_Tot(self): return float(self._scalars()[3])
    def getOk_Tot(self): return float(self._scalars()[4])
    def getReLambda(self): return float(self._scalars()[5])
    def getEk_init(self): return float(self._scalars()[6])
    def getEk_init_file(self): return float(self._scalars()[7])
    def getEnstrophy_init_file(self): return float(self._scalars()[8])
    def getkappa(self): return float(self._scalars()[9])
    def getlast_rad(self): return int(self._scalars()[11])
    def getlast_rad_max(self): return int(self._scalars()[12])
    def setnu(self, nu): self._L.orc_set_nu(self._h, float(nu))

    # --- state access for parity checks ---
    def get_compact(self):
        n = self._L.orc_compact_size(self._h)
        out = np.zeros(3 * 2 * n)
        self._L.orc_get_compact(self._h, _dp(out))
        a = self.args
        return out.view(np.complex128).reshape(3, 2 * (a.Ny // 2) + 1, 2 * (a.Nx // 2) + 1, a.Nz // 2 + 1)

    def set_compact(self, uvw):
        buf = np.ascontiguousarray(uvw, dtype=np.complex128).view(np.float64).ravel()
        self._L.orc_set_compact(self._h, _dp(buf))

    def get_physical(self):
        a = self.args
        out = np.zeros(3 * a.Mx * a.My * a.Mz)
        self._L.orc_get_physical(self._h, _dp(out))
        return out.reshape(3, a.Mx, a.My, a.Mz)


def fft1d(x, sign=-1):
    buf = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().orc_fft1d(len(buf), _dp(buf.view(np.float64)), int(sign))
    return buf


def rfft3d(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    n0, n1, n2 = x.shape
    out = np.zeros((n0, n1, n2 // 2 + 1), dtype=np.complex128)
    lib().orc_rfft3d(n0, n1, n2, _dp(x), _dp(out.view(np.float64)))
    return out


def irfft3d(X, n2):
    X = np.ascontiguousarray(X, dtype=np.complex128)
    n0, n1, _ = X.shape
    out = np.zeros((n0, n1, n2))
    lib().orc_irfft3d(n0, n1, n2, _dp(X.view(np.float64)), _dp(out))
    return out
