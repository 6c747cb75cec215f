"""Python mirror of the reference ``HIT`` class over the C ABI of libspns.

Method names, argument meaning and error behaviour follow src/HIT_LES.h of the
reference (``crash`` there raises ``SpnsError`` here).  All work runs in
libspns.so (CUDA, sm_100a); this module only marshals arguments.  There is no
CPU fallback: a missing library or a machine without a GPU raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from .params import HitArgs

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SPNS_LIB", os.path.join(_HERE, "_lib", "libspns.so"))

SPNS_FP64 = 0
SPNS_FP32_HILO = 1

# Every symbol declared in include/spns.h.
EXPORTED_SYMBOLS = (
    "spns_create", "spns_destroy", "spns_step", "spns_recalculate_timestep", "spns_forcing_energy_cascade",
    "spns_forcing_reynolds_lambda", "spns_recalculate_reynolds_lambda", "spns_recalculate_energy",
    "spns_recalculate_enstrophy", "spns_recalculate_energy_cascade", "spns_velocity_antitransform",
    "spns_complex_conjugate_correction", "spns_check_physfour_energy", "spns_get_scalars", "spns_set_nu",
    "spns_spectral_dims", "spns_physical_dims", "spns_get_spectral", "spns_set_spectral", "spns_get_physical",
    "spns_device_state", "spns_stream", "spns_kernels_per_step", "spns_last_error", "spns_status_string",
    "spns_fft1d_batch_f64", "spns_profile_begin", "spns_profile_read", "spns_profile_kernel_name",
    "spns_energy_cascade_noalloc_f64", "spns_estimate_device_bytes", "spns_seed_field", "spns_step_async",
    "spns_query", "spns_synchronize", "spns_checkpoint_bytes", "spns_checkpoint_save", "spns_checkpoint_load",
    "spns_ensemble_create", "spns_ensemble_step", "spns_ensemble_destroy", "spns_ensemble_last_error",
    "spns_invariant_spectra", "spns_eddy_viscosity_stats", "spns_autotune", "spns_autotune_forget", "spns_set_shapes",
    "spns_slab_block", "spns_slab_create", "spns_slab_layout", "spns_slab_phase", "spns_slab_exchange", "spns_slab_counts",
    "spns_slab_buffers", "spns_ensemble_set_batched",
)


def autotune_forget():
    """Clears the process-wide cache of tuned launch shapes."""
    lib().spns_autotune_forget()


class SpnsError(RuntimeError):
    """A non-zero status of libspns (the reference calls ``crash`` in these cases)."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"libspns status {status}: {msg}")
        self.status = status


class HitArgsC(C.Structure):
    _fields_ = [
        ("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int),
        ("Mx", C.c_int), ("My", C.c_int), ("Mz", C.c_int),
        ("nu", C.c_double), ("C_Smag", C.c_double), ("C_At", C.c_double),
        ("Lx_factor", C.c_int), ("Ly_factor", C.c_int), ("Lz_factor", C.c_int),
        ("omega_x", C.c_double), ("omega_y", C.c_double), ("omega_z", C.c_double),
        ("Nx_file", C.c_int), ("Ny_file", C.c_int), ("Nz_file", C.c_int),
        ("isReLambda", C.c_int), ("isInitialFieldFromFile", C.c_int), ("isNotCubic", C.c_int),
        ("isRotating", C.c_int), ("isLES", C.c_int),
        ("isComplexConjugateCorrected", C.c_int), ("isSelfAdaptive", C.c_int),
        ("precision", C.c_int), ("device", C.c_int), ("k41_ranks", C.c_int),
        ("fixed_dt", C.c_double), ("eps_forcing", C.c_double),
        ("eps_kmin", C.c_int), ("eps_kmax", C.c_int), ("nonlinear_form", C.c_int),
        ("stream_priority", C.c_int),
    ]


class ScalarsC(C.Structure):
    _fields_ = [
        ("time", C.c_double), ("At", C.c_double), ("nu", C.c_double), ("Ek_Tot", C.c_double),
        ("Ok_Tot", C.c_double), ("ReLambda", C.c_double), ("Ek_init", C.c_double), ("Ek_init_file", C.c_double),
        ("Enstrophy_init_file", C.c_double), ("kappa", C.c_double), ("MaxVel", C.c_double),
        ("iter", C.c_int64), ("last_rad", C.c_int64), ("last_rad_max", C.c_int64),
    ]


_lib = None


def lib():
    """Load libspns.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SpnsError(-3, f"{LIB_PATH} is missing: build it with `python __graft_entry__.py build` "
                                "or `make -C spns_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        vp, dp, i, d, ip = C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_double, C.POINTER(C.c_int)
        L.spns_create.argtypes = [C.POINTER(HitArgsC), dp, C.POINTER(vp)]
        L.spns_destroy.argtypes = [vp]
        L.spns_step.argtypes = [vp, i]
        L.spns_recalculate_timestep.argtypes = [vp]
        L.spns_forcing_energy_cascade.argtypes = [vp, dp, i, i]
        L.spns_forcing_reynolds_lambda.argtypes = [vp, d]
        L.spns_recalculate_reynolds_lambda.argtypes = [vp, dp]
        L.spns_recalculate_energy.argtypes = [vp, dp]
        L.spns_recalculate_enstrophy.argtypes = [vp, dp]
        L.spns_recalculate_energy_cascade.argtypes = [vp, dp, dp]
        L.spns_velocity_antitransform.argtypes = [vp]
        L.spns_complex_conjugate_correction.argtypes = [vp]
        L.spns_check_physfour_energy.argtypes = [vp, d, ip, dp, dp]
        L.spns_get_scalars.argtypes = [vp, C.POINTER(ScalarsC)]
        L.spns_set_nu.argtypes = [vp, d]
        L.spns_spectral_dims.argtypes = [vp, ip, ip, ip]
        L.spns_physical_dims.argtypes = [vp, ip, ip, ip]
        L.spns_get_spectral.argtypes = [vp, dp]
        L.spns_set_spectral.argtypes = [vp, dp]
        L.spns_get_physical.argtypes = [vp, dp]
        L.spns_device_state.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]
        L.spns_stream.argtypes = [vp, C.POINTER(vp)]
        L.spns_kernels_per_step.argtypes = [vp, ip]
        L.spns_last_error.argtypes = [vp]
        L.spns_last_error.restype = C.c_char_p
        L.spns_status_string.argtypes = [i]
        L.spns_status_string.restype = C.c_char_p
        L.spns_fft1d_batch_f64.argtypes = [vp, i, i, i]
        L.spns_profile_begin.argtypes = [vp, i]
        L.spns_profile_read.argtypes = [vp, C.POINTER(C.c_float), i, ip, ip]
        L.spns_profile_kernel_name.argtypes = [vp, i]
        L.spns_profile_kernel_name.restype = C.c_char_p
        L.spns_energy_cascade_noalloc_f64.argtypes = [vp, i, i, i, i, i, i, dp, i, dp, vp]
        sz = C.c_size_t
        L.spns_estimate_device_bytes.argtypes = [C.POINTER(HitArgsC), C.POINTER(sz)]
        L.spns_seed_field.argtypes = [vp, C.c_uint64, d, d]
        L.spns_step_async.argtypes = [vp, i]
        L.spns_query.argtypes = [vp, ip]
        L.spns_synchronize.argtypes = [vp]
        L.spns_checkpoint_bytes.argtypes = [vp, C.POINTER(sz)]
        L.spns_checkpoint_save.argtypes = [vp, vp, sz]
        L.spns_checkpoint_load.argtypes = [vp, vp, sz]
        L.spns_ensemble_create.argtypes = [C.POINTER(vp), i, C.POINTER(vp)]
        L.spns_ensemble_step.argtypes = [vp, i]
        L.spns_ensemble_destroy.argtypes = [vp]
        L.spns_ensemble_last_error.argtypes = [vp]
        L.spns_ensemble_last_error.restype = C.c_char_p
        L.spns_ensemble_set_batched.argtypes = [vp, i]
        L.spns_invariant_spectra.argtypes = [vp, dp]
        L.spns_eddy_viscosity_stats.argtypes = [vp, dp]
        L.spns_autotune.argtypes = [vp, i, ip]
        L.spns_autotune_forget.argtypes = []
        L.spns_set_shapes.argtypes = [vp, ip]
        lp = C.POINTER(C.c_longlong)
        L.spns_slab_block.argtypes = [i, i, i, ip, ip]
        L.spns_slab_create.argtypes = [C.POINTER(HitArgsC), i, i, C.POINTER(vp)]
        L.spns_slab_layout.argtypes = [vp, ip, ip, ip, ip]
        L.spns_slab_phase.argtypes = [vp, i]
        L.spns_slab_exchange.argtypes = [vp, i, lp, lp]
        L.spns_slab_counts.argtypes = [i, i, i, i, i, i, i, lp, lp]
        L.spns_slab_buffers.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(sz), C.POINTER(vp), C.POINTER(sz)]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def fft1d_batch_f64(dev_ptr: int, n: int, batch: int, sign: int) -> None:
    """Batched in-place 1-D FFT of device memory (test building block)."""
    L = lib()
    st = L.spns_fft1d_batch_f64(C.c_void_p(dev_ptr), int(n), int(batch), int(sign))
    if st != 0:
        raise SpnsError(st, L.spns_last_error(None).decode())


def make_args_c(args: HitArgs, *, precision: int = SPNS_FP64, device: int = 0, k41_ranks: int = 1,
                fixed_dt: float = 0.0, eps_forcing: float = 0.0, eps_kmin: int = 1, eps_kmax: int = 2,
                nonlinear_form: int = 0, stream_priority: int = 0) -> HitArgsC:
    """spns_hit_args of a HIT constructor call (src/HIT_LES.h:23-29) plus the extensions."""
    a = HitArgsC()
    for f in ("Nx", "Ny", "Nz", "Mx", "My", "Mz", "Nx_file", "Ny_file", "Nz_file"):
        setattr(a, f, int(getattr(args, f)))
    a.Lx_factor, a.Ly_factor, a.Lz_factor = int(args.Lx), int(args.Ly), int(args.Lz)
    for f in ("nu", "C_Smag", "C_At", "omega_x", "omega_y", "omega_z"):
        setattr(a, f, float(getattr(args, f)))
    a.isReLambda = int(args.isReLambda)
    a.isInitialFieldFromFile = int(args.is_file_init)
    a.isNotCubic = int(args.isNotCubic)
    a.isRotating = int(args.isRotating)
    a.isLES = int(args.isLES)
    a.isComplexConjugateCorrected = int(args.isComplexConjugateCorrected)
    a.isSelfAdaptive = int(args.isSelfAdaptive)
    a.precision, a.device, a.k41_ranks = int(precision), int(device), int(k41_ranks)
    a.fixed_dt, a.eps_forcing = float(fixed_dt), float(eps_forcing)
    a.eps_kmin, a.eps_kmax = int(eps_kmin), int(eps_kmax)
    a.nonlinear_form = int(nonlinear_form)
    a.stream_priority = int(stream_priority)
    return a


def estimate_device_bytes(args: HitArgs, **options) -> int:
    """Device bytes a handle with these arguments allocates (admission against a budget)."""
    L = lib()
    n = C.c_size_t()
    st = L.spns_estimate_device_bytes(C.byref(make_args_c(args, **options)), C.byref(n))
    if st != 0:
        raise SpnsError(st, L.spns_last_error(None).decode())
    return int(n.value)


class HIT:
    """GPU solver with the interface of the reference class ``HIT`` (src/HIT_LES.h:21-246)."""

    def __init__(self, args: HitArgs, file_uvw: Optional[np.ndarray] = None, *, precision: int = SPNS_FP64,
                 device: int = 0, k41_ranks: int = 1, fixed_dt: float = 0.0, eps_forcing: float = 0.0,
                 eps_kmin: int = 1, eps_kmax: int = 2, nonlinear_form: int = 0, stream_priority: int = 0):
        L = lib()
        a = make_args_c(args, precision=precision, device=device, k41_ranks=k41_ranks, fixed_dt=fixed_dt,
                        eps_forcing=eps_forcing, eps_kmin=eps_kmin, eps_kmax=eps_kmax, nonlinear_form=nonlinear_form,
                        stream_priority=stream_priority)
        self.precision = int(precision)
        self.args = args
        fp = None
        if args.is_file_init:
            if file_uvw is None:
                raise SpnsError(-1, "file initial field requested without data")
            self._file = np.ascontiguousarray(file_uvw, dtype=np.float64)
            fp = _dp(self._file)
        h = C.c_void_p()
        st = L.spns_create(C.byref(a), fp, C.byref(h))
        if st != 0:
            raise SpnsError(st, L.spns_last_error(None).decode())
        self._h = h
        self._L = L
        kx, ky, kz = C.c_int(), C.c_int(), C.c_int()
        L.spns_spectral_dims(h, C.byref(kx), C.byref(ky), C.byref(kz))
        self.spectral_shape = (3, ky.value, kx.value, kz.value)
        mx, my, mz = C.c_int(), C.c_int(), C.c_int()
        L.spns_physical_dims(h, C.byref(mx), C.byref(my), C.byref(mz))
        self.physical_shape = (3, mx.value, my.value, mz.value)

    def _ck(self, st):
        if st != 0:
            raise SpnsError(st, self._L.spns_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.spns_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- time step ---
    def New_Fractional_Step_Method(self, nsteps: int = 1):
        self._ck(self._L.spns_step(self._h, int(nsteps)))

    def Recalculate_TimeStep(self):
        self._ck(self._L.spns_recalculate_timestep(self._h))

    def Recalculate_Velocity_Antitransform(self):
        self._ck(self._L.spns_velocity_antitransform(self._h))

    # --- forcing ---
    def Forcing_Energy_Cascade(self, Forced_Ek, last_input_rad, isNullifyMissingEk):
        e = np.ascontiguousarray(Forced_Ek, dtype=np.float64)
        if len(e) < int(last_input_rad) + 1:
            raise SpnsError(-1, "Forced_Ek shorter than last_input_rad+1")
        self._ck(self._L.spns_forcing_energy_cascade(self._h, _dp(e), int(last_input_rad), int(bool(isNullifyMissingEk))))

    def Complex_Conjugate_Correction(self):
        self._ck(self._L.spns_complex_conjugate_correction(self._h))

    def Forcing_Reynolds_Lambda(self, ReLambda):
        self._ck(self._L.spns_forcing_reynolds_lambda(self._h, float(ReLambda)))

    # --- integrals ---
    def Recalculate_Reynolds_Lambda(self) -> float:
        out = C.c_double()
        self._ck(self._L.spns_recalculate_reynolds_lambda(self._h, C.byref(out)))
        return out.value

    def Recalculate_Energy(self) -> float:
        out = C.c_double()
        self._ck(self._L.spns_recalculate_energy(self._h, C.byref(out)))
        return out.value

    def Recalculate_Enstrophy(self) -> float:
        out = C.c_double()
        self._ck(self._L.spns_recalculate_enstrophy(self._h, C.byref(out)))
        return out.value

    def Recalculate_Energy_Cascade(self) -> np.ndarray:
        ek = np.zeros(self.getlast_rad_max() + 1)
        tot = C.c_double()
        self._ck(self._L.spns_recalculate_energy_cascade(self._h, _dp(ek), C.byref(tot)))
        return ek

    def Recalculate_Invariants_Distribution(self, filenames=None) -> np.ndarray:
        """Spectra [5][last_rad_max+1] of Q_G, Q_S, R_G, R_S, V^2 (src/HIT_LES.cpp:1297-1319);
        with five file names, each is written as ``K<TAB>value`` lines (src/HIT_LES.cpp:1180-1187)."""
        out = np.zeros((5, self.getlast_rad_max() + 1))
        self._ck(self._L.spns_invariant_spectra(self._h, _dp(out)))
        if filenames is not None:
            for name, sp in zip(filenames, out):
                with open(name, "w") as fh:
                    for K, v in enumerate(sp):
                        fh.write(f"{K}\t{v:g}\n")
        return out

    def Check_PhysFour_Energy(self, atol: float = 1e-13):
        ok, d1, d2 = C.c_int(), C.c_double(), C.c_double()
        self._ck(self._L.spns_check_physfour_energy(self._h, float(atol), C.byref(ok), C.byref(d1), C.byref(d2)))
        return bool(ok.value), d1.value, d2.value

    # --- getters / setters ---
    def scalars(self) -> ScalarsC:
        s = ScalarsC()
        self._ck(self._L.spns_get_scalars(self._h, C.byref(s)))
        return s

    def gettime(self): return self.scalars().time
    def getAt(self): return self.scalars().At
    def getnu(self): return self.scalars().nu
    def getEk_Tot(self): return self.scalars().Ek_Tot
    def getOk_Tot(self): return self.scalars().Ok_Tot
    def getReLambda(self): return self.scalars().ReLambda
    def getEk_init(self): return self.scalars().Ek_init
    def getEk_init_file(self): return self.scalars().Ek_init_file
    def getEnstrophy_init_file(self): return self.scalars().Enstrophy_init_file
    def getkappa(self): return self.scalars().kappa
    def getlast_rad(self): return int(self.scalars().last_rad)
    def getlast_rad_max(self): return int(self.scalars().last_rad_max)
    def getNx(self): return self.args.Nx
    def getNy(self): return self.args.Ny
    def getNz(self): return self.args.Nz

    def setnu(self, nu):
        self._ck(self._L.spns_set_nu(self._h, float(nu)))

    # --- state ---
    def get_compact(self) -> np.ndarray:
        out = np.zeros(self.spectral_shape, dtype=np.complex128)
        self._ck(self._L.spns_get_spectral(self._h, _dp(out.view(np.float64))))
        return out

    def set_compact(self, uvw):
        buf = np.ascontiguousarray(uvw, dtype=np.complex128)
        if buf.shape != self.spectral_shape:
            raise SpnsError(-1, f"spectral state shape {buf.shape} != {self.spectral_shape}")
        self._ck(self._L.spns_set_spectral(self._h, _dp(buf.view(np.float64))))

    def get_physical(self) -> np.ndarray:
        out = np.zeros(self.physical_shape, dtype=np.float64)
        self._ck(self._L.spns_get_physical(self._h, _dp(out)))
        return out

    def kernels_per_step(self) -> int:
        n = C.c_int()
        self._ck(self._L.spns_kernels_per_step(self._h, C.byref(n)))
        return n.value

    def eddy_viscosity_stats(self) -> np.ndarray:
        """Mean, rms and maximum over the grid of nu_t (src/HIT_LES.cpp:130-142) of the current state."""
        out = np.zeros(3)
        self._ck(self._L.spns_eddy_viscosity_stats(self._h, _dp(out)))
        return out

    # --- launch-shape autotuner ---
    def autotune(self, steps: int = 3):
        """Times the default and the alternate launch shape of each pass on this box
        (spns_autotune) and keeps the faster; the state is left as it was.  Returns
        the choice per pass K1..K5 (0 default, 1 alternate)."""
        ch = (C.c_int * 5)()
        self._ck(self._L.spns_autotune(self._h, int(steps), ch))
        return list(ch)

    def set_shapes(self, choice):
        ch = (C.c_int * 5)(*[int(x) for x in choice])
        self._ck(self._L.spns_set_shapes(self._h, ch))

    def profile_begin(self, max_steps: int):
        self._ck(self._L.spns_profile_begin(self._h, int(max_steps)))

    def profile_read(self, max_steps: int):
        """Per-kernel durations (ms) of the profiled steps: (names, array[steps, kernels])."""
        cap = int(max_steps) * 16
        buf = (C.c_float * cap)()
        nk, ns = C.c_int(), C.c_int()
        self._ck(self._L.spns_profile_read(self._h, buf, cap, C.byref(nk), C.byref(ns)))
        names = [self._L.spns_profile_kernel_name(self._h, i).decode() for i in range(nk.value)]
        arr = np.frombuffer(buf, dtype=np.float32, count=nk.value * ns.value).reshape(ns.value, nk.value).copy()
        return names, arr

    # --- extensions: seeded field, asynchronous stepping, checkpoints ---
    def seed_field(self, seed: int, kp: float = 4.0, urms: float = 1.0):
        """Seeded Philox field (spns_seed_field); then refresh the grid velocity and the time step."""
        self._ck(self._L.spns_seed_field(self._h, int(seed) & 0xFFFFFFFFFFFFFFFF, float(kp), float(urms)))
        self.Recalculate_Velocity_Antitransform()
        self.Recalculate_TimeStep()

    def step_async(self, nsteps: int = 1):
        self._ck(self._L.spns_step_async(self._h, int(nsteps)))

    def query(self) -> bool:
        idle = C.c_int()
        self._ck(self._L.spns_query(self._h, C.byref(idle)))
        return bool(idle.value)

    def synchronize(self):
        self._ck(self._L.spns_synchronize(self._h))

    def checkpoint_save(self) -> bytes:
        n = C.c_size_t()
        self._ck(self._L.spns_checkpoint_bytes(self._h, C.byref(n)))
        buf = (C.c_char * n.value)()
        self._ck(self._L.spns_checkpoint_save(self._h, buf, n.value))
        return bytes(buf)

    def checkpoint_load(self, data: bytes):
        buf = (C.c_char * len(data)).from_buffer_copy(data)
        self._ck(self._L.spns_checkpoint_load(self._h, buf, len(data)))

    def stream_handle(self) -> int:
        p = C.c_void_p()
        self._ck(self._L.spns_stream(self._h, C.byref(p)))
        return p.value or 0


class Ensemble:
    """Members advanced together, one CUDA graph per step (spns_ensemble_*)."""

    def __init__(self, members, batched: bool = False):
        L = lib()
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m._h for m in self.members])
        e = C.c_void_p()
        st = L.spns_ensemble_create(arr, len(self.members), C.byref(e))
        if st != 0:
            raise SpnsError(st, L.spns_last_error(None).decode())
        self._e, self._L = e, L
        if batched:
            L.spns_ensemble_set_batched(e, 1)

    def step(self, nsteps: int = 1):
        st = self._L.spns_ensemble_step(self._e, int(nsteps))
        if st != 0:
            raise SpnsError(st, self._L.spns_ensemble_last_error(self._e).decode())

    def close(self):
        if getattr(self, "_e", None):
            self._L.spns_ensemble_destroy(self._e)
            self._e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
