"""Parameters file reader and the driver's derivations, as the reference driver does them.

The reference keeps its key/value parameters file (parsed by ``CParamInitManager``,
src/parser.cpp:451-484) and derives the ``HIT`` constructor arguments in
src/MAIN.cpp:117-318.  This module restates both so that a run configured by the
reference's own parameters file reaches the GPU solver with the same arguments.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field, asdict
from typing import Dict, Optional

_INT_KEYS = {
    "Nx", "Ny", "Nz", "Reynolds_lambda_Freq", "Velocity_Physical", "Velocity_Fourier", "Energy_Cascade",
    "VelGradInv_Spectra", "Velocity_Phys_Freq", "Velocity_Four_Freq", "Energy_Cascade_Freq",
    "VelGradInv_Spectra_Freq", "Nx_file", "Ny_file", "Nz_file", "Last_K", "Nullify_MissingK", "Lx", "Ly", "Lz",
    "SelfAdaptiveTimestep", "ComplexConjugateCorrection", "OMP_Threads",
}
_FLOAT_KEYS = {"nu", "Reynolds_lambda", "Final_Time", "Final_Forced_Time", "omega_x", "omega_y", "omega_z",
               "C_Smag", "C_At"}
_WORD_KEYS = {"Velocity_Phys_Folder", "Velocity_Four_Folder", "Spectra_Folder", "ASCII_Input_Filename",
              "Binary_Input_Filename", "InputEkFilename"}
_REQUIRED = ("Nx", "Ny", "Nz", "Final_Time")


class ParamsError(ValueError):
    """Raised where the reference driver calls ``crash`` on a bad parameters file."""


def read_params(path: str) -> Dict[str, object]:
    """Key/value reader for the reference's parameters format ('#' starts a comment)."""
    out: Dict[str, object] = {}
    with open(path, "r", errors="replace") as fh:
        for line in fh:
            line = line.split("#", 1)[0].strip()
            if not line:
                continue
            words = line.split()
            if len(words) < 2:
                continue
            key, val = words[0], words[1]
            if key in _INT_KEYS:
                out[key] = int(val)
            elif key in _FLOAT_KEYS:
                out[key] = float(val)
            elif key in _WORD_KEYS:
                out[key] = val
    for k in _REQUIRED:
        if k not in out:
            raise ParamsError(f"Parameter {k} is not set!")
    return out


def _lcm(a: int, b: int) -> int:
    return a * b // math.gcd(a, b)


def _actual(n: int, L: int) -> int:
    return n // L if n % 2 == 0 else (n - 1) // L + 1


@dataclass
class HitArgs:
    """Arguments of the ``HIT`` constructor (src/HIT_LES.h:23-29) plus driver flags."""
    Nx: int
    Ny: int
    Nz: int
    Mx: int
    My: int
    Mz: int
    nu: float
    C_Smag: float
    C_At: float
    Lx: int
    Ly: int
    Lz: int
    omega_x: float
    omega_y: float
    omega_z: float
    Nx_file: int
    Ny_file: int
    Nz_file: int
    isReLambda: bool
    isInitialFieldFromBinaryFile: bool
    isInitialFieldFromASCIIFile: bool
    isNotCubic: bool
    isRotating: bool
    isLES: bool
    isComplexConjugateCorrected: bool
    isSelfAdaptive: bool
    # driver-level settings (src/MAIN.cpp)
    ReLambda: float = 0.0
    isReLambda_iter: bool = False
    ReLambda_Freq: int = 0
    Final_Time: float = 0.0
    isForcedEk: bool = False
    isNullifyMissingEk: bool = False
    last_input_rad: int = 0
    Final_Forced_Time: float = 0.0
    EkFilename: Optional[str] = None
    ASCII_Input_Filename: Optional[str] = None
    Binary_Input_Filename: Optional[str] = None
    OMP_Threads: int = 1

    @property
    def is_file_init(self) -> bool:
        return self.isInitialFieldFromBinaryFile or self.isInitialFieldFromASCIIFile

    def actual_file_dims(self):
        return (_actual(self.Nx_file, self.Lx), _actual(self.Ny_file, self.Ly), _actual(self.Nz_file, self.Lz))

    def as_dict(self):
        return asdict(self)


def derive_hit_args(P: Dict[str, object], base_dir: str = ".") -> HitArgs:
    """src/MAIN.cpp:174-318: flags, 3/2 grid, length-factor expansion."""
    isset = lambda k: k in P  # noqa: E731
    if isset("nu") and isset("Reynolds_lambda"):
        raise ParamsError("Kinematic viscosity and Reynolds lambda cannot be defined simoultaniously!!!")
    if not isset("nu") and not isset("Reynolds_lambda"):
        raise ParamsError("Either kinematic viscosity or Reynolds lambda has to be defined!!!")
    Nx, Ny, Nz = int(P["Nx"]), int(P["Ny"]), int(P["Nz"])
    Mx, My, Mz = (3 * Nx) // 2, (3 * Ny) // 2, (3 * Nz) // 2
    isReLambda = isset("Reynolds_lambda")
    RL_freq = int(P.get("Reynolds_lambda_Freq", 0))
    isReLambda_iter = isReLambda and isset("Reynolds_lambda_Freq") and RL_freq > 0
    Nx_file = Ny_file = Nz_file = -1
    isBin = isAsc = False
    if isset("Nx_file") and isset("Ny_file") and isset("Nz_file"):
        Nx_file, Ny_file, Nz_file = int(P["Nx_file"]), int(P["Ny_file"]), int(P["Nz_file"])
        if isset("Binary_Input_Filename"):
            isBin = True
            if isset("ASCII_Input_Filename"):
                raise ParamsError("both a binary and an ASCII input file have been defined")
        elif isset("ASCII_Input_Filename"):
            isAsc = True
    if not (isBin or isAsc):
        Nx_file = Ny_file = Nz_file = -1
    isForcedEk = isset("InputEkFilename") and isset("Last_K") and isset("Final_Forced_Time")
    Final_Time = float(P["Final_Time"])
    Final_Forced_Time = float(P.get("Final_Forced_Time", 0.0))
    isNullify = False
    if isForcedEk:
        isNullify = bool(isset("Nullify_MissingK") and int(P["Nullify_MissingK"]))
        Final_Forced_Time = Final_Forced_Time if Final_Forced_Time > 0.0 else Final_Time
    Lx, Ly, Lz = int(P.get("Lx", 1)), int(P.get("Ly", 1)), int(P.get("Lz", 1))
    isNotCubic = False
    if (isset("Lx") and Lx > 1) or (isset("Ly") and Ly > 1) or (isset("Lz") and Lz > 1):
        l = _lcm(Lx, _lcm(Ly, Lz))
        Lx, Ly, Lz = l // Lx, l // Ly, l // Lz
        if Lx > 1 or Ly > 1 or Lz > 1:
            isNotCubic = True
            Mx = Mx + 1 if (Lx > 1 and Mx % 2 != 0) else Mx
            My = My + 1 if (Ly > 1 and My % 2 != 0) else My
            Mz = Mz + 1 if (Lz > 1 and Mz % 2 != 0) else Mz
            ex = lambda n, L: n * L if n % 2 == 0 else (n - 1) * L + 1  # noqa: E731
            Nx, Ny, Nz = ex(Nx, Lx), ex(Ny, Ly), ex(Nz, Lz)
            Mx, My, Mz = ex(Mx, Lx), ex(My, Ly), ex(Mz, Lz)
            if isAsc or isBin:
                Nx_file, Ny_file, Nz_file = ex(Nx_file, Lx), ex(Ny_file, Ly), ex(Nz_file, Lz)
    else:
        Lx = Ly = Lz = 1
    ox, oy, oz = float(P.get("omega_x", 0.0)), float(P.get("omega_y", 0.0)), float(P.get("omega_z", 0.0))
    isRotating = abs(ox) > 0.0 or abs(oy) > 0.0 or abs(oz) > 0.0
    C_Smag = float(P.get("C_Smag", 0.0))
    isLES = C_Smag > 0
    isSelf = int(P.get("SelfAdaptiveTimestep", 0)) == 1
    isConj = int(P.get("ComplexConjugateCorrection", 0)) == 1
    resolve = lambda f: None if f is None else (f if os.path.isabs(f) else os.path.join(base_dir, f))  # noqa: E731
    return HitArgs(
        Nx=Nx, Ny=Ny, Nz=Nz, Mx=Mx, My=My, Mz=Mz,
        nu=float(P.get("nu", 0.0)), C_Smag=C_Smag, C_At=float(P.get("C_At", 1.0)),
        Lx=Lx, Ly=Ly, Lz=Lz, omega_x=ox, omega_y=oy, omega_z=oz,
        Nx_file=Nx_file, Ny_file=Ny_file, Nz_file=Nz_file,
        isReLambda=isReLambda, isInitialFieldFromBinaryFile=isBin, isInitialFieldFromASCIIFile=isAsc,
        isNotCubic=isNotCubic, isRotating=isRotating, isLES=isLES,
        isComplexConjugateCorrected=isConj, isSelfAdaptive=isSelf,
        ReLambda=float(P.get("Reynolds_lambda", 0.0)), isReLambda_iter=isReLambda_iter, ReLambda_Freq=RL_freq,
        Final_Time=Final_Time, isForcedEk=isForcedEk, isNullifyMissingEk=isNullify,
        last_input_rad=int(P.get("Last_K", 0)), Final_Forced_Time=Final_Forced_Time,
        EkFilename=resolve(P.get("InputEkFilename")),
        ASCII_Input_Filename=resolve(P.get("ASCII_Input_Filename")),
        Binary_Input_Filename=resolve(P.get("Binary_Input_Filename")),
        OMP_Threads=int(P.get("OMP_Threads", 1)),
    )


def read_initial_field(args: HitArgs, path: Optional[str] = None):
    """Initial physical velocity as the reference reads it (src/HIT_LES.cpp:604-709).

    Returns float64 array [3, ActualNx_file, ActualNy_file, ActualNz_file].  Binary
    files hold the three components one after another in float64 or float32;
    ASCII files hold one ``u v w`` row per point.
    """
    import numpy as np
    nx, ny, nz = args.actual_file_dims()
    n = nx * ny * nz
    if args.isInitialFieldFromBinaryFile:
        path = path or args.Binary_Input_Filename
        size = os.path.getsize(path)
        if size == 8 * 3 * n:
            data = np.fromfile(path, dtype="<f8")
        elif size == 4 * 3 * n:
            data = np.fromfile(path, dtype="<f4").astype(np.float64)
        else:
            raise ParamsError(f'Incorrect size of "{path}": {size} bytes instead of {4*3*n} or {8*3*n}')
        return data.reshape(3, nx, ny, nz)
    if args.isInitialFieldFromASCIIFile:
        path = path or args.ASCII_Input_Filename
        vals = np.loadtxt(path, dtype=np.float64, max_rows=n).reshape(n, 3)
        return np.ascontiguousarray(vals.T.reshape(3, nx, ny, nz))
    return None


def read_forced_ek(path: str, last_k: int):
    """src/MAIN.cpp:564-592: (K, E) pairs into E[0..Last_K]; E[0] must stay 0."""
    import numpy as np
    Ek = np.zeros(last_k + 1, dtype=np.float64)
    with open(path) as fh:
        toks = fh.read().split()
    for i in range(0, len(toks) - 1, 2):
        K, val = int(toks[i]), float(toks[i + 1])
        if K < 0 or K > last_k:
            raise ParamsError(f"Read_Ek_Input_File(): K={K} out of range [0, {last_k}] in \"{path}\"")
        Ek[K] = val
    if Ek[0] > 0.0:
        raise ParamsError("Read_Ek_Input_File(): Ek_input[0] must be 0")
    return Ek
