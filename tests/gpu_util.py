"""Helpers for the GPU parity tests (GPU solver vs the CPU oracle)."""
import numpy as np

from spns_b200.params import HitArgs


def make_args(N, nu=1e-2, C_At=0.5, Ns=None, L=(1, 1, 1), rotating=None, les=0.0, self_adaptive=False,
              conj=False, relambda=False):
    Nx, Ny, Nz = Ns or (N, N, N)
    Lx, Ly, Lz = L
    ex = lambda n, f: n * f if n % 2 == 0 else (n - 1) * f + 1  # noqa: E731
    M = lambda n: (3 * n) // 2  # noqa: E731
    om = rotating or (0.0, 0.0, 0.0)
    return HitArgs(Nx=ex(Nx, Lx), Ny=ex(Ny, Ly), Nz=ex(Nz, Lz), Mx=ex(M(Nx), Lx), My=ex(M(Ny), Ly), Mz=ex(M(Nz), Lz),
                   nu=nu, C_Smag=les, C_At=C_At, Lx=Lx, Ly=Ly, Lz=Lz, omega_x=om[0], omega_y=om[1], omega_z=om[2],
                   Nx_file=-1, Ny_file=-1, Nz_file=-1, isReLambda=relambda, isInitialFieldFromBinaryFile=False,
                   isInitialFieldFromASCIIFile=False, isNotCubic=(L != (1, 1, 1)), isRotating=rotating is not None,
                   isLES=les > 0, isComplexConjugateCorrected=conj, isSelfAdaptive=self_adaptive)


def oracle_compact_to_true(U, args):
    """Oracle compact state (expanded wavenumbers) -> compact state of the true grid."""
    Lx, Ly, Lz = args.Lx, args.Ly, args.Lz
    hx, hy, hz = args.Nx // 2, args.Ny // 2, args.Nz // 2
    Kx, Ky = 2 * hx + 1, 2 * hy + 1
    act = lambda n, f: n // f if n % 2 == 0 else (n - 1) // f + 1  # noqa: E731
    gx, gy, gz = act(args.Nx, Lx) // 2, act(args.Ny, Ly) // 2, act(args.Nz, Lz) // 2
    gKx, gKy = 2 * gx + 1, 2 * gy + 1
    m1 = np.where(np.arange(gKx) <= gx, np.arange(gKx), np.arange(gKx) - gKx)
    m2 = np.where(np.arange(gKy) <= gy, np.arange(gKy), np.arange(gKy) - gKy)
    ix = np.where(m1 >= 0, Lx * m1, Lx * m1 + Kx)
    iy = np.where(m2 >= 0, Ly * m2, Ly * m2 + Ky)
    iz = Lz * np.arange(gz + 1)
    return U[:, iy][:, :, ix][:, :, :, iz]


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
