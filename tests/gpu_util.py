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


def broadband_field(Nx, Ny, Nz, seed=0, slope=-5.0 / 3.0, urms=1.0):
    """Solenoidal field with energy in EVERY retained mode, the +-N/2 planes included.

    Complex Gaussian draws per mode, projected onto k-perp, Hermitian on kz=0 (the
    half m1<0 or m1=0, m2<0 mirrors its partner), shell amplitude ~ K^(slope/2 - 1)
    so that E(K) ~ K^slope, scaled to u_rms = urms with the shell-sum weights of the
    reference (kz>0 counted twice).  Every FFT input row of every pass is then
    non-zero, so a parity check exercises the whole transform at its length.
    Layout [3][Ky][Kx][Kz] as the compact state of libspns and the oracle."""
    hx, hy, hz = Nx // 2, Ny // 2, Nz // 2
    Kx, Ky, Kz = 2 * hx + 1, 2 * hy + 1, hz + 1
    ax = lambda h, K: np.where(np.arange(K) <= h, np.arange(K), np.arange(K) - K)  # noqa: E731
    m1, m2, m3 = ax(hx, Kx), ax(hy, Ky), np.arange(Kz)
    K2, K1, K3 = np.meshgrid(m2.astype(float), m1.astype(float), m3.astype(float), indexing="ij")
    k2 = K1 * K1 + K2 * K2 + K3 * K3
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((3, Ky, Kx, Kz)) + 1j * rng.standard_normal((3, Ky, Kx, Kz))
    safe = np.where(k2 > 0, k2, 1.0)
    div = (K1 * u[0] + K2 * u[1] + K3 * u[2]) / safe
    u[0] -= div * K1
    u[1] -= div * K2
    u[2] -= div * K3
    u *= np.where(k2 > 0, safe ** (0.5 * (slope / 2.0 - 1.0)), 0.0)[None]
    MY, MX = m2[:, None], m1[None, :]
    neg = (MX < 0) | ((MX == 0) & (MY < 0))
    iy_src = np.where(-MY >= 0, -MY, -MY + Ky) + 0 * MX
    ix_src = np.where(-MX >= 0, -MX, -MX + Kx) + 0 * MY
    for c in range(3):
        plane = u[c, :, :, 0]
        plane[neg] = np.conj(plane[iy_src[neg], ix_src[neg]])
        u[c, :, :, 0] = plane
    w = np.where(np.arange(Kz) > 0, 2.0, 1.0)[None, None, None, :]
    e = 0.5 * np.sum(w * np.abs(u) ** 2)
    return u * np.sqrt(1.5 * urms * urms / e)
