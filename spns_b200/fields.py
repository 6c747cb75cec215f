"""Seeded synthetic initial fields in the compact spectral layout of libspns.

Solenoidal random-phase velocity with the model spectrum
E(K) = C * K^4 * exp(-2 (K/kp)^2), scaled so that the energy integral of the
reference (shell sums with the conjugate weight of src/HIT_LES.cpp:1137-1214)
equals 3/2, i.e. u_rms = 1.  The reference has no such generator (its own
initial fields are the K41 draw of src/HIT_LES.cpp:502-540 and input files), so
this is the synthetic stand-in for the seeded fields of the benchmark configs.

Layout: complex128 array [3][Ky][Kx][Kz]; iy -> k2 = iy (iy <= N/2) or iy - Ky,
same for ix, kz = 0..N/2.  Modes with some |k_i| > (N-1)/2 are zero, as after
the reference's file truncation (src/HIT_LES.cpp:743).  Each ky plane draws
from its own seed sequence, so the field does not depend on chunking.
"""
from __future__ import annotations

import numpy as np


def _axis(n_half: int, K: int, scale: int = 1) -> np.ndarray:
    i = np.arange(K)
    return scale * np.where(i <= n_half, i, i - K)


def seeded_spectral_field(Nx: int, Ny: int, Nz: int, kp: float = 4.0, seed: int = 0, urms: float = 1.0,
                          scale=(1, 1, 1)) -> np.ndarray:
    hx, hy, hz = Nx // 2, Ny // 2, Nz // 2
    Kx, Ky, Kz = 2 * hx + 1, 2 * hy + 1, hz + 1
    sx, sy, sz = scale
    kx = _axis(hx, Kx, sx).astype(np.float64)
    kz = (sz * np.arange(Kz)).astype(np.float64)
    mx = _axis(hx, Kx)
    mz = np.arange(Kz)
    U = np.zeros((3, Ky, Kx, Kz), dtype=np.complex128)
    lim_x, lim_y, lim_z = (Nx - 1) // 2, (Ny - 1) // 2, (Nz - 1) // 2
    nbins = int(np.ceil(np.sqrt((sx * hx) ** 2 + (sy * hy) ** 2 + (sz * hz) ** 2))) + 2
    Eraw = np.zeros(nbins)
    for iy in range(Ky):
        my = iy if iy <= hy else iy - Ky
        ky = float(sy * my)
        rng = np.random.default_rng(np.random.SeedSequence([int(seed), iy]))
        g = rng.standard_normal((3, Kx, Kz, 2))
        u = g[..., 0] + 1j * g[..., 1]
        KX, KZ = np.meshgrid(kx, kz, indexing="ij")
        k2 = KX * KX + ky * ky + KZ * KZ
        keep = (np.abs(mx)[:, None] <= lim_x) & (abs(my) <= lim_y) & (mz[None, :] <= lim_z) & (k2 > 0)
        safe = np.where(k2 > 0, k2, 1.0)
        div = (KX * u[0] + ky * u[1] + KZ * u[2]) / safe
        u[0] -= div * KX
        u[1] -= div * ky
        u[2] -= div * KZ
        u *= keep[None]
        U[:, iy] = u
    # Hermitian kz=0 plane: u(-k1,-k2,0) = conj(u(k1,k2,0)) for the half k1<0 or (k1=0, k2<0)
    MY = _axis(hy, Ky)[:, None]
    MX = _axis(hx, Kx)[None, :]
    neg = (MX < 0) | ((MX == 0) & (MY < 0))
    iy_src = np.where(-MY >= 0, -MY, -MY + Ky)
    ix_src = np.where(-MX >= 0, -MX, -MX + Kx)
    for c in range(3):
        plane = U[c, :, :, 0]
        src = np.conj(plane[iy_src, ix_src])
        plane[neg] = src[neg]
        U[c, :, :, 0] = plane
    U[:, 0, 0, 0] = 0.0
    # shell energies with the reference's conjugate weight
    K, w = shell_index(Nx, Ny, Nz, scale)
    e = 0.5 * np.sum(np.abs(U) ** 2, axis=0) * w
    Eraw = np.bincount(K.ravel(), weights=e.ravel(), minlength=nbins)
    Ks = np.arange(len(Eraw), dtype=np.float64)
    target = Ks ** 4 * np.exp(-2.0 * (Ks / kp) ** 2)
    target[0] = 0.0
    target *= np.where(Eraw > 0, 1.0, 0.0)
    target *= (1.5 * urms ** 2) / target.sum()
    fac = np.sqrt(np.divide(target, Eraw, out=np.zeros_like(target), where=Eraw > 0))
    U *= fac[K][None]
    return U


def shell_index(Nx: int, Ny: int, Nz: int, scale=(1, 1, 1)):
    """K=round(|k|) and the conjugate weight (2 for kz>0) of every compact mode."""
    hx, hy, hz = Nx // 2, Ny // 2, Nz // 2
    Kx, Ky, Kz = 2 * hx + 1, 2 * hy + 1, hz + 1
    kx = _axis(hx, Kx, scale[0]).astype(np.float64)
    ky = _axis(hy, Ky, scale[1]).astype(np.float64)
    kz = (scale[2] * np.arange(Kz)).astype(np.float64)
    k2 = ky[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
    K = np.rint(np.sqrt(k2)).astype(np.int64)
    w = np.where(np.arange(Kz)[None, None, :] > 0, 2.0, 1.0) * np.ones_like(k2)
    return K, w


def energy_spectrum(U: np.ndarray, Nx: int, Ny: int, Nz: int, scale=(1, 1, 1), nbins=None) -> np.ndarray:
    """E(K) of a compact spectral field (the reference's shell integral)."""
    K, w = shell_index(Nx, Ny, Nz, scale)
    e = 0.5 * np.sum(np.abs(U) ** 2, axis=0) * w
    n = nbins or int(K.max()) + 1
    return np.bincount(K.ravel(), weights=e.ravel(), minlength=n)[:n]


# ---------------------------------------------------------------------------
# Philox4x32-10 seeded field: the host restatement of the device generator of
# libspns (spns_seed_field), used to check it.  Philox4x32-10 is the published
# counter-based generator of Salmon, Moraes, Dror and Shaw (SC'11).
# ---------------------------------------------------------------------------
_M32 = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox4x32-10 over uint64 arrays holding 32-bit words."""
    c0, c1, c2, c3 = (np.asarray(v, dtype=np.uint64) & _M32 for v in (c0, c1, c2, c3))
    k0 = np.uint64(int(k0) & 0xFFFFFFFF)
    k1 = np.uint64(int(k1) & 0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c0
        p1 = np.uint64(0xCD9E8D57) * c2
        c0, c1, c2, c3 = (((p1 >> np.uint64(32)) ^ c1 ^ k0) & _M32, p1 & _M32,
                          ((p0 >> np.uint64(32)) ^ c3 ^ k1) & _M32, p0 & _M32)
        k0 = (k0 + np.uint64(0x9E3779B9)) & _M32
        k1 = (k1 + np.uint64(0xBB67AE85)) & _M32
    return c0, c1, c2, c3


def _philox_normals(idx, draw, seed):
    r = philox4x32_10(idx & 0xFFFFFFFF, idx >> np.uint64(32), np.full_like(idx, draw), np.zeros_like(idx),
                      seed & 0xFFFFFFFF, seed >> 32)
    u0 = ((r[0] >> np.uint64(5)) * np.uint64(1 << 26) + (r[1] >> np.uint64(6))).astype(np.float64) * 2.0 ** -53
    u1 = ((r[2] >> np.uint64(5)) * np.uint64(1 << 26) + (r[3] >> np.uint64(6))).astype(np.float64) * 2.0 ** -53
    rad = np.sqrt(-2.0 * np.log(1.0 - u0))
    return rad * np.cos(2.0 * np.pi * u1), rad * np.sin(2.0 * np.pi * u1)


def philox_spectral_field(Nx: int, Ny: int, Nz: int, kp: float = 4.0, seed: int = 0, urms: float = 1.0,
                          scale=(1, 1, 1)) -> np.ndarray:
    """The field spns_seed_field writes, computed on the host ([3][Ky][Kx][Kz] complex128)."""
    hx, hy, hz = Nx // 2, Ny // 2, Nz // 2
    Kx, Ky, Kz = 2 * hx + 1, 2 * hy + 1, hz + 1
    sx, sy, sz = scale
    lim_x, lim_y, lim_z = (Nx - 1) // 2, (Ny - 1) // 2, (Nz - 1) // 2
    iy, ix, kz = np.meshgrid(np.arange(Ky), np.arange(Kx), np.arange(Kz), indexing="ij")
    m1 = np.where(ix <= hx, ix, ix - Kx)
    m2 = np.where(iy <= hy, iy, iy - Ky)
    k1, k2, k3 = float(sx) * m1, float(sy) * m2, float(sz) * kz
    k2s = k1 * k1 + k2 * k2 + k3 * k3
    keep = (np.abs(m1) <= lim_x) & (np.abs(m2) <= lim_y) & (kz <= lim_z) & (k2s > 0)
    mirror = (kz == 0) & ((m1 < 0) | ((m1 == 0) & (m2 < 0)))
    p1, p2 = -m1, -m2
    src_mirror = ((np.where(p2 >= 0, p2, p2 + Ky) * Kx + np.where(p1 >= 0, p1, p1 + Kx)) * Kz)
    idx = (iy * Kx + ix) * Kz + kz
    src = np.where(mirror, src_mirror, idx).astype(np.uint64)
    re, im = [], []
    for c in range(3):
        a, b = _philox_normals(src, c, int(seed))
        re.append(a)
        im.append(b)
    kk = [np.where(mirror, -k1, k1), np.where(mirror, -k2, k2), k3]
    safe = np.where(k2s > 0, k2s, 1.0)
    dr = (kk[0] * re[0] + kk[1] * re[1] + kk[2] * re[2]) / safe
    di = (kk[0] * im[0] + kk[1] * im[1] + kk[2] * im[2]) / safe
    U = np.zeros((3, Ky, Kx, Kz), dtype=np.complex128)
    for c in range(3):
        r = re[c] - dr * kk[c]
        i = im[c] - di * kk[c]
        i = np.where(mirror, -i, i)
        U[c] = np.where(keep, r + 1j * i, 0.0)
    K, w = shell_index(Nx, Ny, Nz, scale)
    last_rad_max = int(np.ceil(np.sqrt((sx * hx) ** 2 + (sy * hy) ** 2 + (sz * hz) ** 2)))
    e = 0.5 * np.sum(np.abs(U) ** 2, axis=0) * w
    E = np.bincount(K.ravel(), weights=e.ravel(), minlength=last_rad_max + 1)[:last_rad_max + 1]
    Ks = np.arange(last_rad_max + 1, dtype=np.float64)
    shape = np.where((Ks >= 1) & (E > 0), Ks ** 4 * np.exp(-2.0 * (Ks / kp) ** 2), 0.0)
    target = shape * (1.5 * urms * urms) / shape.sum()
    fac = np.sqrt(np.divide(target, E, out=np.zeros_like(target), where=E > 0))
    return U * fac[np.minimum(K, last_rad_max)][None]
