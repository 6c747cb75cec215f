"""Host restatement of the device seeded field (no GPU): Philox4x32-10 against
the published known-answer vectors of its authors (Salmon et al., SC'11,
Random123 distribution), and the properties of the seeded spectrum."""
import numpy as np

from spns_b200.fields import energy_spectrum, philox4x32_10, philox_spectral_field

KAT = [  # (counter, key, output), 32-bit words
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]


def test_philox_known_answers():
    for ctr, key, out in KAT:
        r = philox4x32_10(*[np.array([v], dtype=np.uint64) for v in ctr], *key)
        assert tuple(int(x[0]) for x in r) == out


def test_seeded_field_spectrum_and_symmetry():
    N, kp = 32, 3.0
    U = philox_spectral_field(N, N, N, kp=kp, seed=99)
    E = energy_spectrum(U, N, N, N)
    assert abs(E.sum() - 1.5) < 1e-12
    K = np.arange(len(E), dtype=float)
    shape = np.where((K >= 1) & (E > 0), K ** 4 * np.exp(-2 * (K / kp) ** 2), 0.0)
    m = shape > 1e-12 * shape.max()
    assert np.allclose(E[m] / E[m].sum(), shape[m] / shape[m].sum(), rtol=1e-10)
    # solenoidal: k . u = 0
    h = N // 2
    k = np.where(np.arange(N + 1) <= h, np.arange(N + 1), np.arange(N + 1) - (N + 1)).astype(float)
    KY, KX, KZ = np.meshgrid(k, k, np.arange(h + 1, dtype=float), indexing="ij")
    assert np.max(np.abs(KX * U[0] + KY * U[1] + KZ * U[2])) < 1e-13 * np.max(np.abs(U))
    # Hermitian kz=0 plane: u(-k1,-k2,0) = conj u(k1,k2,0)
    P = U[:, :, :, 0]
    mirror = P[:, (-np.arange(N + 1)) % (N + 1)][:, :, (-np.arange(N + 1)) % (N + 1)]
    assert np.max(np.abs(P - np.conj(mirror))) < 1e-15
    # the seed matters, the call does not
    assert np.array_equal(U, philox_spectral_field(N, N, N, kp=kp, seed=99))
    assert not np.allclose(U, philox_spectral_field(N, N, N, kp=kp, seed=98))
