"""Deterministic test inputs, independent of any library's random streams.

splitmix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number
generators", 2014) in numpy uint64 arithmetic: the same bits on every
platform, so committed fixtures can store outputs only.
"""
import numpy as np

_G = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def uniform(seed, n):
    """n doubles in [0, 1) from stream `seed`."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) * _G + (np.arange(1, n + 1, dtype=np.uint64) * _G)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def field(seed, n):
    """n doubles in [-1, 1)."""
    return uniform(seed, n) * 2.0 - 1.0


def gauge(seed, V):
    """72*V doubles: per link a matrix with rows 0, 1 orthonormalised and
    row 2 = conj(row0 x row1), i.e. SU(3) up to rounding."""
    m = field(seed, 72 * V).reshape(V * 4, 3, 3, 2)
    u = m[..., 0] + 1j * m[..., 1]
    r0 = u[:, 0, :]
    r0 = r0 / np.sqrt(np.sum(np.abs(r0) ** 2, axis=1))[:, None]
    r1 = u[:, 1, :]
    r1 = r1 - np.sum(np.conj(r0) * r1, axis=1)[:, None] * r0
    r1 = r1 / np.sqrt(np.sum(np.abs(r1) ** 2, axis=1))[:, None]
    r2 = np.conj(np.cross(r0, r1))
    out = np.stack([r0, r1, r2], axis=1)
    return np.stack([out.real, out.imag], axis=-1).reshape(72 * V).copy()


def neighbours(dims, site):
    """The 8 nearest neighbours of a site (lexicographic)."""
    T, LX, LY, LZ = dims
    t, r = divmod(site, LX * LY * LZ)
    x, r = divmod(r, LY * LZ)
    y, z = divmod(r, LZ)
    c, L = [t, x, y, z], [T, LX, LY, LZ]
    out = []
    for m in range(4):
        for d in (1, -1):
            cc = list(c)
            cc[m] = (cc[m] + d) % L[m]
            out.append(((cc[0] * LX + cc[1]) * LY + cc[2]) * LZ + cc[3])
    return out


def sample_sites(dims, site, n, seed=2024):
    """The source, its 8 neighbours, then n distinct further sites (numpy
    PCG64 stream `seed`), sorted after the first 9."""
    V = int(np.prod(dims))
    head = [site] + neighbours(dims, site)
    rng = np.random.Generator(np.random.PCG64(seed))
    rest = rng.choice(V, size=n + 64, replace=False)
    rest = np.sort(np.array([s for s in rest if s not in head][:n]))
    return np.concatenate([np.array(head), rest]).astype(np.int64)
