"""Synthetic specimen generator (stands in for PDMaterialPoints.create,
which the reference loads as an external package).

Points sit at cell centres of a cubic lattice, x fastest, then y, then z
(the same 3xN column-major layout the reference passes around).  Jitter
comes from splitmix64 so that every consumer (GPU path, oracle, CPU
baseline) sees bit-identical inputs.
"""
import math

import numpy as np

_MASK = (1 << 64) - 1


def splitmix64(seed, n):
    """n uint64 values of the splitmix64 sequence starting from ``seed``."""
    out = np.empty(n, dtype=np.uint64)
    s = seed & _MASK
    # vectorised: state_k = seed + (k+1)*gamma
    gamma = np.uint64(0x9E3779B97F4A7C15)
    k = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(s) + k * gamma
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    out[:] = z
    return out


def uniform(seed, n, lo=0.0, hi=1.0):
    """n doubles uniform in [lo, hi) from splitmix64 (53-bit mantissas)."""
    u = (splitmix64(seed, n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return lo + (hi - lo) * u


def cuboid(nx, ny, nz, spacing, origin=(0.0, 0.0, 0.0), jitter=0.0, seed=1, centered=True):
    """(x 3xN, volume N) of an nx x ny x nz lattice.  ``centered`` puts
    points at cell centres (origin + (i + 1/2) * spacing), otherwise at
    origin + i * spacing.  ``jitter`` adds U(-jitter, jitter) per coordinate."""
    off = 0.5 if centered else 0.0
    i = np.arange(nx, dtype=np.float64)
    j = np.arange(ny, dtype=np.float64)
    k = np.arange(nz, dtype=np.float64)
    K, J, I = np.meshgrid(k, j, i, indexing="ij")
    x = np.empty((3, nx * ny * nz), order="F")
    x[0] = origin[0] + (I.reshape(-1) + off) * spacing
    x[1] = origin[1] + (J.reshape(-1) + off) * spacing
    x[2] = origin[2] + (K.reshape(-1) + off) * spacing
    if jitter:
        r = uniform(seed, 3 * x.shape[1], -jitter, jitter)
        x += r.reshape(3, -1, order="F")
    vol = np.full(x.shape[1], spacing ** 3)
    return x, vol


def disk(radius, thickness, spacing, center=(0.0, 0.0, 0.0)):
    """Disk in the x-y plane, axis along z, from a cell-centred lattice."""
    n = int(math.ceil(2 * radius / spacing))
    nz = max(1, int(round(thickness / spacing)))
    x, vol = cuboid(n, n, nz, spacing, origin=(center[0] - n * spacing / 2, center[1] - n * spacing / 2,
                                               center[2] - nz * spacing / 2))
    r2 = (x[0] - center[0]) ** 2 + (x[1] - center[1]) ** 2
    keep = r2 <= radius * radius
    return np.asfortranarray(x[:, keep]), vol[keep]


def sphere(radius, spacing, center=(0.0, 0.0, 0.0)):
    n = int(math.ceil(2 * radius / spacing))
    x, vol = cuboid(n, n, n, spacing, origin=tuple(c - n * spacing / 2 for c in center))
    r2 = ((x - np.asarray(center).reshape(3, 1)) ** 2).sum(axis=0)
    keep = r2 <= radius * radius
    return np.asfortranarray(x[:, keep]), vol[keep]


def gaussian_pulse(x, peak, sigma, axis=0, face="min"):
    """Velocity pulse along ``axis``: peak * exp(-d^2 / (2 sigma^2)), d the
    distance to the centre of the min (or max) face of the bounding box."""
    lo, hi = x.min(axis=1), x.max(axis=1)
    c = (lo + hi) / 2
    c[axis] = lo[axis] if face == "min" else hi[axis]
    d2 = ((x - c.reshape(3, 1)) ** 2).sum(axis=0)
    v = np.zeros_like(x, order="F")
    v[axis] = peak * np.exp(-d2 / (2 * sigma * sigma))
    return v
