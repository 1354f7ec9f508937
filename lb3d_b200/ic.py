"""Seeded synthetic initial states for the benchmark workloads.

The reference's random initial conditions use the compiler's intrinsic
random_number (code/lb3d_ic.F90:474-602), whose stream is specific to the
Fortran runtime, so every parity run instead starts from a checkpoint-style
state written by this generator (the init_cond = 7 path).  The generator is
counter based: SplitMix64 of (seed, stream, index), so any sub-lattice can
be regenerated independently and the state does not depend on thread or
launch order.

Populations follow the reference's uniform initial condition
n_{c,i} = rho_c * boltz_dist(0)_i (code/lb3d_ic.F90:474-522), i.e.
w_i = 1/36 on the 18 moving directions and 1/3 at rest, with
rho_c = base + uniform noise; surfactant dipoles are unit vectors uniform on
the sphere with da = db = d (code/lb3d_ic.F90:509-513).
"""
from __future__ import annotations

import numpy as np

W = np.array([1.0 / 36.0] * 18 + [1.0 / 3.0], dtype=np.float64)
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser (Steele, Lea, Flood 2014) on uint64 arrays."""
    with np.errstate(over="ignore"):
        z = x + _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, stream: int, count: int, offset: int = 0) -> np.ndarray:
    """count doubles in [0,1) from counter (seed, stream, offset + i)."""
    idx = np.arange(offset, offset + count, dtype=np.uint64)
    with np.errstate(over="ignore"):
        key = (idx + (np.uint64(stream) << np.uint64(40))) ^ (
            np.uint64(seed) * np.uint64(0xD1B54A32D192ED03))
    bits = splitmix64(key)
    return (bits >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def noise(seed: int, stream: int, shape, amp: float) -> np.ndarray:
    n = int(np.prod(shape))
    return (uniform01(seed, stream, n) * (2.0 * amp) - amp).reshape(shape)


def uniform_mixture(nx, ny, nz, ncomp, seed=1, rho=(0.7, 0.7, 0.7), amp=0.01):
    """Returns dict(n, db, rock, shear_sum): populations [ncomp][19][nz][ny][nx]
    with rho_c = rho[c] + U(-amp, amp) per site, and unit dipoles."""
    shape = (nz, ny, nx)
    n = np.empty((ncomp, 19) + shape, dtype=np.float64)
    for c in range(ncomp):
        r = rho[c] + noise(seed, 1 + c, shape, amp)
        n[c] = r[None] * W[:, None, None, None]
    db = None
    if ncomp == 3:
        db = unit_dipoles(seed, shape)
    return dict(n=n, db=db, rock=np.zeros(shape), shear_sum=0.0)


def unit_dipoles(seed, shape):
    u1 = uniform01(seed, 11, int(np.prod(shape))).reshape(shape)
    u2 = uniform01(seed, 12, int(np.prod(shape))).reshape(shape)
    z = 2.0 * u1 - 1.0
    phi = 2.0 * np.pi * u2
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    return np.stack([r * np.cos(phi), r * np.sin(phi), z])


def sphere_pack(nx, ny, nz, seed=1, porosity=0.4, rmin=6, rmax=12, overlap=False, max_tries=400000):
    """Rock mask [nz][ny][nx] (1 = rock) from seeded random spheres of radius
    rmin..rmax (periodic distances), added until the void fraction drops to
    `porosity` or `max_tries` candidates were drawn.  With overlap=False a
    candidate overlapping an earlier sphere is rejected (random sequential
    addition, which jams near a solid fraction of 0.38); overlap=True keeps
    every candidate, so any porosity is reachable."""
    rock = np.zeros((nz, ny, nx), dtype=np.uint8)
    target = (1.0 - porosity) * nx * ny * nz
    u = uniform01(seed, 21, 4 * max_tries).reshape(max_tries, 4)
    cen = np.zeros((0, 4))
    filled = 0
    dims = np.array([nx, ny, nz], dtype=np.float64)
    for t in range(max_tries):
        if filled >= target:
            break
        c = u[t, :3] * dims
        r = rmin + u[t, 3] * (rmax - rmin)
        if not overlap and len(cen):
            d = np.abs(cen[:, :3] - c)
            d = np.minimum(d, dims - d)
            if np.any((d * d).sum(1) < (cen[:, 3] + r) ** 2):
                continue
        cen = np.vstack([cen, [c[0], c[1], c[2], r]])
        x0, x1 = int(np.floor(c[0] - r)), int(np.ceil(c[0] + r)) + 1
        y0, y1 = int(np.floor(c[1] - r)), int(np.ceil(c[1] + r)) + 1
        z0, z1 = int(np.floor(c[2] - r)), int(np.ceil(c[2] + r)) + 1
        xs, ys, zs = np.arange(x0, x1) % nx, np.arange(y0, y1) % ny, np.arange(z0, z1) % nz
        dx = (np.arange(x0, x1) + 0.5 - c[0])[None, None, :]
        dy = (np.arange(y0, y1) + 0.5 - c[1])[None, :, None]
        dz = (np.arange(z0, z1) + 0.5 - c[2])[:, None, None]
        inside = (dx * dx + dy * dy + dz * dz) <= r * r
        sub = rock[np.ix_(zs, ys, xs)]
        filled += int(np.count_nonzero(inside & (sub == 0)))
        sub[inside] = 1
        rock[np.ix_(zs, ys, xs)] = sub
    return rock


def invasion_state(nx, ny, nz, rock, seed=1, slab=16, rho=0.7, amp=0.01):
    """Binary porous-invasion initial state: the first `slab` x-planes filled
    with red at rho, the rest with blue at rho (each + U(-amp, amp)), zero
    velocity, no populations at rock sites."""
    shape = (nz, ny, nx)
    n = np.zeros((2, 19) + shape)
    red = np.zeros(shape)
    red[:, :, :slab] = 1.0
    r_r = red * (rho + noise(seed, 1, shape, amp))
    r_b = (1.0 - red) * (rho + noise(seed, 2, shape, amp))
    n[0] = r_r[None] * W[:, None, None, None]
    n[1] = r_b[None] * W[:, None, None, None]
    n[:, :, rock != 0] = 0.0
    return dict(n=n, db=None, rock=rock.astype(np.float64), shear_sum=0.0)
