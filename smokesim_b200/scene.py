"""Seeded synthetic scenes of the benchmark workloads.

No public dataset or benchmark suite is involved: every workload is a seeded
scene (emitters, obstacles, boxes) plus, where asked for, a seeded Gaussian
random velocity field.  Randomness comes from splitmix64 (vectorised in numpy)
turned into uniforms and Box-Muller normals in FP64 on the host, so every
consumer of a scene sees identical bits.

Workloads (cell size 1, ambient temperature 0, solid walls, dt = 0.1,
alpha = 0.05, beta = 0.3, epsilon = 0.2; schedule 2+2 red-black sweeps, 80 on
the coarsest level, 4 V-cycles, coarsest level 8):
  plume2d  - 256^2, one r=12 disc emitter at y=16, x ~ U[64,192], one 40x20 box
             in the middle third.
  plume3d  - 128^3, two r=8 emitters at y=8, (x,z) ~ U[32,96]^2, an r=16 sphere
             at the centre and three cubes of side ~ U[8,24].
  grf256   - plume3d scaled x2 at 256^3 (emitter r=16, sphere r=32, cubes 16-48)
             with a unit-variance Gaussian random initial velocity (sigma 8 cells).
  rollout64 - 64^3, one r=6 emitter at (32,6,32), an r=8 sphere at the centre,
             divergence-free random initial velocity of amplitude 0.5.
"""
from __future__ import annotations

import numpy as np

from . import abi

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """n consecutive splitmix64 outputs of the stream `seed` starting at `offset`."""
    with np.errstate(over="ignore"):
        i = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * GOLDEN
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        z = z ^ (z >> np.uint64(31))
    return z


class Rng:
    """Sequential splitmix64 stream with FP64 uniforms and Box-Muller normals."""

    def __init__(self, seed: int):
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self.pos = 0

    def u64(self, n):
        z = splitmix64(self.seed, n, self.pos)
        self.pos += n
        return z

    def uniform(self, n=None, lo=0.0, hi=1.0):
        k = 1 if n is None else n
        u = (self.u64(k) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
        u = lo + (hi - lo) * u
        return float(u[0]) if n is None else u

    def integer(self, lo, hi):
        """uniform integer in [lo, hi]"""
        return int(np.floor(self.uniform(None, lo, hi + 1 - 1e-9)))

    def normal(self, n):
        m = (n + 1) // 2
        u1 = self.uniform(m)
        u2 = self.uniform(m)
        r = np.sqrt(-2.0 * np.log1p(-u1))
        t = 2.0 * np.pi * u2
        return np.concatenate([r * np.cos(t), r * np.sin(t)])[:n]


def emitter(pos, radius, density=1.0, temperature=1.0, velocity=(0.0, 2.0, 0.0), falloff=0):
    e = abi.Emitter()
    e.pos[0], e.pos[1], e.pos[2] = pos
    e.radius = radius
    e.density[0] = density
    e.temperature = temperature
    e.delay = 0
    e.last_emit = 0
    e.emit = 0
    e.falloff = falloff
    e.set_velocity = 1
    e.velocity[0], e.velocity[1], e.velocity[2] = velocity
    return e


def obstacle(pos, radius, velocity=(0.0, 0.0, 0.0), anchored=1.0):
    o = abi.Obstacle()
    o.pos[0], o.pos[1], o.pos[2] = pos
    o.radius = radius
    o.velocity[0], o.velocity[1], o.velocity[2] = velocity
    o.anchored = anchored
    return o


def box(lo, hi, velocity=(0.0, 0.0, 0.0), anchored=1.0):
    b = abi.Box()
    b.lo[0], b.lo[1], b.lo[2] = lo
    b.hi[0], b.hi[1], b.hi[2] = hi
    b.velocity[0], b.velocity[1], b.velocity[2] = velocity
    b.anchored = anchored
    return b


def workload_params(**kw):
    base = dict(dt=0.1, rho=1.0, t_ambient=0.0, alpha=0.05, beta=0.3, eps=0.2, n_pre=2, n_post=2, n_coarse=80,
                n_vcycles=4, tol=0.0, ref_quirks=1)
    base.update(kw)
    return abi.make_params(**base)


def gaussian_filter_axis(a, sigma, axis, radius):
    """Separable Gaussian filter along one axis with zero padding (FP64)."""
    x = np.arange(-radius, radius + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    a = np.moveaxis(a, axis, -1)
    n = a.shape[-1]
    pad = np.zeros(a.shape[:-1] + (n + 2 * radius,), np.float64)
    pad[..., radius:radius + n] = a
    out = np.zeros_like(a, dtype=np.float64)
    for j, w in enumerate(k):
        out += w * pad[..., j:j + n]
    return np.moveaxis(out, -1, axis)


def grf(rng: Rng, shape, sigma=8.0, radius=None):
    """Unit-variance Gaussian random field: white N(0,1) smoothed by a separable
    Gaussian of standard deviation sigma cells (truncated at 3 sigma, zero
    padding), then renormalised."""
    radius = int(3 * sigma) if radius is None else radius
    w = rng.normal(int(np.prod(shape))).reshape(shape)
    try:
        from scipy.ndimage import gaussian_filter1d
        for ax in range(len(shape)):
            if shape[ax] > 1:
                w = gaussian_filter1d(w, sigma, axis=ax, mode="constant", truncate=radius / sigma)
    except ImportError:
        for ax in range(len(shape)):
            if shape[ax] > 1:
                w = gaussian_filter_axis(w, sigma, ax, radius)
    w -= w.mean()
    sd = w.std()
    return (w / sd) if sd > 0 else w


def divergence_free_velocity(rng: Rng, n, amplitude=0.5, sigma=4.0):
    """Discrete curl of a random vector potential on cell corners: exactly
    divergence-free MAC velocities (3D), scaled to the given RMS amplitude."""
    nx, ny, nz = n
    A = [grf(rng, (nz + 1, ny + 1, nx + 1), sigma) for _ in range(3)]
    Ax, Ay, Az = A
    u = (Az[:-1, 1:, :] - Az[:-1, :-1, :]) - (Ay[1:, :-1, :] - Ay[:-1, :-1, :])
    v = (Ax[1:, :, :-1] - Ax[:-1, :, :-1]) - (Az[:-1, :, 1:] - Az[:-1, :, :-1])
    w = (Ay[:, :-1, 1:] - Ay[:, :-1, :-1]) - (Ax[:, 1:, :-1] - Ax[:, :-1, :-1])
    rms = np.sqrt((np.mean(u ** 2) + np.mean(v ** 2) + np.mean(w ** 2)) / 3.0)
    s = amplitude / rms if rms > 0 else 1.0
    return (u * s).astype(np.float32), (v * s).astype(np.float32), (w * s).astype(np.float32)


def _cube(rng, n, side_lo, side_hi):
    side = rng.integer(side_lo, side_hi)
    lo = [rng.integer(2, max(2, n[d] - 2 - side)) for d in range(3)]
    return box(tuple(float(v) for v in lo), tuple(float(v + side) for v in lo))


def plume2d(seed=0, n=256):
    rng = Rng(seed)
    ex = float(rng.integer(n // 4, 3 * n // 4))
    em = [emitter((ex, 16.0 * n / 256, 0.0), 12.0 * n / 256, velocity=(0.0, 2.0, 0.0))]
    third = n // 3
    bw, bh = 40 * n // 256, 20 * n // 256
    bxl = float(rng.integer(third, 2 * third - bw))
    byl = float(rng.integer(third, 2 * third - bh))
    bxs = [box((bxl, byl, 0.0), (bxl + bw, byl + bh, 1.0))]
    desc = abi.make_desc(2, (n, n), cell_size=1.0, density_channels=1, enclosed=1, min_coarse=8)
    return dict(desc=desc, params=workload_params(), emitters=em, obstacles=[], boxes=bxs, fields={}, steps=200)


def plume3d(seed=0, n=128, steps=500):
    """Two emitters, a centre sphere and three cubes; all sizes scale with n/128."""
    rng = Rng(seed)
    f = n / 128.0
    em = []
    for _ in range(2):
        x = float(rng.integer(int(32 * f), int(96 * f)))
        z = float(rng.integer(int(32 * f), int(96 * f)))
        em.append(emitter((x, 8.0 * f, z), 8.0 * f, velocity=(0.0, 2.0, 0.0)))
    ob = [obstacle((n / 2.0, n / 2.0, n / 2.0), 16.0 * f)]
    bxs = [_cube(rng, (n, n, n), max(2, int(8 * f)), max(3, int(24 * f))) for _ in range(3)]
    desc = abi.make_desc(3, (n, n, n), cell_size=1.0, density_channels=1, enclosed=1, min_coarse=8)
    return dict(desc=desc, params=workload_params(), emitters=em, obstacles=ob, boxes=bxs, fields={}, steps=steps,
                rng=rng)


def grf256(seed=0, n=256, with_grf=True, steps=100):
    sc = plume3d(seed, n=n, steps=steps)
    rng = sc.pop("rng")
    if with_grf:
        sc["fields"] = {
            abi.FIELD_VX: grf(rng, (n, n, n + 1)).astype(np.float32),
            abi.FIELD_VY: grf(rng, (n, n + 1, n)).astype(np.float32),
            abi.FIELD_VZ: grf(rng, (n + 1, n, n)).astype(np.float32),
        }
    return sc


def rollout64(seed=0, n=64, steps=64):
    rng = Rng(seed)
    em = [emitter((n / 2.0, 6.0 * n / 64, n / 2.0), 6.0 * n / 64, velocity=(0.0, 2.0, 0.0))]
    ob = [obstacle((n / 2.0, n / 2.0, n / 2.0), 8.0 * n / 64)]
    u, v, w = divergence_free_velocity(rng, (n, n, n), amplitude=0.5)
    desc = abi.make_desc(3, (n, n, n), cell_size=1.0, density_channels=1, enclosed=1, min_coarse=8)
    return dict(desc=desc, params=workload_params(), emitters=em, obstacles=ob, boxes=[],
                fields={abi.FIELD_VX: u, abi.FIELD_VY: v, abi.FIELD_VZ: w}, steps=steps)


def random_state(rng: Rng, dim, n, nch=1, vel_scale=1.0, t_scale=1.0):
    """Random fields for parity tests (velocities, density, temperature, pressure)."""
    nx, ny = n[0], n[1]
    nz = 1 if dim == 2 else n[2]
    f = {
        abi.FIELD_VX: (rng.normal((nx + 1) * ny * nz) * vel_scale).astype(np.float32),
        abi.FIELD_VY: (rng.normal(nx * (ny + 1) * nz) * vel_scale).astype(np.float32),
        abi.FIELD_DENSITY: np.abs(rng.normal(nx * ny * nz * nch)).astype(np.float32),
        abi.FIELD_TEMPERATURE: (rng.normal(nx * ny * nz) * t_scale).astype(np.float32),
        abi.FIELD_PRESSURE: rng.normal(nx * ny * nz).astype(np.float32),
    }
    if dim == 3:
        f[abi.FIELD_VZ] = (rng.normal(nx * ny * (nz + 1)) * vel_scale).astype(np.float32)
    return f


def apply(sim, sc):
    """Load a scene dict into a Sim (or an oracle sim with the same methods)."""
    sim.set_scene(sc["emitters"], sc["obstacles"], sc["boxes"])
    for f, a in sc.get("fields", {}).items():
        sim.set_field(f, a)
