"""Particle seeding and the named scenes (host NumPy).

Seeding reproduces the reference's jittered lattice (``pfflip/scenes.py:17-45``)
bit for bit: lattice sites in ``meshgrid(..., indexing="ij")`` order, one
``default_rng(seed).random`` draw of shape (n, 3) in float64, the same
float64 expression ``(idx + 0.5)*step + (u - 0.5)*step*0.8``, then a cast to
float32.  The draw is consumed in row chunks, which yields the same stream as
one large call, so the 56.6M-particle 128^3 / 27 ppc lattice is built without
the reference's ~5 GB of float64 temporaries.

The scenes of the reference (``dam_break``, ``still_pool``, ``asteroid_impact``,
``rayleigh_taylor``, ``wave_vs_tower``) keep their signatures.  Added are the
asteroid-with-learnable-velocity and 16-mode Rayleigh-Taylor scenes and the
standalone 128^3 pressure-solve problem used by the benchmarks.
"""

from __future__ import annotations

import numpy as np

from .config import Config

AIR, LIQUID = 0, 1
_CHUNK = 1 << 21  # lattice sites per chunk


def _per_axis(ppc: int) -> int:
    pa = round(ppc ** (1.0 / 3.0))
    if pa**3 != ppc:
        raise ValueError("ppc must be a perfect cube (8, 27, ...)")
    return pa


def _lattice_chunks(res, dx, ppc, rng):
    """Yield (start, float64 positions) chunks of the jittered lattice."""
    pa = _per_axis(ppc)
    nx, ny, nz = (int(r) * pa for r in res)
    step = dx / pa
    n = nx * ny * nz
    for s in range(0, n, _CHUNK):
        e = min(n, s + _CHUNK)
        lin = np.arange(s, e, dtype=np.int64)
        idx = np.empty((e - s, 3), np.int64)
        idx[:, 0] = lin // (ny * nz)
        idx[:, 1] = (lin // nz) % ny
        idx[:, 2] = lin % nz
        pos = (idx + 0.5) * step
        pos += (rng.random(pos.shape) - 0.5) * step * 0.8
        yield s, pos


def _lattice(res, dx, ppc, rng):
    """Jittered ``ppc``-per-cell lattice over the whole domain (float64)."""
    pa = _per_axis(ppc)
    n = int(np.prod(res)) * pa**3
    out = np.empty((n, 3), np.float64)
    for s, pos in _lattice_chunks(res, dx, ppc, rng):
        out[s : s + len(pos)] = pos
    return out


def seed(cfg: Config, liquid_mask_fn, velocity_fn=None):
    """Particles from a predicate on world position.

    ``liquid_mask_fn(pos) -> bool array`` marks liquid; ``velocity_fn(pos, liq)``
    optionally returns (n, 3) initial velocities.  Returns float32 positions,
    float32 velocities and int32 types (0 air, 1 liquid).
    """
    rng = np.random.default_rng(cfg.seed)
    pa = _per_axis(cfg.ppc)
    n = int(np.prod(cfg.res)) * pa**3
    pos32 = np.empty((n, 3), np.float32)
    vel32 = np.zeros((n, 3), np.float32)
    ptype = np.empty(n, np.int32)
    for s, pos in _lattice_chunks(cfg.res, cfg.dx, cfg.ppc, rng):
        e = s + len(pos)
        liq = np.asarray(liquid_mask_fn(pos), dtype=bool)
        ptype[s:e] = np.where(liq, LIQUID, AIR)
        if velocity_fn is not None:
            vel32[s:e] = np.asarray(velocity_fn(pos, liq), float)
        pos32[s:e] = pos
    return pos32, vel32, ptype


# ---------------------------------------------------------------------------
def dam_break(cfg: Config, frac=(0.4, 0.6, 1.0)):
    """Liquid column ``x < frac0*Lx, y < frac1*Ly, z < frac2*Lz`` in a closed box."""
    sx, sy, sz = cfg.domain_size

    def mask(p):
        return (p[:, 0] < frac[0] * sx) & (p[:, 1] < frac[1] * sy) & (p[:, 2] < frac[2] * sz)

    return seed(cfg, mask)


def still_pool(cfg: Config, fill=0.5):
    """Hydrostatic pool ``y < fill*Ly``."""
    sy = cfg.domain_size[1]
    return seed(cfg, lambda p: p[:, 1] < fill * sy)


def asteroid_impact(cfg: Config, *, water_level=0.45, radius_frac=0.08, speed=None):
    """A liquid ball fired down into a deep pool."""
    sx, sy, sz = cfg.domain_size
    r = radius_frac * sx
    centre = np.array([0.5 * sx, water_level * sy + 0.35 * sy, 0.5 * sz])
    v_impact = speed if speed is not None else -0.9 * np.sqrt(2 * 9.81 * 0.35 * sy)

    def ball(p):
        return np.linalg.norm(p - centre, axis=1) < r

    def mask(p):
        return (p[:, 1] < water_level * sy) | ball(p)

    def vel(p, liq):
        v = np.zeros_like(p)
        v[ball(p), 1] = v_impact
        return v

    return seed(cfg, mask, vel)


def rayleigh_taylor(cfg: Config, *, ratio=None):
    """Heavy phase above ``y = Ly/2 + 0.02 Ly (cos 2πx/Lx + cos 2πz/Lz)``."""
    sx, sy, sz = cfg.domain_size

    def mask(p):
        h = 0.5 * sy + 0.02 * sy * (np.cos(2 * np.pi * p[:, 0] / sx) + np.cos(2 * np.pi * p[:, 2] / sz))
        return p[:, 1] > h

    return seed(cfg, mask)


def wave_vs_tower(cfg: Config, *, sea_level=0.22, column=0.26, tower_r=0.075, tower_at=(0.62, 0.5), surge=None):
    """Surge released onto a cylindrical tower.  Returns (pos, vel, ptype, solid)."""
    sx, sy, sz = cfg.domain_size
    nx, ny, nz = cfg.res
    v0 = surge if surge is not None else 0.55 * np.sqrt(9.81 * sy)

    def block(p):
        return (p[:, 0] < column * sx) & (p[:, 1] < 0.72 * sy)

    def mask(p):
        return (p[:, 1] < sea_level * sy) | block(p)

    def vel(p, liq):
        v = np.zeros_like(p)
        v[block(p) & liq, 0] = v0
        return v

    pos, pvel, ptype = seed(cfg, mask, vel)
    ci = (np.arange(nx) + 0.5) / nx
    ck = (np.arange(nz) + 0.5) / nz
    I, K = np.meshgrid(ci, ck, indexing="ij")
    disc = (I - tower_at[0]) ** 2 + (K - tower_at[1]) ** 2 < tower_r**2
    solid = np.broadcast_to(disc[:, None, :], (nx, ny, nz)).copy()
    solid[:, -2:, :] = False
    keep = ~(((pos[:, 0] / sx - tower_at[0]) ** 2 + (pos[:, 2] / sz - tower_at[1]) ** 2) < tower_r**2)
    return pos[keep], pvel[keep], ptype[keep], solid


SCENES = {
    "dam_break": dam_break,
    "still_pool": still_pool,
    "asteroid": asteroid_impact,
    "rayleigh_taylor": rayleigh_taylor,
}
SCENES["wave_vs_tower"] = wave_vs_tower


# ---------------------------------------------------------------------------
# scenes of the benchmark workloads
# ---------------------------------------------------------------------------
def asteroid_pool(cfg: Config, *, v0=(0.0, -2.0, 0.0), pool=0.3, centre=(0.5, 0.7, 0.5), radius=0.1,
                  sigma=0.01, seed_offset=1):
    """Liquid pool ``y < pool*Ly`` plus a liquid sphere (fractions of the domain),
    the sphere moving with ``v0`` plus i.i.d. N(0, sigma^2) per-particle
    perturbations drawn from ``default_rng(cfg.seed + seed_offset)``.

    Returns (pos, vel, ptype, sphere_mask, perturbation)."""
    sx, sy, sz = cfg.domain_size
    c = np.array([centre[0] * sx, centre[1] * sy, centre[2] * sz])
    r = radius * sx

    def ball(p):
        return np.linalg.norm(p - c, axis=1) < r

    pos, vel, ptype = seed(cfg, lambda p: (p[:, 1] < pool * sy) | ball(p))
    sphere = ball(pos.astype(np.float64))
    rng = np.random.default_rng(cfg.seed + seed_offset)
    pert = (rng.standard_normal((len(pos), 3)) * sigma).astype(np.float32)
    pert[~sphere] = 0.0
    vel = np.zeros_like(pos)
    vel[sphere] = np.asarray(v0, np.float32)[None, :] + pert[sphere]
    return pos, vel.astype(np.float32), ptype, sphere, pert


def rt_modes(seed: int, n_modes: int = 16, amp_max: float = 0.01):
    """Amplitudes a_k ~ U(0, amp_max) and integer wave numbers (m_k, n_k) in 1..4."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.0, amp_max, n_modes)
    mn = rng.integers(1, 5, size=(n_modes, 2))
    return a, mn


def rayleigh_taylor_modes(cfg: Config, amps=None, waves=None, n_modes: int = 16):
    """Heavy phase above ``y = 0.5 + Σ a_k cos(2π(m_k x + n_k z))`` (unit-box
    coordinates).  Returns (pos, vel, ptype, amps, waves)."""
    a_def, mn_def = rt_modes(cfg.seed, n_modes)
    amps = a_def if amps is None else np.asarray(amps, np.float64)
    waves = mn_def if waves is None else np.asarray(waves)
    sx, sy, sz = cfg.domain_size

    def mask(p):
        xu, zu = p[:, 0] / sx, p[:, 2] / sz
        h = 0.5 + np.cos(2 * np.pi * (np.outer(xu, waves[:, 0]) + np.outer(zu, waves[:, 1]))) @ amps
        return p[:, 1] / sy > h

    pos, vel, ptype = seed(cfg, mask)
    return pos, vel, ptype, amps, waves


def solve_problem(res=(128, 128, 128), seed: int = 42, rho_l=1000.0, density_ratio=1000.0):
    """The standalone pressure-solve workload: φ = max(slab y<0.5, sphere r=0.15 at
    (0.5,0.75,0.5)), each a tanh profile 2 cells wide; face φ is the mean of the
    two adjacent cells; β = 1/((1-φ)ρ_g + φρ_l) with zero boundary faces; a zero-mean
    N(0,1) right-hand side from ``default_rng(seed)``.  Returns float32
    (bx, by, bz, b, phi_cell)."""
    nx, ny, nz = res
    dx = 1.0 / nx
    rho_g = rho_l / density_ratio
    c = (np.arange(nx) + 0.5) * dx, (np.arange(ny) + 0.5) * dx, (np.arange(nz) + 0.5) * dx
    X, Y, Z = np.meshgrid(*c, indexing="ij")
    slab = 0.5 * (1.0 - np.tanh((Y - 0.5) / (2 * dx)))
    dist = np.sqrt((X - 0.5) ** 2 + (Y - 0.75) ** 2 + (Z - 0.5) ** 2)
    sphere = 0.5 * (1.0 - np.tanh((dist - 0.15) / (2 * dx)))
    phi = np.maximum(slab, sphere)
    out = []
    for ax in range(3):
        pad = [(0, 0)] * 3
        pad[ax] = (1, 1)
        pp = np.pad(phi, pad, mode="edge")
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax] = slice(0, -1)
        hi[ax] = slice(1, None)
        pf = 0.5 * (pp[tuple(lo)] + pp[tuple(hi)])
        beta = 1.0 / ((1.0 - pf) * rho_g + pf * rho_l)
        sl = [slice(None)] * 3
        sl[ax] = 0
        beta[tuple(sl)] = 0.0
        sl[ax] = -1
        beta[tuple(sl)] = 0.0
        out.append(beta.astype(np.float32))
    rng = np.random.default_rng(seed)
    b = rng.standard_normal(res)
    b -= b.mean()
    return out[0], out[1], out[2], b.astype(np.float32), phi.astype(np.float32)


def rayleigh_taylor_lattice(cfg: Config, n_modes: int = 16):
    """The Rayleigh-Taylor scene in a form that is differentiable in the mode
    amplitudes: the jittered lattice of ``seed`` with the heavy phase (liquid
    tag) where the *reference* height y_ref > 0.5 Ly, to be displaced by
    ``rt_displace``.  The tags do not depend on a_k; the positions do,
    smoothly.  Returns (pos_ref, ptype, amps, waves)."""
    amps, waves = rt_modes(cfg.seed, n_modes)
    sy = cfg.domain_size[1]
    pos, _, ptype = seed(cfg, lambda p: p[:, 1] > 0.5 * sy)
    return pos, ptype, amps, waves


def rt_profile(pos, waves, domain, xp=np):
    """Per particle and mode: the vertical displacement a unit amplitude of
    mode k gives the particle at reference position pos,
        D[p, k] = Ly sin^2(pi y/Ly) cos(2 pi (m_k x/Lx + n_k z/Lz)).
    sin^2 is 1 at y = Ly/2 and 0 at the floor and the lid, so
    y -> y + D a maps the plane y_ref = Ly/2 onto 0.5 + sum_k a_k cos(...) (in
    unit-box coordinates), keeps particles inside the box, and is monotone in y
    while pi |sum_k a_k cos(...)| < 1 (always for a_k <= 0.01 and 16 modes).
    ``xp`` is numpy (float64 host) or torch (device tensors)."""
    sx, sy, sz = domain
    x, y, z = pos[:, 0:1], pos[:, 1:2], pos[:, 2:3]
    if xp is np:
        w = np.asarray(waves, np.float64)
        m, n = w[None, :, 0], w[None, :, 1]
    else:
        w = xp.as_tensor(np.asarray(waves), dtype=pos.dtype, device=pos.device)
        m, n = w[None, :, 0], w[None, :, 1]
    return sy * xp.sin(np.pi * y / sy) ** 2 * xp.cos(2 * np.pi * (m * x / sx + n * z / sz))


def rt_displace(pos_ref, amps, waves, domain):
    """Positions of the Rayleigh-Taylor lattice for amplitudes ``amps`` (host,
    float64 arithmetic; float32 result)."""
    p = np.asarray(pos_ref, np.float64)
    out = p.copy()
    out[:, 1] += rt_profile(p, waves, domain) @ np.asarray(amps, np.float64)
    return out
