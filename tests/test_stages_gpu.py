"""GPU parity of every particle/grid stage of the step against the CPU oracle.

Each test feeds the same inputs to libpfflip.so (through the C ABI or the
drop-in Simulator's stage methods) and to the oracle (oracle/pf_oracle.hpp,
the restatement of pfflip/kernels.py), then compares:

* sort keys, permutation and cell offsets: bit-exact (integer work);
* P2G accumulators: |gpu - oracle| <= 1e-5 * max|oracle| per array (summation
  order differs; the reference's own atomics are unordered too);
* phi, beta, is_liquid, extrapolated velocities: phi/beta within 1e-6
  relative, tags exact except where phi lies within 1e-5 of 0.5;
* projection, divergence, G2P/RK3: within 1e-5 relative (FMA contraction).
"""

import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle as O
from pfflip import Config, Simulator, scenes
from pfflip import _native as N

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def gpu_sort(pos, vel, res, dx):
    n = len(pos)
    g = N.grid(res, np.float32(dx))
    p4 = torch.zeros((max(n, 1), 4), dtype=torch.float32, device=DEV)
    v4 = torch.zeros((max(n, 1), 4), dtype=torch.float32, device=DEV)
    if n:
        p4[:n, :3] = torch.from_numpy(pos).to(DEV)
        v4[:n, :3] = torch.from_numpy(vel).to(DEV)
        v4.view(torch.int32)[:n, 3] = torch.arange(n, dtype=torch.int32, device=DEV)
    po, vo = torch.empty_like(p4), torch.empty_like(v4)
    keys = torch.empty(max(n, 1), dtype=torch.int32, device=DEV)
    perm = torch.empty(max(n, 1), dtype=torch.int32, device=DEV)
    start = torch.empty(int(np.prod(res)) + 1, dtype=torch.int32, device=DEV)
    ws = torch.empty(int(N.lib().pf_sort_workspace_bytes(C.byref(g), n)), dtype=torch.uint8, device=DEV)
    N.call("pf_sort_particles", C.byref(g), n, p4.data_ptr(), v4.data_ptr(), po.data_ptr(), vo.data_ptr(),
           keys.data_ptr(), perm.data_ptr(), start.data_ptr(), ws.data_ptr(), ws.numel(), N.stream())
    torch.cuda.synchronize()
    return keys[:n].cpu().numpy(), perm[:n].cpu().numpy(), start.cpu().numpy(), po[:n].cpu().numpy(), vo[:n].cpu().numpy()


def _near_faces(rng, res, dx, n):
    """Coordinates on and within 4 ulps of the cell faces k * dx (binary32),
    where x * (1/dx) and x / dx can round to different sides of an integer."""
    out = np.empty((n, 3), np.float32)
    for a in range(3):
        f = (rng.integers(0, res[a] + 1, n).astype(np.float32) * np.float32(dx)).astype(np.float32)
        steps = rng.integers(-4, 5, n)
        for s in range(-4, 5):
            m = steps == s
            v = f[m]
            for _ in range(abs(s)):
                v = np.nextafter(v, np.float32(np.inf if s > 0 else -np.inf)).astype(np.float32)
            f[m] = v
        out[:, a] = f
    return out


@pytest.mark.parametrize("case", ["random", "dam_break", "clustered", "walls", "empty", "one_cell", "faces",
                                  "faces_odd_dx", "one_cell_200k"])
def test_sort_bit_exact(case):
    rng = np.random.default_rng(11)
    res, dx = (24, 20, 36), np.float32(1 / 24)
    if case == "faces_odd_dx":
        dx = np.float32(0.0137)
    L = np.array(res, np.float64) * float(dx)
    if case.startswith("faces"):  # keys of coordinates at the cell faces follow the division
        pos = _near_faces(rng, res, dx, 120_000)
    elif case == "random":
        pos = (rng.random((200_003, 3)) * L).astype(np.float32)
    elif case == "dam_break":
        cfg = Config(res=(32,) * 3, dx=1 / 32, ppc=8)
        pos, _, _ = scenes.dam_break(cfg)
        res, dx = cfg.res, np.float32(cfg.dx)
        pos = pos[rng.permutation(len(pos))]
    elif case == "clustered":  # cells with > 32 particles hit the long-segment path
        base = (rng.random((300, 3)) * L).astype(np.float32)
        pos = np.repeat(base, 150, axis=0) + (rng.random((45000, 3)) * 1e-3 * float(dx)).astype(np.float32)
        pos = pos[rng.permutation(len(pos))]
    elif case == "walls":  # on/outside the walls: keys clamp
        pos = (rng.random((5000, 3)) * L).astype(np.float32)
        pos[:500] = 0.0
        pos[500:1000] = L.astype(np.float32)
        pos[1000:1500] = -0.5
        pos[1500:2000] = 7.0
    elif case == "empty":
        pos = np.zeros((0, 3), np.float32)
    elif case == "one_cell_200k":  # one cell holds 200,000 particles in random order, beside a sparse grid
        inner = (np.array([3, 4, 5]) + rng.random((200_000, 3))) * float(dx)
        pos = np.concatenate([inner, rng.random((5000, 3)) * L]).astype(np.float32)
        pos = pos[rng.permutation(len(pos))]
    else:
        pos = np.full((777, 3), 0.5 * float(dx), np.float32)
    vel = rng.standard_normal(pos.shape).astype(np.float32)
    import time

    t0 = time.perf_counter()
    keys, perm, start, po, vo = gpu_sort(pos, vel, res, dx)
    assert time.perf_counter() - t0 < 10.0  # the long segment's order fix is bounded work
    k_ref, p_ref, s_ref = O.sort_by_cell(pos, dx, res)
    assert np.array_equal(start, s_ref)
    assert np.array_equal(perm, p_ref)
    assert np.array_equal(keys, k_ref[p_ref])
    assert np.array_equal(po[:, :3], pos[p_ref]) and np.array_equal(vo[:, :3], vel[p_ref])
    assert np.array_equal(vo[:, 3].view(np.int32), p_ref)


def _oracle_from_sim(sim, cfg):
    o = O.OracleSim(cfg, stencil=cfg.stencil)
    o.set_particles(sim.px.numpy(), sim.pv.numpy(), sim.ptype.numpy(), sim.pstate.numpy())
    if sim.has_solids:
        o.set_solids(sim.solid.numpy())
    return o


def _grid_close(g, o, tol):
    for name in ("mass", "mom"):
        for ax in range(3):
            a, b = getattr(g, name)[ax].numpy(), getattr(o, name)[ax]
            assert rel(a, b) <= tol, (name, ax, rel(a, b))
    assert rel(g.cell_mass.numpy(), o.cell_mass) <= tol
    assert rel(g.cell_wsum.numpy(), o.cell_wsum) <= tol


@pytest.mark.parametrize("ppc", [8, 27])
def test_p2g_matches_oracle(ppc):
    cfg = Config(res=(32, 24, 40), dx=1 / 32, ppc=ppc, droplets=False)
    sim = Simulator(cfg)
    pos, vel, pt = scenes.dam_break(cfg)
    vel = np.random.default_rng(1).standard_normal(pos.shape).astype(np.float32)
    sim.set_particles(pos, vel, pt)
    st = np.zeros(len(pos), np.int32)
    st[::17] = 1  # droplets and dead particles must not splat
    st[5::29] = 2
    sim.pstate.assign(st)
    sim._p2g()
    o = _oracle_from_sim(sim, cfg)
    o._p2g()
    _grid_close(sim, o, 1e-5)


def test_phase_beta_forces_rhs_match_oracle():
    cfg = Config(res=(32, 32, 32), dx=1 / 32, ppc=8, droplets=False)
    sim = Simulator(cfg)
    pos, vel, pt, solid = scenes.wave_vs_tower(cfg)
    sim.set_particles(pos, vel, pt)
    sim.set_solids(solid)
    sim._p2g()
    sim._phase_field_and_coefficients()
    o = _oracle_from_sim(sim, cfg)
    for ax in range(3):  # same P2G input on both sides
        o.mass[ax][...] = sim.mass[ax].numpy()
        o.mom[ax][...] = sim.mom[ax].numpy()
    o.cell_mass[...] = sim.cell_mass.numpy()
    o.cell_wsum[...] = sim.cell_wsum.numpy()
    eps = np.float32(1e-12 * o.rho_0l)
    for ax in range(3):
        O._fn("face_velocity", np.float32)(o.mass[ax], o.mom[ax], o.vel[ax], o.valid[ax], o.mass[ax].size, eps)
    o._phase_field_and_coefficients()
    near = np.abs(o.phi_cell - 0.5) < 1e-5
    assert np.array_equal(sim.is_liquid.numpy()[~near], o.is_liquid[~near])
    assert rel(sim.phi_cell.numpy(), o.phi_cell) < 1e-6
    for ax in range(3):
        assert rel(sim.beta[ax].numpy(), o.beta[ax]) < 1e-6
        assert rel(sim.vel[ax].numpy(), o.vel[ax]) < 1e-6
        assert np.array_equal(sim.valid[ax].numpy(), o.valid[ax])
        assert rel(sim.phi_face[ax].numpy(), o.phi_face[ax]) < 1e-6
    dt = 2e-3
    sim._add_forces(dt, save_vel_star=True)
    o._save_vel_star()
    o._add_forces(dt)
    for ax in range(3):
        assert rel(sim.vel[ax].numpy(), o.vel[ax]) < 1e-6
        assert rel(sim.vel_star[ax].numpy(), o.vel_star[ax]) < 1e-6
    # right-hand side from identical velocities
    for ax in range(3):
        o.vel[ax][...] = sim.vel[ax].numpy()
    N.call("pf_build_rhs", C.byref(sim._g), *(N.ptr(a) for a in sim.vel), N.ptr(sim.cell_wsum), N.ptr(sim.rhs),
           float(dt), float(sim.rho_tilde_0), 0.0, N.stream())
    o._build_rhs(dt)
    assert rel(sim.rhs.numpy(), o.rhs) < 1e-5


@pytest.mark.parametrize("stencil", ["flux", "reference"])
def test_solve_project_divergence_match_oracle(stencil):
    cfg = Config(res=(32, 32, 32), dx=1 / 32, ppc=8, droplets=False, pcg_tol=1e-5, stencil=stencil)
    sim = Simulator(cfg)
    sim.set_particles(*scenes.dam_break(cfg))
    sim._p2g()
    sim._phase_field_and_coefficients()
    dt = 1e-3
    sim._add_forces(dt, save_vel_star=True)
    o = _oracle_from_sim(sim, cfg)
    for ax in range(3):
        o.vel[ax][...] = sim.vel[ax].numpy()
        o.beta[ax][...] = sim.beta[ax].numpy()
    o.cell_wsum[...] = sim.cell_wsum.numpy()
    div0 = sim._max_divergence()
    assert abs(div0 - o._max_divergence()) <= 1e-5 * div0
    it, r = sim._pressure_solve(dt)
    ito, ro = o._pressure_solve(dt)
    assert r < 1e-5 and ro < 1e-5 and abs(it - ito) <= 1
    p, po = sim.pressure.numpy(), o.pressure
    assert rel(p - p.mean(), po - po.mean()) < 1e-4
    # projection from the same pressure
    o.pressure[...] = p
    sim._project(dt)
    o._project(dt)
    for ax in range(3):
        assert rel(sim.vel[ax].numpy(), o.vel[ax]) < 1e-5
    div1 = sim._max_divergence()
    assert abs(div1 - o._max_divergence()) <= 1e-4 * div0
    assert div1 < 0.05 * div0


def test_extrapolation_matches_oracle_bitwise():
    cfg = Config(res=(36, 20, 44), dx=1 / 36, ppc=8, droplets=False)
    sim = Simulator(cfg)
    rng = np.random.default_rng(2)
    liq = (rng.random(cfg.res) < 0.15).astype(np.int32)
    sim.is_liquid.assign(liq)
    vel = [rng.standard_normal(s).astype(np.float32) for s in sim.face_shapes]
    for ax in range(3):
        sim.vel[ax].assign(vel[ax])
    o = O.OracleSim(cfg)
    o.is_liquid[...] = liq
    for ax in range(3):
        o.vel[ax][...] = vel[ax]
    for sweeps in (0, 1, 3, 4):
        sim.cfg.extrap_cells = sweeps
        o.cfg.extrap_cells = sweeps
        sim._extrapolate_liquid_velocity()
        o._extrapolate_liquid_velocity()
        for ax in range(3):
            assert np.array_equal(sim.vel_liq[ax].numpy(), o.vel_liq[ax]), (sweeps, ax)
            assert np.array_equal(sim._known[ax].numpy(), o._known[ax]), (sweeps, ax)


def test_g2p_advect_match_oracle():
    cfg = Config(res=(32, 32, 32), dx=1 / 32, ppc=8, droplets=False)
    sim = Simulator(cfg)
    pos, _, pt = scenes.dam_break(cfg)
    rng = np.random.default_rng(4)
    vel = rng.standard_normal(pos.shape).astype(np.float32)
    sim.set_particles(pos, vel, pt)
    st = np.zeros(len(pos), np.int32)
    st[::23] = 1
    st[7::31] = 2
    sim.pstate.assign(st)
    o = _oracle_from_sim(sim, cfg)
    for ax, s in enumerate(sim.face_shapes):
        u = rng.standard_normal(s).astype(np.float32)
        us = (u + 0.1 * rng.standard_normal(s)).astype(np.float32)
        ul = rng.standard_normal(s).astype(np.float32)
        sim.vel[ax].assign(u)
        sim.vel_star[ax].assign(us)
        sim.vel_liq[ax].assign(ul)
        o.vel[ax][...] = u
        o.vel_star[ax][...] = us
        o.vel_liq[ax][...] = ul
    dt = 0.5 / 32 / 3.0
    sim._g2p()
    o._g2p()
    assert rel(sim.pv.numpy(), o.pv) < 1e-5
    sim._advect(dt)
    o._advect(dt)
    assert np.abs(sim.px.numpy() - o.px).max() < 1e-5 * cfg.dx
    assert rel(sim.pv.numpy(), o.pv) < 1e-5


def test_step_matches_oracle_dam_break_32():
    """The 32^3 dam break with 8 ppc at a fixed dt, the reference's CPU-sized
    case: three full steps on the GPU and on the oracle from the same seeded
    particles."""
    cfg = Config(res=(32, 32, 32), dx=1 / 32, ppc=8, seed=42, droplets=False, pcg_tol=1e-6)
    dt = 0.5 * cfg.dx / np.sqrt(2 * 9.81 * 0.6)
    sim = Simulator(cfg)
    sim.set_particles(*scenes.dam_break(cfg))
    o = O.OracleSim(cfg, stencil=cfg.stencil)
    o.set_particles(*scenes.dam_break(cfg))
    for _ in range(3):
        rg = sim.step(dt)
        ro = o.step(dt)
        assert abs(rg["pcg_iter"] - ro["pcg_iter"]) <= 1
        assert rg["pcg_res"] < 1e-6 and ro["pcg_res"] < 1e-6
    assert np.abs(sim.px.numpy() - o.px).max() < 1e-4 * cfg.dx
    assert rel(sim.pv.numpy(), o.pv) < 1e-3
    assert rel(sim.phi_cell.numpy(), o.phi_cell) < 1e-4


@pytest.mark.parametrize("flags", [(1, 1), (1, 0), (0, 1)])
def test_g2p_packed_matches_unpaired(flags):
    """pf_g2p_advect_packed reads (j, k) quads of the fields and interpolates
    by lerp chains with the wall clamps folded into the weights; the unpaired
    kernel forms the reference's weighted sum of eight taps.  Same taps, so
    results agree to rounding: 2e-6 of the largest velocity, and positions to
    2e-6 of the largest coordinate."""
    do_g2p, do_adv = flags
    res = (24, 20, 36)
    dx = np.float32(1 / 24)
    g = N.grid(res, dx)
    rng = np.random.default_rng(21)
    n = 100_000
    L = np.array(res) * float(dx)
    pos = (rng.random((n, 3)) * L).astype(np.float32)
    pos[:2000] = (rng.random((2000, 3)) * 1e-3).astype(np.float32)  # at the low walls: clamped taps
    pos[2000:4000] = (L - rng.random((2000, 3)) * 1e-3).astype(np.float32)  # at the high walls
    fs = ((25, 20, 36), (24, 21, 36), (24, 20, 37))
    f = lambda: [torch.tensor(rng.standard_normal(s).astype(np.float32), device=DEV) for s in fs]  # noqa: E731
    u, us, ul = f(), f(), f()
    p4 = torch.zeros((n, 4), device=DEV)
    p4[:, :3] = torch.tensor(pos, device=DEV)
    p4.view(torch.int32)[:, 3] = torch.tensor((rng.random(n) < 0.5).astype(np.int32), device=DEV)
    v4 = torch.zeros((n, 4), device=DEV)
    v4[:, :3] = torch.tensor(rng.standard_normal((n, 3)).astype(np.float32), device=DEV)
    eps = 1e-4 * float(dx)
    lo = (C.c_float * 3)(eps, eps, eps)
    hi = (C.c_float * 3)(*[float(x) - eps for x in L])
    ws = torch.empty(int(N.lib().pf_g2p_workspace_bytes(C.byref(g))), dtype=torch.uint8, device=DEV)
    outs = []
    for packed in (False, True):
        p, v = p4.clone(), v4.clone()
        args = [C.byref(g), n, p.data_ptr(), v.data_ptr(), *(t.data_ptr() for t in u), *(t.data_ptr() for t in us),
                *(t.data_ptr() for t in ul), None, 0.985, 0.96, 0.01, lo, hi, do_g2p, do_adv]
        if packed:
            N.call("pf_g2p_advect_packed", *args, None, ws.data_ptr(), ws.numel(), N.stream())
        else:
            N.call("pf_g2p_advect", *args, N.stream())
        outs.append((p.cpu().numpy(), v.cpu().numpy()))
    (pa, va), (pb, vb) = outs
    assert np.array_equal(pa[:, 3].view(np.int32), pb[:, 3].view(np.int32))
    assert np.abs(pa[:, :3] - pb[:, :3]).max() <= 2e-6 * np.abs(pa[:, :3]).max()
    assert np.abs(va[:, :3] - vb[:, :3]).max() <= 2e-6 * np.abs(va[:, :3]).max()


@pytest.mark.parametrize("sweeps", [0, 2, 3, 4])
def test_extrapolation_level_passes_equal_tiled_sweeps(sweeps):
    """pf_extrapolate computes level by level in place when known arrays are
    given and with tiled shared-memory sweeps when they are NULL: bit-equal."""
    res = (30, 18, 40)
    g = N.grid(res, np.float32(1 / 30))
    rng = np.random.default_rng(13)
    fs = ((31, 18, 40), (30, 19, 40), (30, 18, 41))
    liq = torch.tensor((rng.random(res) < 0.1).astype(np.int32), device=DEV)
    u = [torch.tensor(rng.standard_normal(s).astype(np.float32), device=DEV) for s in fs]
    a = [torch.full(s, np.nan, device=DEV) for s in fs]
    b = [torch.full(s, np.nan, device=DEV) for s in fs]
    kn = [torch.full(s, -5, dtype=torch.int32, device=DEV) for s in fs]
    N.call("pf_extrapolate", C.byref(g), *(t.data_ptr() for t in u), liq.data_ptr(), sweeps,
           *(t.data_ptr() for t in a), None, None, None, N.stream())
    N.call("pf_extrapolate", C.byref(g), *(t.data_ptr() for t in u), liq.data_ptr(), sweeps,
           *(t.data_ptr() for t in b), *(t.data_ptr() for t in kn), N.stream())
    for x, y, k in zip(a, b, kn):
        assert torch.equal(x.view(torch.int32), y.view(torch.int32))
        assert set(torch.unique(k).tolist()) <= {0, 1}


def test_particle_max_speed_matches_oracle():
    """CFL speed (pfflip/kernels.py:552-564): max |v| over FLIP particles only;
    droplets and dead particles, given far larger speeds here, do not count."""
    cfg = Config(res=(24, 20, 36), dx=1 / 24, ppc=8, droplets=False)
    sim = Simulator(cfg)
    rng = np.random.default_rng(31)
    n = 150_001
    L = np.array(cfg.res) * cfg.dx
    pos = (rng.random((n, 3)) * L).astype(np.float32)
    vel = rng.standard_normal((n, 3)).astype(np.float32)
    st = np.zeros(n, np.int32)
    st[::97] = 1
    st[5::101] = 2
    vel[st != 0] *= 100.0
    sim.set_particles(pos, vel, (rng.random(n) < 0.5).astype(np.int32))
    sim.pstate.assign(st)
    N.call("pf_particle_max_speed", sim.n_particles, sim._pos4.data_ptr(), sim._vel4.data_ptr(),
           sim._scal.data_ptr(), N.stream())
    got = float(sim._scal[0].item())
    ref = float(O._fn("particle_max_speed", np.float32)(n, np.ascontiguousarray(vel), st))
    assert abs(got - ref) <= 1e-6 * ref
    assert got < 10.0  # the droplets' speeds (~100x) are excluded


def test_step_leaves_the_cfl_speed_on_the_device():
    """The step's last particle pass reduces the FLIP particles' max speed, so
    dt_from_cfl after a step reads it without a particle pass; it equals the
    separate reduction over the particles the step left and the oracle's."""
    cfg = Config(res=(32, 32, 32), dx=1 / 32, ppc=8, seed=42, droplets=False)
    sim = Simulator(cfg)
    sim.set_particles(*scenes.dam_break(cfg))
    assert not sim._vmax_valid
    for _ in range(3):
        sim.step(sim.dt_from_cfl())
    assert sim._vmax_valid
    launches = N.launch_count()
    fused = float(sim._scal[2].item())
    dt_fused = sim.dt_from_cfl()
    assert N.launch_count() == launches  # no particle pass
    sim._vmax_valid = False
    dt_sep = sim.dt_from_cfl()
    sep = float(sim._scal[0].item())
    assert abs(fused - sep) <= 1e-6 * sep and abs(dt_fused - dt_sep) <= 1e-6 * dt_sep
    ref = float(O._fn("particle_max_speed", np.float32)(sim.n_particles, np.ascontiguousarray(sim.pv.numpy()),
                                                        sim.pstate.numpy()))
    assert abs(fused - ref) <= 1e-6 * ref
    sim.pv.assign(sim.pv.numpy() * 2.0)  # any write outside the step invalidates it
    assert not sim._vmax_valid
