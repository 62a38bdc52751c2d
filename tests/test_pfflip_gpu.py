"""The reference's end-to-end property tests (tests/test_pfflip.py) run against
the drop-in Simulator on the GPU.

Same scenes, sizes, step counts, droplet settings and thresholds as the
reference file (line numbers in each docstring).
"""

import math

import numpy as np
import pytest

from pfflip import Config, Simulator, copy, scenes

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.fixture(scope="module")
def pool():
    cfg = Config(res=(32, 32, 32), dx=1.0 / 32, cfl=1.0, device=DEV, droplets=False)
    sim = Simulator(cfg)
    sim.set_particles(*scenes.still_pool(cfg, fill=0.5))
    return sim


def test_rho_tilde_0_matches_closed_form():
    """tests/test_pfflip.py:35-41"""
    cfg = Config(res=(8, 8, 8), dx=1.0 / 8, device=DEV, droplets=False)
    sim = Simulator(cfg)
    n_p = cfg.ppc / cfg.dx**3
    analytic = n_p * 64.0 * np.pi * cfg.r_p**3 / 315.0
    assert abs(sim.rho_tilde_0 - analytic) / analytic < 0.05


def test_phase_field_saturates(pool):
    """tests/test_pfflip.py:44-62"""
    pool.step()
    phi = pool.phi_cell.numpy()
    ny = phi.shape[1]
    air = phi[:, 3 * ny // 4:, :]
    liq = phi[:, : ny // 4, :]
    assert air.max() == 0.0, f"air phase is not clean: max phi = {air.max()}"
    assert liq.mean() > 0.95, f"liquid bulk not saturated on average: {liq.mean()}"
    assert liq.min() > 0.6, f"noise reaches the 0.5 tag threshold: min phi = {liq.min()}"


def test_interface_thickness_one_cell(pool):
    """tests/test_pfflip.py:65-74"""
    pool.step()
    phi = pool.phi_cell.numpy()
    col = phi[16, :, 16]
    inside = np.where(col > 0.95)[0]
    outside = np.where(col < 0.05)[0]
    gap = outside[outside > inside.max()].min() - inside.max()
    assert gap <= 3, f"interface spans {gap} cells; eps_phi should be ~1 cell"


def test_mass_conserved_exactly():
    """tests/test_pfflip.py:77-87"""
    cfg = Config(res=(24, 24, 24), dx=1.0 / 24, cfl=1.0, device=DEV, droplets=False)
    sim = Simulator(cfg)
    sim.set_particles(*scenes.dam_break(cfg))
    m0 = sim.pmass.numpy().sum()
    n0 = (sim.ptype.numpy() == 1).sum()
    for _ in range(10):
        sim.step()
    assert sim.pmass.numpy().sum() == m0
    assert (sim.ptype.numpy() == 1).sum() == n0


def test_hydrostatic_equilibrium_is_stable(pool):
    """tests/test_pfflip.py:90-103"""
    liq = pool.ptype.numpy() == 1
    y0 = pool.px.numpy()[liq, 1].mean()
    speeds = []
    for _ in range(30):
        pool.step()
        speeds.append(np.linalg.norm(pool.pv.numpy()[liq], axis=1).max())
    y1 = pool.px.numpy()[liq, 1].mean()
    g_dt = 9.81 * pool.stats[-1]["dt"]
    assert max(speeds) < 0.5 * g_dt, f"spurious liquid motion {max(speeds):.3f} vs g*dt {g_dt:.3f}"
    assert abs(y1 - y0) < 0.01 * pool.cfg.domain_size[1], "liquid centroid drifted"
    assert speeds[-1] <= speeds[0] * 1.5, "velocities are growing, not decaying"


@pytest.mark.parametrize("stencil", ["flux", "reference"])
def test_projection_reduces_divergence(stencil):
    """tests/test_pfflip.py:106-120"""
    cfg = Config(res=(32, 32, 32), dx=1.0 / 32, cfl=1.0, device=DEV, pcg_tol=1e-5, droplets=False,
                 stencil=stencil)
    sim = Simulator(cfg)
    sim.set_particles(*scenes.dam_break(cfg))
    sim._p2g()
    sim._phase_field_and_coefficients()
    for ax in range(3):
        copy(sim.vel_star[ax], sim.vel[ax])
    dt = 1e-3
    sim._add_forces(dt)
    div_before = sim._max_divergence()
    sim._pressure_solve(dt)
    sim._project(dt)
    div_after = sim._max_divergence()
    assert div_after < 0.05 * div_before, f"{div_before:.3e} -> {div_after:.3e}"


def test_bubbles_are_deleted_and_droplets_merge_back():
    """tests/test_pfflip.py:124-137: the escaped-particle transitions fire."""
    cfg = Config(res=(32,) * 3, dx=1 / 32, cfl=1.0, device=DEV, ppc=27, droplets=True, delta_phi=0.2)
    sim = Simulator(cfg)
    sim.set_particles(*scenes.asteroid_impact(cfg))
    for _ in range(25):
        sim.step()
    s = sim.droplet_stats
    assert s["bubbles"] > 0, "air particles trapped in liquid are never deleted"
    counts = sim.state_counts()
    assert counts["flip"] + counts["droplet"] + counts["dead"] == sim.n_particles
    assert counts["dead"] == s["bubbles"] or counts["dead"] >= s["bubbles"] - s["merged"]


def test_droplet_threshold_is_coupled_to_particle_count():
    """tests/test_pfflip.py:140-167"""
    for ppc in (8, 27):
        cfg = Config(res=(16,) * 3, dx=1 / 16, device=DEV, ppc=ppc)
        sim = Simulator(cfg)
        phi_single = 1.0 / math.sqrt(cfg.alpha_phi * sim.rho_tilde_0)
        predicted = 0.638 * ppc
        assert abs(sim.rho_tilde_0 - predicted) / predicted < 0.10
        assert (phi_single < 0.5 - cfg.delta_phi) == (ppc >= 18)


def test_droplets_do_not_contribute_to_the_grid():
    """tests/test_pfflip.py:170-189: particles with pstate != 0 do not splat."""
    cfg = Config(res=(16,) * 3, dx=1 / 16, cfl=1.0, device=DEV, ppc=8, droplets=True)
    sim = Simulator(cfg)
    sim.set_particles(*scenes.still_pool(cfg, fill=0.5))
    sim.step()
    m_all = sim.cell_mass.numpy().sum()
    st = sim.pstate.numpy()
    liq = np.flatnonzero(sim.ptype.numpy() == 1)
    st[liq[::10]] = 1
    sim.pstate.assign(st)
    sim._p2g()
    m_flip = sim.cell_mass.numpy().sum()
    assert m_flip < m_all
    removed = 1.0 - m_flip / m_all
    assert abs(removed - 0.10) < 0.02, f"expected ~10% of mass removed, got {100 * removed:.1f}%"


def test_obstacle_does_not_leak_gravity():
    """tests/test_pfflip.py:193-222"""
    cfg = Config(res=(32,) * 3, dx=1 / 32, cfl=1.0, device=DEV, ppc=8, droplets=False)
    sim = Simulator(cfg)
    pos, vel, pt, solid = scenes.wave_vs_tower(cfg)
    sim.set_particles(pos, vel, pt)
    sim.set_solids(solid)
    assert solid.sum() > 0
    for _ in range(5):
        sim.step()
    for ax in range(3):
        beta = sim.beta[ax].numpy()
        v = sim.vel[ax].numpy()
        blocked = beta == 0.0
        assert blocked.any()
        assert np.abs(v[blocked]).max() == 0.0


def test_obstacle_scene_stays_bounded():
    """tests/test_pfflip.py:225-242"""
    cfg = Config(res=(32,) * 3, dx=1 / 32, cfl=1.0, device=DEV, ppc=8, droplets=False)
    sim = Simulator(cfg)
    pos, vel, pt, solid = scenes.wave_vs_tower(cfg)
    sim.set_particles(pos, vel, pt)
    sim.set_solids(solid)
    v0 = float(np.abs(sim.pv.numpy()).max())
    speeds = []
    for _ in range(40):
        sim.step()
        st = sim.pstate.numpy()
        speeds.append(float(np.linalg.norm(sim.pv.numpy()[st == 0], axis=1).max()))
    assert max(speeds) < 12 * v0, f"|v| reached {max(speeds):.1f} from v0 = {v0:.2f}"
    assert np.isfinite(speeds).all()


def test_droplets_do_not_throttle_the_time_step():
    """tests/test_pfflip.py:245-268"""
    cfg = Config(res=(32,) * 3, dx=1 / 32, cfl=1.0, device=DEV, ppc=8, droplets=True)
    sim = Simulator(cfg)
    sim.set_particles(*scenes.asteroid_impact(cfg))
    sim.step()
    v = sim.pv.numpy()
    st = sim.pstate.numpy()
    v[0] = (500.0, 0.0, 0.0)
    st[0] = 1
    v[1] = (500.0, 0.0, 0.0)
    st[1] = 2
    sim.pv.assign(v)
    sim.pstate.assign(st)
    dt = sim.dt_from_cfl()
    assert dt > cfg.dx / 50.0, f"a single fast droplet collapsed dt to {dt:.2e}"


def test_particle_views_round_trip():
    """px/pv/ptype/pstate present the caller's original order across sorts."""
    cfg = Config(res=(16,) * 3, dx=1 / 16, ppc=8, droplets=False)
    sim = Simulator(cfg)
    pos, vel, pt = scenes.dam_break(cfg)
    rng = np.random.default_rng(0)
    vel = rng.standard_normal(pos.shape).astype(np.float32)
    sim.set_particles(pos, vel, pt)
    assert np.array_equal(sim.px.numpy(), pos) and np.array_equal(sim.pv.numpy(), vel)
    assert np.array_equal(sim.ptype.numpy(), pt)
    pos2 = pos[::-1].copy()
    sim.px.assign(pos2)
    sim._sort()
    assert np.array_equal(sim.px.numpy(), pos2) and np.array_equal(sim.pv.numpy(), vel)
    assert sim.pmass.numpy().dtype == np.float32
    assert sim.state_counts() == {"flip": len(pos), "droplet": 0, "dead": 0}


def test_save_frame_writes_the_reference_format(tmp_path):
    """pfflip/io.py:10-29: keys, dtypes, strided particles in the caller's order."""
    from pfflip import io

    cfg = Config(res=(16,) * 3, dx=1 / 16, device=DEV, ppc=8, droplets=False)
    sim = Simulator(cfg)
    pos, vel, pt = scenes.dam_break(cfg)
    sim.set_particles(pos, vel, pt)
    sim.step()
    path = str(tmp_path / "frames" / "frame_0001.npz")
    io.save_frame(sim, path, stride=3)
    f = io.load_frame(path)
    assert set(f) == {"t", "step", "dx", "phi", "px", "ptype"}
    assert f["t"].dtype == np.float32 and f["step"].dtype == np.int32 and f["dx"].dtype == np.float32
    assert f["phi"].dtype == np.float16 and f["px"].dtype == np.float16 and f["ptype"].dtype == np.int8
    assert int(f["step"]) == 1 and float(f["dx"]) == np.float32(cfg.dx)
    assert np.array_equal(f["phi"], sim.phi_cell.numpy().astype(np.float16))
    assert np.array_equal(f["px"], sim.px.numpy()[::3].astype(np.float16))
    assert np.array_equal(f["ptype"], pt[::3].astype(np.int8))
    io.save_frame(sim, str(tmp_path / "f2.npz"), particles=False)
    assert set(io.load_frame(str(tmp_path / "f2.npz"))) == {"t", "step", "dx", "phi"}


def test_host_round_trip_with_overlapped_copies_is_exact(monkeypatch):
    """set_particles from the very host buffers read_particles is still filling
    (chunked downloads; each upload chunk waits for the download of its host
    bytes) delivers every chunk's new contents.  Between upload and download a
    deterministic device update changes every value (the step itself sums with
    atomics, so it is not bitwise repeatable); an upload that raced its
    download would bring back stale values.  Small chunks, so that each array
    spans many of them."""
    import torch

    monkeypatch.setattr(Simulator, "_CHUNK", 1 << 16)
    cfg = Config(res=(32,) * 3, dx=1 / 32, ppc=8, droplets=False)
    pos, vel, pt = scenes.dam_break(cfg)
    exp_p, exp_v = pos.copy(), vel.copy()
    for _ in range(4):
        exp_p = exp_p + np.float32(1e-3)
        exp_v = exp_v * np.float32(1.5)
    for sync in (False, True):
        sim = Simulator(cfg)
        hp = torch.from_numpy(pos.copy()).pin_memory()
        hv = torch.from_numpy(vel.copy()).pin_memory()
        ht = torch.from_numpy(pt.astype(np.int32)).pin_memory()
        for _ in range(4):
            sim.set_particles(hp, hv, ht)
            sim._pos4[:, :3] += 1e-3
            sim._vel4[:, :3] *= 1.5
            if not sync:
                torch.cuda._sleep(20_000_000)  # ~10 ms: the next uploads are queued before these downloads run
            sim.read_particles(hp, hv, sync=sync)
        torch.cuda.synchronize()
        assert np.array_equal(hp.numpy(), exp_p), sync
        assert np.array_equal(hv.numpy(), exp_v), sync


def test_host_round_trip_steps_read_back_the_device_state():
    """Whole steps through pinned host buffers: after the last read the host
    arrays are exactly the simulator's particles in the caller's order."""
    import torch

    cfg = Config(res=(32,) * 3, dx=1 / 32, ppc=8, droplets=False)
    pos, vel, pt = scenes.dam_break(cfg)
    dt = 0.5 * cfg.dx / math.sqrt(2 * 9.81 * 0.6)
    sim = Simulator(cfg)
    hp = torch.from_numpy(pos.copy()).pin_memory()
    hv = torch.from_numpy(vel.copy()).pin_memory()
    ht = torch.from_numpy(pt.astype(np.int32)).pin_memory()
    for _ in range(3):
        sim.set_particles(hp, hv, ht)
        sim.step(dt)
        sim.read_particles(hp, hv, sync=False)
    torch.cuda.synchronize()
    assert np.array_equal(hp.numpy(), sim.px.numpy()) and np.array_equal(hv.numpy(), sim.pv.numpy())
    assert np.abs(hp.numpy() - pos).max() > 0


def _frame_loop(sim, frames, fps, save=None):
    """The frame loop of the reference's scripts/run.py:54-66: CFL sub-steps up
    to each frame time, the last one shortened to land on it, then a frame."""
    frame_dt = 1.0 / fps
    subs = []
    for frame in range(frames):
        target = (frame + 1) * frame_dt
        nsub = 0
        while sim.time < target - 1e-9:
            dt = min(sim.dt_from_cfl(), target - sim.time)
            sim.step(dt)
            nsub += 1
        subs.append(nsub)
        if save is not None:
            save(sim, frame)
    return subs


def test_frame_loop_matches_oracle(tmp_path):
    """Four frames at 24 fps of a 16^3 dam break through the run.py loop, the
    library against the oracle running the same loop: the same sub-step count
    per frame, every dt within 1e-4 relative (the CFL speed comes from the
    fused G2P reduction on the GPU, from a separate pass in the oracle), the
    frames landing on their times, phi within 1e-3 of its maximum after the
    free run, and the written frames in the reference's format."""
    import os

    from oracle import oracle as O
    from pfflip import io

    fps = 24.0
    cfg = Config(res=(16,) * 3, dx=1 / 16, ppc=8, seed=3, droplets=False, pcg_tol=1e-6, cfl=1.0, dt_max=1 / fps,
                 device=DEV)
    pos, vel, pt = scenes.dam_break(cfg)
    sim = Simulator(cfg)
    sim.set_particles(pos, vel, pt)
    o = O.OracleSim(cfg, nthreads=os.cpu_count() or 1, stencil=cfg.stencil)
    o.set_particles(pos, vel, pt)

    def save(s, f):
        io.save_frame(s, str(tmp_path / f"frame_{f:04d}.npz"), stride=4)

    subs_g = _frame_loop(sim, 4, fps, save)
    subs_o = _frame_loop(o, 4, fps)
    assert subs_g == subs_o and sum(subs_g) > 4, (subs_g, subs_o)
    dt_g = np.array([r["dt"] for r in sim.stats])
    dt_o = np.array([r["dt"] for r in o.stats])
    assert np.abs(dt_g - dt_o).max() <= 1e-4 * dt_o.max(), np.abs(dt_g / dt_o - 1).max()
    assert dt_g.min() < 1 / fps  # the CFL limit or a frame's last sub-step shortened the step
    assert abs(sim.time - 4 / fps) < 1e-9
    phi, phi_o = sim.phi_cell.numpy(), o.phi_cell
    assert np.abs(phi - phi_o).max() <= 1e-3 * np.abs(phi_o).max()
    for f in range(4):
        fr = io.load_frame(str(tmp_path / f"frame_{f:04d}.npz"))
        assert abs(float(fr["t"]) - (f + 1) / fps) < 1e-6
        assert fr["phi"].shape == cfg.res


def test_step_without_particles_matches_oracle():
    """An empty particle set, which the reference runs with its kernels
    launched over zero threads: the grid is all air (phi = 0), gravity is
    balanced against the walls by the pressure, and the library's steps match
    the oracle's (CG iterations within one, pressure within 1e-4 of its
    maximum after mean removal, the same CFL dt)."""
    import os

    from oracle import oracle as O

    cfg = Config(res=(8,) * 3, dx=1 / 8, ppc=8, pcg_tol=1e-6, device=DEV)  # droplets on, as by default
    e3, et = np.zeros((0, 3), np.float32), np.zeros(0, np.int32)
    sim = Simulator(cfg)
    sim.set_particles(e3, e3, et)
    o = O.OracleSim(cfg, nthreads=os.cpu_count() or 1, stencil=cfg.stencil)
    o.set_particles(e3, e3, et)
    dt = sim.dt_from_cfl()
    assert dt == pytest.approx(o.dt_from_cfl(), rel=1e-12)
    for _ in range(2):
        rg, ro = sim.step(dt), o.step(dt)
        assert abs(rg["pcg_iter"] - ro["pcg_iter"]) <= 1 and rg["pcg_res"] < 1e-6 and rg["droplets"] == 0
    assert np.abs(sim.phi_cell.numpy()).max() == 0.0
    p, po = sim.pressure.numpy(), o.pressure
    p, po = p - p.mean(), po - po.mean()
    assert np.abs(p - po).max() <= 1e-4 * np.abs(po).max()
    pos, vel = sim.read_particles()
    assert pos.shape == (0, 3) and vel.shape == (0, 3)
    assert sim.state_counts() == {"flip": 0, "droplet": 0, "dead": 0}
    sim.set_particles(*scenes.dam_break(cfg))  # and particles can arrive later
    assert sim.step(dt)["pcg_res"] < 1e-6
