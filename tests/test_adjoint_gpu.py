"""Adjoint of the PF-FLIP step (pfflip.adjoint, the pf_adj_* kernels) against
FP64 central finite differences of the CPU oracle.

The gradients come from the FP32 GPU step.  The finite differences run the
oracle in binary64 with the solve converged to 1e-12.  The perturbation is
small (1e-6), so no wall clamp, liquid tag, extrapolation mask or
interpolation cell boundary is crossed in practice, and the difference
quotient measures the derivative away from the kinks.  Tolerance: 1e-3
relative, which leaves room for the FP32 forward's rounding and its 1e-6
solver tolerance.

The linear stages are also checked on their own with the transpose identity
<A u, w> = <u, A^T w>, evaluated on the GPU in FP32 (1e-5 relative).
"""

import ctypes as C
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from pfflip import Config, scenes
from pfflip import _native as N
from pfflip.adjoint import DiffSim

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
NTHR = max(1, min(os.cpu_count() or 1, 32))


def small_cfg(res=16, ppc=8, seed=3):
    return Config(res=(res,) * 3, dx=1.0 / res, ppc=ppc, seed=seed, droplets=False, pcg_tol=1e-6,
                  pcg_max_iter=400, device=DEV)


def step_dt(cfg, speed=2.5, cfl=0.25):
    return cfl * cfg.dx / speed


def oracle_run(cfg, pos, vel, ptype, dt, steps):
    sim = O.OracleSim(_with(cfg, pcg_tol=1e-12, pcg_max_iter=1000), dtype=np.float64, nthreads=NTHR, stencil="flux")
    sim.set_particles(pos, vel, ptype)
    for _ in range(steps):
        sim.step(dt)
    return sim


def _with(cfg, **kw):
    import dataclasses

    return dataclasses.replace(cfg, **kw)


def oracle_phi(sim):
    sim._p2g()
    sim._phase_field_and_coefficients()
    return sim.phi_cell.copy()


# ---------------------------------------------------------------- full steps
@pytest.mark.parametrize("steps,every", [(1, 1), (3, 2)])
def test_step_adjoint_matches_fp64_finite_differences(steps, every):
    """L = <a, x_T> + <b, v_T> after `steps` steps; directional derivative
    along a random (dx0, dv0) from the adjoint vs the FP64 central difference."""
    cfg = small_cfg()
    dt = step_dt(cfg)
    pos, vel, ptype, _, _ = scenes.asteroid_pool(cfg)
    n = len(pos)
    rng = np.random.default_rng(7)
    a = rng.standard_normal((n, 3))
    b = rng.standard_normal((n, 3))
    dxd = rng.standard_normal((n, 3)) * cfg.dx
    dvd = rng.standard_normal((n, 3))

    ds = DiffSim(cfg, ptype, dt, checkpoint_every=every, adjoint_tol=1e-6)
    x0 = torch.tensor(pos, device=DEV, requires_grad=True)
    v0 = torch.tensor(vel, device=DEV, requires_grad=True)
    xT, vT = ds.rollout(x0, v0, steps)
    L = (torch.tensor(a, device=DEV) * xT.double()).sum() + (torch.tensor(b, device=DEV) * vT.double()).sum()
    L.backward()
    d_adj = float((x0.grad.double().cpu().numpy() * dxd).sum() + (v0.grad.double().cpu().numpy() * dvd).sum())

    def loss(eps):
        s = oracle_run(cfg, pos.astype(np.float64) + eps * dxd, vel.astype(np.float64) + eps * dvd, ptype, dt, steps)
        return float((a * s.px).sum() + (b * s.pv).sum())

    eps = 1e-6
    d_fd = (loss(eps) - loss(-eps)) / (2 * eps)
    assert abs(d_adj - d_fd) <= 1e-3 * abs(d_fd), (d_adj, d_fd)
    assert all(rel < 1e-5 for _, rel in ds.adjoint_solves)


def test_phase_loss_gradient_wrt_sphere_velocity():
    """The differentiable-asteroid loss |phi_T - phi*|^2 at a reduced size:
    gradient with respect to the sphere's velocity v0 (3 numbers), with
    checkpointing, against FP64 central differences."""
    cfg = small_cfg(res=24)
    dt = step_dt(cfg)
    steps, every = 4, 2
    pos, vel, ptype, sphere, pert = scenes.asteroid_pool(cfg, v0=(0.0, -2.0, 0.0))
    base = np.zeros_like(vel)
    base[sphere] = pert[sphere]
    # target from a run with v0 = (0.5, -2, 0)
    tgt = base.astype(np.float64).copy()
    tgt[sphere] += np.array([0.5, -2.0, 0.0])
    phi_star = oracle_phi(oracle_run(cfg, pos, tgt, ptype, dt, steps))

    ds = DiffSim(cfg, ptype, dt, checkpoint_every=every, adjoint_tol=1e-6)
    v0 = torch.tensor([0.0, -2.0, 0.0], dtype=torch.float32, device=DEV, requires_grad=True)
    mask = torch.tensor(sphere, device=DEV)[:, None].float()
    x0 = torch.tensor(pos, device=DEV)
    vinit = torch.tensor(base, device=DEV) + mask * v0[None, :]
    xT, _ = ds.rollout(x0, vinit, steps)
    phi = ds.phase_field(xT)
    L = ((phi.double() - torch.tensor(phi_star, device=DEV)) ** 2).sum()
    L.backward()
    g_adj = v0.grad.double().cpu().numpy()

    def loss(v):
        vv = base.astype(np.float64).copy()
        vv[sphere] += v
        phi_o = oracle_phi(oracle_run(cfg, pos, vv, ptype, dt, steps))
        return float(((phi_o - phi_star) ** 2).sum())

    eps = 1e-6
    v = np.array([0.0, -2.0, 0.0])
    g_fd = np.array([(loss(v + eps * e) - loss(v - eps * e)) / (2 * eps) for e in np.eye(3)])
    scale = np.abs(g_fd).max()
    assert scale > 0
    assert np.abs(g_adj - g_fd).max() <= 1e-3 * scale, (g_adj, g_fd)


# ---------------------------------------------------------------- linear stages
def test_extrapolation_transpose():
    """<E u, w> = <u, E^T w> for the seed + 3 Jacobi sweeps."""
    res = (20, 24, 28)
    g = N.grid(res, np.float32(1 / 24))
    rng = np.random.default_rng(5)
    fs = ((res[0] + 1, res[1], res[2]), (res[0], res[1] + 1, res[2]), (res[0], res[1], res[2] + 1))
    liq = torch.tensor((rng.random(res) < 0.15).astype(np.int32), device=DEV)
    u = [torch.tensor(rng.standard_normal(s).astype(np.float32), device=DEV) for s in fs]
    w = [torch.tensor(rng.standard_normal(s).astype(np.float32), device=DEV) for s in fs]
    eu = [torch.zeros(s, device=DEV) for s in fs]
    known = [torch.zeros(s, dtype=torch.int32, device=DEV) for s in fs]
    N.call("pf_extrapolate", C.byref(g), *(t.data_ptr() for t in u), liq.data_ptr(), 3,
           *(t.data_ptr() for t in eu), *(t.data_ptr() for t in known), N.stream())
    wt = [t.clone() for t in w]
    tmp = [torch.zeros(s, device=DEV) for s in fs]
    lv = [torch.empty(s, dtype=torch.uint8, device=DEV) for s in fs]
    lv2 = [torch.empty(s, dtype=torch.uint8, device=DEV) for s in fs]
    etw = [torch.zeros(s, device=DEV) for s in fs]
    N.call("pf_adj_extrapolate", C.byref(g), liq.data_ptr(), 3, *(t.data_ptr() for t in wt),
           *(t.data_ptr() for t in tmp), *(t.data_ptr() for t in lv), *(t.data_ptr() for t in lv2),
           *(t.data_ptr() for t in etw), N.stream())
    lhs = sum(float((a.double() * b.double()).sum()) for a, b in zip(eu, w))
    rhs = sum(float((a.double() * b.double()).sum()) for a, b in zip(u, etw))
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), 1.0), (lhs, rhs)


def test_g2p_field_transpose():
    """G2P is linear in (u, u*) at fixed positions: <dv', w> = <du, G^T w>."""
    cfg = small_cfg(res=16)
    res = cfg.res
    g = N.grid(res, np.float32(cfg.dx))
    rng = np.random.default_rng(9)
    n = 5000
    fs = ((17, 16, 16), (16, 17, 16), (16, 16, 17))
    pos4 = torch.zeros((n, 4), device=DEV)
    pos4[:, :3] = torch.tensor(rng.random((n, 3)).astype(np.float32), device=DEV)
    pos4.view(torch.int32)[:, 3] = torch.tensor((rng.random(n) < 0.5).astype(np.int32), device=DEV)
    vel4 = torch.zeros((n, 4), device=DEV)
    u = [torch.tensor(rng.standard_normal(s).astype(np.float32), device=DEV) for s in fs]
    us = [torch.tensor(rng.standard_normal(s).astype(np.float32), device=DEV) for s in fs]
    lo = (C.c_float * 3)(0, 0, 0)
    hi = (C.c_float * 3)(1, 1, 1)

    def g2p(uu, uss):
        p, v = pos4.clone(), vel4.clone()
        N.call("pf_g2p_advect", C.byref(g), n, p.data_ptr(), v.data_ptr(), *(t.data_ptr() for t in uu),
               *(t.data_ptr() for t in uss), None, None, None, None, 0.985, 0.96, 0.0, lo, hi, 1, 0, N.stream())
        return v[:, :3].double()

    w4 = torch.zeros((n, 4), device=DEV)
    w4[:, :3] = torch.tensor(rng.standard_normal((n, 3)).astype(np.float32), device=DEV)
    gu = [torch.zeros(s, device=DEV) for s in fs]
    gus = [torch.zeros(s, device=DEV) for s in fs]
    z4 = torch.zeros((n, 4), device=DEV)
    gp, gv = torch.zeros((n, 4), device=DEV), torch.zeros((n, 4), device=DEV)
    N.call("pf_adj_g2p_advect", C.byref(g), n, pos4.data_ptr(), vel4.data_ptr(), *(t.data_ptr() for t in u),
           *(t.data_ptr() for t in us), None, None, None, 0.985, 0.96, 0.0, lo, hi, 1, 0, z4.data_ptr(),
           w4.data_ptr(), gp.data_ptr(), gv.data_ptr(), *(t.data_ptr() for t in gu), *(t.data_ptr() for t in gus),
           None, None, None, N.stream())
    lhs = float((g2p(u, us) * w4[:, :3].double()).sum())  # v = 0, so v' = G(u, u*)
    rhs = sum(float((a.double() * b.double()).sum()) for a, b in zip(u + us, gu + gus))
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), 1.0), (lhs, rhs)


def test_unsort_inverts_the_sort_gather():
    n = 10007
    rng = np.random.default_rng(2)
    perm = torch.tensor(rng.permutation(n).astype(np.int32), device=DEV)
    a = torch.tensor(rng.standard_normal((n, 4)).astype(np.float32), device=DEV)
    b = torch.tensor(rng.standard_normal((n, 4)).astype(np.float32), device=DEV)
    oa, ob = torch.zeros_like(a), torch.zeros_like(b)
    N.call("pf_adj_unsort", n, perm.data_ptr(), a.data_ptr(), b.data_ptr(), oa.data_ptr(), ob.data_ptr(), N.stream())
    assert torch.equal(oa[perm.long()], a) and torch.equal(ob[perm.long()], b)


def test_rt_amplitude_gradient_matches_fp64_finite_differences():
    """Gradient of the final interface-height variance of the Rayleigh-Taylor
    scene (16 modes) with respect to the mode amplitudes, 32^3 / 8 ppc, 20
    steps, checkpoints every 5, against FP64 central differences of the oracle
    (the same displaced lattice).  The loss has small jumps: as particles move,
    liquid tags, valid-face tests and extrapolation masks flip, which the
    adjoint holds fixed.  A difference is therefore taken only where two
    consecutive step sizes agree (oracle.stable_central_difference); two
    components of the largest four must be checked that way."""
    from pfflip.adjoint import RTAmplitudeGradient

    cfg = small_cfg(res=32, ppc=8, seed=42)
    dt = 0.5 * cfg.dx / np.sqrt(2 * 9.81 * 0.6)
    steps = 20
    g = RTAmplitudeGradient(cfg, dt, steps, checkpoint_every=5, adjoint_tol=1e-6)
    loss, grad = g.gradient()

    def oracle_loss(amps):
        pos = scenes.rt_displace(g.pos_ref_host, amps, g.waves, cfg.domain_size)
        return O.rt_interface_variance(cfg, pos, g.ptype, dt, steps, nthreads=NTHR)

    l64 = oracle_loss(g.amps0)
    assert abs(loss - l64) <= 1e-3 * l64, (loss, l64)
    checked = []
    for k in np.argsort(-np.abs(grad))[:4]:
        fd, eps, fds = O.stable_central_difference(lambda e: oracle_loss(g.amps0 + e * np.eye(16)[k]))
        if fd is None:
            continue
        assert abs(grad[k] - fd) <= 1e-3 * abs(fd), (k, grad[k], fd, eps, fds)
        checked.append(k)
        if len(checked) == 2:
            break
    assert len(checked) == 2, checked
