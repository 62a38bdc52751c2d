"""Differentiable uniform PF-FLIP rollout.

The reference step (pfflip/sim.py:168-202) is not differentiable.  Here each
block of ``checkpoint_every`` steps is one ``torch.autograd.Function``.  Its
forward pass runs the plain step on the GPU and keeps only the particle state
at the start of the block.  Its backward pass replays the block to recover
the state before each step.  It then walks the steps in reverse: it re-runs
one step's grid stages and applies the hand-written adjoint kernels of
libpfflip.so (include/pfflip.h, "adjoint"):

    G2P + RK3 + reflection   -> pf_adj_g2p_advect   (scatter onto the faces)
    liquid extrapolation     -> pf_adj_extrapolate  (transposed sweeps)
    projection               -> pf_adj_project      (pressure and beta adjoints)
    pressure solve           -> a second MG-PCG solve with the same operator
    RHS/forces/beta/u = P/m  -> pf_adj_face_sources
    P2G                      -> pf_adj_p2g          (per-particle gather)
    sort                     -> pf_adj_unsort

Positions and velocities cross the autograd boundary as (n, 3) float32 CUDA
tensors in the caller's particle order.  Particle types are fixed.  Discrete
decisions are held fixed, so the gradient is the derivative of the step away
from its clamp/max kinks: sort order, liquid tags, extrapolation masks, wall
clamps and the valid-face test.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _native as N
from ._arrays import as_tensor
from .config import Config


class DiffSim:
    """Differentiable rollout of the uniform PF-FLIP step at a fixed dt.

    ``rollout(x, v, steps)`` returns the particle positions and velocities
    after ``steps`` steps; ``phase_field(x)`` returns the eq. (7) cell phase
    field of a particle set.  Both take part in torch autograd.
    """

    def __init__(self, cfg: Config, ptype, dt: float, checkpoint_every: int = 5, adjoint_tol: float | None = None,
                 adjoint_max_iter: int | None = None):
        from .sim import Simulator

        if cfg.k_div > 0:
            raise N.NativeError(N.PF_ERR_UNSUPPORTED, "the adjoint supports k_div = 0 only")
        if checkpoint_every < 1:
            raise ValueError("checkpoint_every must be >= 1")
        self.cfg = cfg
        self.dt = float(dt)
        self.k = int(checkpoint_every)
        self.adjoint_tol = float(cfg.pcg_tol if adjoint_tol is None else adjoint_tol)
        self.adjoint_max_iter = int(cfg.pcg_max_iter if adjoint_max_iter is None else adjoint_max_iter)
        self.sim = Simulator(cfg)
        if self.sim.has_solids:  # pragma: no cover - a fresh simulator has none
            raise N.NativeError(N.PF_ERR_UNSUPPORTED, "the adjoint does not support solids")
        dev = self.sim.dev
        t = ptype if isinstance(ptype, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(ptype))
        self.ptype = t.to(device=dev, dtype=torch.int32).reshape(-1)
        self.n = int(self.ptype.numel())
        fs = self.sim.face_shapes
        z = lambda s: torch.zeros(s, dtype=torch.float32, device=dev)  # noqa: E731
        self._gu = [z(s) for s in fs]
        self._gus = [z(s) for s in fs]
        self._gul = [z(s) for s in fs]
        self._tmp = [z(s) for s in fs]
        self._gbeta = [z(s) for s in fs]
        self._gmass = [z(s) for s in fs]
        self._gmom = [z(s) for s in fs]
        self._lv = [torch.empty(s, dtype=torch.uint8, device=dev) for s in fs]
        self._lv_tmp = [torch.empty(s, dtype=torch.uint8, device=dev) for s in fs]
        self._gp = z(self.sim.res)
        self._lam = z(self.sim.res)
        self._gphi_cell = z(self.sim.res)
        self._g4 = [torch.zeros((self.n, 4), dtype=torch.float32, device=dev) for _ in range(4)]
        self.adjoint_solves = []  # (iterations, residual) of every adjoint solve

    # ---------------------------------------------------------------- helpers
    def _load(self, x, v):
        self.sim.set_particles(x.detach(), v.detach(), self.ptype)

    def _to_ids(self, a4):
        """(n, 3) tensor in the caller's order from a float4 stream in array order."""
        ids = self.sim._ids().long()
        out = torch.empty((self.n, 3), dtype=torch.float32, device=self.sim.dev)
        out[ids] = a4[:, :3]
        return out

    def _from_ids(self, g, out4):
        """float4 stream in array order from an (n, 3) tensor in the caller's order."""
        ids = self.sim._ids().long()
        out4.zero_()
        if g is not None:
            out4[:, :3] = g.to(torch.float32)[ids]
        return out4

    def _grid_stages(self):
        """One step's forward grid stages on the current particles: sort, P2G,
        phi/beta, forces, solve, projection, extrapolation (no G2P/advection)."""
        s, dt = self.sim, self.dt
        s._p2g()
        s._phase_field_and_coefficients()
        s._add_forces(dt, save_vel_star=True)
        s._pressure_solve(dt)
        s._project(dt)
        s._extrapolate_liquid_velocity()

    def _step_adjoint(self, gpos4, gvel4, out_pos4, out_vel4):
        """Adjoint of the step whose grid stages were just run.  gpos4/gvel4
        hold the adjoints of the particles after the step (sorted order); the
        adjoints before the step's sort land in out_pos4/out_vel4."""
        s, cfg, dt = self.sim, self.cfg, self.dt
        g = C.byref(s._g)
        st = N.stream()
        P = N.ptr
        for a in self._gu + self._gus + self._gul:
            a.zero_()
        lo, hi = s._bounds()
        tmp_p, tmp_v = self._g4[2], self._g4[3]
        N.call("pf_adj_g2p_advect", g, self.n, s._pos4.data_ptr(), s._vel4.data_ptr(),
               *(P(a) for a in s.vel), *(P(a) for a in s.vel_star), *(P(a) for a in s.vel_liq),
               float(cfg.alpha_flip_liquid), float(cfg.alpha_flip_air), dt, lo, hi, 1, 1,
               gpos4.data_ptr(), gvel4.data_ptr(), tmp_p.data_ptr(), tmp_v.data_ptr(),
               *(P(a) for a in self._gu), *(P(a) for a in self._gus), *(P(a) for a in self._gul), st)
        N.call("pf_adj_extrapolate", g, P(s.is_liquid), int(cfg.extrap_cells), *(P(a) for a in self._gul),
               *(P(a) for a in self._tmp), *(P(a) for a in self._lv), *(P(a) for a in self._lv_tmp),
               *(P(a) for a in self._gu), st)
        N.call("pf_adj_project", g, P(s.pressure), *(P(a) for a in s.beta), *(P(a) for a in self._gu), dt,
               P(self._gp), *(P(a) for a in self._gbeta), st)
        it, rel = s.solver.solve(self._gp, self._lam, tol=self.adjoint_tol, max_iter=self.adjoint_max_iter)
        self.adjoint_solves.append((it, rel))
        N.call("pf_adj_face_sources", g, P(s.pressure), P(self._lam), *(P(a) for a in s.beta),
               *(P(a) for a in s.mass), *(P(a) for a in s.mom), P(s.is_liquid), float(1e-12 * s.rho_0l),
               float(s.rho_min), float(cfg.alpha_phi), float(s.rho_0l), float(cfg.rho_l), float(cfg.rho_g), dt,
               *(P(a) for a in self._gu), *(P(a) for a in self._gus), *(P(a) for a in self._gbeta),
               *(P(a) for a in self._gmass), *(P(a) for a in self._gmom), st)
        N.call("pf_adj_p2g", g, self.n, s._pos4.data_ptr(), s._vel4.data_ptr(), float(cfg.rho_l), float(cfg.rho_g),
               float(np.float32(cfg.r_p)), *(P(a) for a in self._gmass), *(P(a) for a in self._gmom), None,
               tmp_p.data_ptr(), tmp_v.data_ptr(), st)
        N.call("pf_adj_unsort", self.n, s._perm.data_ptr(), tmp_p.data_ptr(), tmp_v.data_ptr(),
               out_pos4.data_ptr(), out_vel4.data_ptr(), st)

    # ---------------------------------------------------------------- blocks
    def _forward_block(self, x, v, nsteps):
        self._load(x, v)
        for _ in range(nsteps):
            self.sim.step(self.dt)
        return self._to_ids(self.sim._pos4), self._to_ids(self.sim._vel4)

    def _saved_fields(self):
        s = self.sim
        return [as_tensor(a) for a in (*s.vel, *s.vel_star, *s.vel_liq, *s.beta, *s.mass, *s.mom, s.is_liquid,
                                        s.pressure)]

    def _snapshot(self):
        """Everything the step's adjoint reads, right after its grid stages: the
        sorted particles, the sort permutation and the grid fields."""
        s = self.sim
        return (s._pos4.clone(), s._vel4.clone(), s._perm.clone(), [t.clone() for t in self._saved_fields()])

    def _restore(self, snap):
        s = self.sim
        p4, v4, perm, fields = snap
        s._pos4.copy_(p4)
        s._vel4.copy_(v4)
        s._perm.copy_(perm)
        for t, src in zip(self._saved_fields(), fields):
            t.copy_(src)
        s.solver.build_hierarchy(*s.beta)  # the adjoint solve uses this step's operator
        s._particles_changed()

    def _backward_block(self, x, v, nsteps, gx, gv):
        """Replay the block once, keeping each step's grid state (its sorted
        particles, permutation and fields: about 0.1 GB per step at 64^3 / 8
        ppc), then walk the steps in reverse, restoring that state for each
        step's adjoint instead of recomputing the step's grid stages."""
        s = self.sim
        self._load(x, v)
        s._particles_changed()  # step 0 sorts again (the identity), so its permutation maps onto this order
        snaps = []
        for _ in range(nsteps):
            self._grid_stages()
            snaps.append(self._snapshot())
            s._g2p_advect(self.dt, do_g2p=True, do_advect=True)
        ga, gb = self._g4[0], self._g4[1]
        self._from_ids(gx, ga)
        self._from_ids(gv, gb)
        for k in range(nsteps - 1, -1, -1):
            self._restore(snaps[k])
            snaps[k] = None
            # ga/gb are in the order of the arrays after the step, which is the
            # order after the step's sort; the result is in the order before it
            nxt_p, nxt_v = torch.empty_like(ga), torch.empty_like(gb)
            self._step_adjoint(ga, gb, nxt_p, nxt_v)
            ga, gb = nxt_p, nxt_v
        # step 0's sort was the identity on the loaded order, so the snapshot's
        # ids give the order ga/gb use
        return self._to_ids(ga), self._to_ids(gb)

    def rollout(self, x, v, steps: int):
        """Positions and velocities after ``steps`` steps of size dt."""
        left = int(steps)
        while left > 0:
            m = min(self.k, left)
            x, v = _Block.apply(x, v, self, m)
            left -= m
        return x, v

    def phase_field(self, x):
        """eq. (7) cell phase field of the particles at x (shape = cfg.res)."""
        return _Phase.apply(x, self)

    def _phase_forward(self, x):
        s = self.sim
        self._load(x, torch.zeros_like(x))
        s._p2g()
        s._phase_field_and_coefficients()
        return as_tensor(s.phi_cell).clone()

    def _phase_backward(self, x, gphi):
        s, cfg = self.sim, self.cfg
        self._load(x, torch.zeros_like(x))
        s._p2g()
        s._phase_field_and_coefficients()
        self._gphi_cell.copy_(gphi)
        gcell = self._gp  # cell-sized scratch
        N.call("pf_adj_phase_cell", C.byref(s._g), N.ptr(s.cell_mass), self._gphi_cell.data_ptr(),
               float(s.rho_min), float(cfg.alpha_phi), float(s.rho_0l), gcell.data_ptr(), N.stream())
        ga, gb = self._g4[0], self._g4[1]
        ga.zero_()
        gb.zero_()
        N.call("pf_adj_p2g", C.byref(s._g), self.n, s._pos4.data_ptr(), s._vel4.data_ptr(), float(cfg.rho_l),
               float(cfg.rho_g), float(np.float32(cfg.r_p)), None, None, None, None, None, None, gcell.data_ptr(),
               ga.data_ptr(), gb.data_ptr(), N.stream())
        return self._to_ids(ga)


class _Block(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, v, dsim, nsteps):
        ctx.dsim = dsim
        ctx.nsteps = nsteps
        ctx.save_for_backward(x.detach().clone(), v.detach().clone())
        with torch.no_grad():
            return dsim._forward_block(x, v, nsteps)

    @staticmethod
    def backward(ctx, gx, gv):
        x, v = ctx.saved_tensors
        with torch.no_grad():
            ax, av = ctx.dsim._backward_block(x, v, ctx.nsteps, gx, gv)
        return ax, av, None, None


class _Phase(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, dsim):
        ctx.dsim = dsim
        ctx.save_for_backward(x.detach().clone())
        with torch.no_grad():
            return dsim._phase_forward(x)

    @staticmethod
    def backward(ctx, gphi):
        (x,) = ctx.saved_tensors
        with torch.no_grad():
            gx = ctx.dsim._phase_backward(x, gphi.contiguous())
        return gx, None


class RTAmplitudeGradient:
    """Gradient of the final interface-height variance of the Rayleigh-Taylor
    scene with respect to its 16 mode amplitudes a_k.

    The liquid (heavy, rho_l) tags are piecewise constant in a_k, so the
    amplitudes enter through the particle positions instead: the jittered
    lattice is tagged by its reference height (heavy above Ly/2) and displaced
    vertically by D a, D[p, k] = Ly sin^2(pi y/Ly) cos(2 pi (m_k x + n_k z))
    (scenes.rt_profile), which carries the plane Ly/2 onto the interface
    0.5 + sum_k a_k cos(...).  After ``steps`` steps the light-phase height of
    every (x, z) column is h = dx sum_y (1 - phi) and the loss is the variance
    of h over the columns.  d loss / d a = D^T (d loss / d x0) through the
    adjoint rollout (DiffSim) and the adjoint of eq. (7)."""

    def __init__(self, cfg: Config, dt: float, steps: int, checkpoint_every: int = 5,
                 adjoint_tol: float | None = 1e-6, n_modes: int = 16):
        from . import scenes

        pos_ref, ptype, amps, waves = scenes.rayleigh_taylor_lattice(cfg, n_modes)
        self.cfg = cfg
        self.steps = int(steps)
        self.amps0 = np.asarray(amps, np.float64)
        self.waves = np.asarray(waves)
        self.pos_ref_host = pos_ref
        self.ptype = ptype
        self.ds = DiffSim(cfg, ptype, dt, checkpoint_every=checkpoint_every, adjoint_tol=adjoint_tol)
        dev = self.ds.sim.dev
        ref = torch.from_numpy(pos_ref).to(dev)
        self.pos_ref = ref
        self.profile = scenes.rt_profile(ref.double(), self.waves, cfg.domain_size, xp=torch).float()

    def positions(self, a):
        """Initial positions for amplitudes a ((n_modes,) tensor)."""
        dy = self.profile @ a.to(device=self.profile.device, dtype=torch.float32)
        x = self.pos_ref
        return torch.stack((x[:, 0], x[:, 1] + dy, x[:, 2]), dim=1)

    def interface_variance(self, phi):
        h = (1.0 - phi.double()).sum(dim=1) * self.cfg.dx  # (nx, nz) light-phase column heights
        return ((h - h.mean()) ** 2).mean()

    def loss(self, a):
        x0 = self.positions(a)
        xT, _ = self.ds.rollout(x0, torch.zeros_like(x0), self.steps)
        return self.interface_variance(self.ds.phase_field(xT))

    def gradient(self, a=None):
        """(loss, d loss / d a) at amplitudes a (default: the seeded ones)."""
        a = torch.tensor(self.amps0 if a is None else a, dtype=torch.float64, device=self.ds.sim.dev,
                         requires_grad=True)
        loss = self.loss(a)
        loss.backward()
        return float(loss.detach()), a.grad.double().cpu().numpy()
