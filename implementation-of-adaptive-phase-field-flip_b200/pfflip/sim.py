"""PF-FLIP simulator on a uniform MAC grid (B200, sm_100a).

``Simulator`` keeps the constructor, methods, stage methods, attributes and
stats of the reference's ``pfflip.sim.Simulator`` (``pfflip/sim.py:37-424``) for
the uniform step; all stage work runs in libpfflip.so:

==========================  ===============================================
reference stage              libpfflip entry point(s)
==========================  ===============================================
(new) particle sort          pf_sort_particles
``_p2g``                     pf_p2g (+ the face velocities in pf_phase_beta)
``_phase_field_and_coef.``   pf_phase_beta
vel_star copy + forces       pf_save_and_force
``_pressure_solve``          pf_build_rhs, pf_mg_build_hierarchy, pf_mg_solve
``_project``                 pf_project
``_max_divergence``          pf_max_divergence
``_extrapolate_liquid_vel.`` pf_extrapolate
``_g2p`` + ``_advect``       pf_g2p_advect_packed (one fused pass inside
                             ``step`` when droplets are off)
``_droplets``                pf_droplet_classify, pf_velocity_gradient,
                             pf_spray_emit, pf_droplet_advance
``rasterize_spray``          pf_spray_rasterize
==========================  ===============================================

Particles live on the device as two float4 streams sorted by cell (see
include/pfflip.h); ``px``, ``pv``, ``ptype``, ``pmass``, ``pstate``, ``pdrop_r``
present them in the caller's original order.  With ``cfg.droplets`` the step
keeps the reference's order G2P -> extrapolation -> droplets -> advection.
"""

from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np
import torch

from . import _native as N
from ._arrays import DeviceArray, as_tensor
from .config import Config
from .poisson import MGPCG, default_coef_scale


def calibrate_rho_tilde_0(dx: float, r: float, ppc: int) -> float:
    """rho~_0: eq. (6) kernel-weight sum at a point of a perfect lattice.

    The lattice has ``round(ppc^(1/3))`` sites per cell and axis; the sample
    point sits half a lattice step off every site, as in the reference's
    calibration (pfflip/sim.py:119-140)."""
    pa = round(ppc ** (1.0 / 3.0))
    step = dx / pa
    R = int(math.ceil(r / step)) + 1
    o2 = (np.arange(-R, R + 1) + 0.5) ** 2
    d2 = (o2[:, None, None] + o2[None, :, None] + o2[None, None, :]) * step * step
    t = np.maximum(1.0 - d2 / (r * r), 0.0)
    return float((t * t * t).sum())


class ParticleField:
    """One particle attribute in the caller's original order.

    ``numpy()`` un-permutes the sorted device streams; ``assign(a)`` writes an
    array given in original order into the sorted slots."""

    def __init__(self, sim, kind):
        self._sim = sim
        self._kind = kind

    @property
    def shape(self):
        n = self._sim.n_particles
        return (n, 3) if self._kind in ("pos", "vel") else (n,)

    def _tensor(self):
        s, k = self._sim, self._kind
        ids = s._ids().long()
        if k in ("pos", "vel"):
            src = (s._pos4 if k == "pos" else s._vel4)[:, :3]
            out = torch.empty_like(src)
            out[ids] = src
            return out
        flags = s._flags()
        if k == "ptype":
            v = flags & N_FLAG_LIQUID
        elif k == "pstate":
            v = (flags >> N_PSTATE_SHIFT) & 3
        elif k == "pmass":
            cfg = s.cfg
            v = torch.where((flags & N_FLAG_LIQUID) != 0, torch.tensor(cfg.rho_l, dtype=torch.float32, device=s.dev),
                            torch.tensor(cfg.rho_g, dtype=torch.float32, device=s.dev))
        elif k == "prad":
            v = torch.full_like(flags, 0, dtype=torch.float32) + float(np.float32(s.cfg.r_p))
        elif k == "pdrop_r":
            v = s._drop_r
        out = torch.empty_like(v)
        out[ids] = v
        return out

    def numpy(self):
        return self._tensor().cpu().numpy()

    def __array__(self, dtype=None, copy=None):
        a = self.numpy()
        return a if dtype is None else a.astype(dtype)

    def assign(self, a):
        s, k = self._sim, self._kind
        s._particles_changed()
        ids = s._ids().long()
        t = torch.as_tensor(np.ascontiguousarray(np.asarray(a))).to(s.dev)
        if k in ("pos", "vel"):
            dst = s._pos4 if k == "pos" else s._vel4
            dst[:, :3] = t.reshape(-1, 3).to(torch.float32)[ids]
            return self
        if k == "pdrop_r":
            s._drop_r[:] = t.reshape(-1).to(torch.float32)[ids]
            return self
        if k not in ("ptype", "pstate"):
            raise TypeError(f"{k} is derived from the particle type and cannot be assigned")
        flags = s._flags()
        v = t.reshape(-1).to(torch.int32)[ids]
        if k == "ptype":
            flags = (flags & ~N_FLAG_LIQUID) | (v == 1).to(torch.int32)
        else:
            flags = (flags & N_FLAG_LIQUID) | ((v & 3) << N_PSTATE_SHIFT)
        s._pos4.view(torch.int32)[:, 3] = flags
        return self


N_FLAG_LIQUID = 1
N_PSTATE_SHIFT = 1


class Simulator:
    def __init__(self, cfg: Config):
        self.cfg = cfg
        self.dev = N.require_cuda(cfg.device)
        nx, ny, nz = (int(n) for n in cfg.res)
        self.res = (nx, ny, nz)
        self._g = N.grid(self.res, np.float32(cfg.dx))
        self.face_shapes = ((nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1))
        z = lambda shape: DeviceArray.zeros(shape, torch.float32, self.dev)  # noqa: E731
        zi = lambda shape: DeviceArray.zeros(shape, torch.int32, self.dev)  # noqa: E731
        fs = self.face_shapes
        self.vel = [z(s) for s in fs]
        self.vel_star = [z(s) for s in fs]
        self.vel_liq = [z(s) for s in fs]
        self.mass = [z(s) for s in fs]
        self.mom = [z(s) for s in fs]
        self.beta = [z(s) for s in fs]
        self.phi_face = [z(s) for s in fs]
        self.valid = [zi(s) for s in fs]
        self._known = [zi(s) for s in fs]
        self.cell_mass = z(self.res)
        self.cell_wsum = z(self.res)
        self.phi_cell = z(self.res)
        self.is_liquid = zi(self.res)
        self.solid = zi(self.res)
        self.pressure = z(self.res)
        self.rhs = z(self.res)
        self._scal = torch.zeros(8, dtype=torch.float32, device=self.dev)

        self.solver = MGPCG(
            self.res, self.dev, omega=cfg.mg_omega, pre=cfg.mg_pre_sweeps, post=cfg.mg_post_sweeps,
            coarsest=cfg.mg_coarsest_sweeps, min_dim=cfg.mg_min_dim, precision=cfg.precision,
            stencil=cfg.stencil, coef_scale=default_coef_scale(cfg.rho_l, cfg.rho_g), use_graphs=cfg.cuda_graphs,
        )

        self.n_particles = 0
        # True only between set_particles (which sorts) and the next stage: the
        # step's own sort would then repeat it on the same particles
        self._fresh_sort = False
        # True while _scal[2] holds the CFL speed of the particles as they are:
        # the step's last particle pass leaves it there, and anything else that
        # changes particle velocities or states clears this
        self._vmax_valid = False
        self._pending_d2h = []  # (host lo, host hi, event) of read_particles' chunked downloads
        self._pos4 = self._vel4 = None
        self.droplet_stats = {"emitted": 0, "bubbles": 0, "merged": 0, "spray": 0}

        self.rho_tilde_0 = calibrate_rho_tilde_0(cfg.dx, cfg.r_p, cfg.ppc)
        self.rho_0l = self.rho_tilde_0 * cfg.rho_l
        self.rho_min = cfg.eta_phi * cfg.rho_g * self.rho_tilde_0

        self.has_solids = False
        self.time = 0.0
        self.step_index = 0
        self.stats: list[dict] = []
        self._marks = None  # per-stage CUDA events when stage timing is on
        self._g2p_ws = None  # (j, k) quads of the face fields read by the G2P/advection pass

        self.px = ParticleField(self, "pos")
        self.pv = ParticleField(self, "vel")
        self.ptype = ParticleField(self, "ptype")
        self.pstate = ParticleField(self, "pstate")
        self.pdrop_r = ParticleField(self, "pdrop_r")
        # spray density field at spray_resolution_factor x the grid (pfflip/sim.py:94-98)
        f = max(1, int(cfg.spray_resolution_factor))
        self.spray_res = tuple(n * f for n in self.res)
        self.dx_spray = cfg.dx / f
        self.spray_density = None  # float16, allocated by the first rasterize_spray()
        self.shear = None
        self._counters = torch.zeros(4, dtype=torch.int32, device=self.dev)
        self.pmass = ParticleField(self, "pmass")
        self.prad = ParticleField(self, "prad")

    # ------------------------------------------------------------------ setup
    def set_solids(self, mask: np.ndarray):
        """Install an obstacle mask (True = solid) on the cell grid."""
        self.solid.assign(np.ascontiguousarray(mask, np.int32))
        self.has_solids = bool(np.any(mask))

    def set_particles(self, pos, vel, ptype):
        """Upload particles: (n,3) positions and velocities, (n,) types (0 air,
        1 liquid), as NumPy arrays or host/device torch tensors.  Buffers are
        reused when the particle count is unchanged."""
        t = lambda a, dt: (a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a))).to(dt)  # noqa: E731
        pos = t(pos, torch.float32).reshape(-1, 3)
        vel = t(vel, torch.float32).reshape(-1, 3)
        ptype = t(ptype, torch.int32).reshape(-1)
        n = pos.shape[0]
        if vel.shape[0] != n or ptype.shape[0] != n:
            raise ValueError("pos, vel and ptype must have the same length")
        dev = self.dev
        if self._pos4 is None or self.n_particles != n:
            self._alloc_particles(n)
        self.n_particles = n
        p4, v4 = self._pos4, self._vel4
        main = torch.cuda.current_stream(dev)
        if pos.device.type == "cpu" and vel.device.type == "cpu" and ptype.device.type == "cpu":
            # host arrays: the uploads run on the upload stream, each one
            # overlapping the packing of the previous array on this stream.
            # A host range that read_particles is still filling is uploaded
            # chunk by chunk behind the download of that range (see _upload)
            up = self._copy_streams()[1]
            pending, self._pending_d2h = self._pending_d2h, []
            staged = {}
            with torch.cuda.stream(up):
                for name, a in (("t", ptype), ("p", pos), ("v", vel)):  # the types first: nothing writes them
                    d = self._upload(a, pending, up)
                    staged[name] = (d, up.record_event())
            for d, _ in staged.values():
                d.record_stream(main)
            (dpos, ep), (dvel, ev), (dpt, et) = staged["p"], staged["v"], staged["t"]
        else:
            dpos, dvel, dpt = pos.to(dev), vel.to(dev), ptype.to(dev)
            ep = ev = et = None
        if ep is not None:
            main.wait_event(ep)
        p4[:, :3].copy_(dpos)
        if ev is not None:
            main.wait_event(ev)
        v4[:, :3].copy_(dvel)
        if et is not None:
            main.wait_event(et)
        # the liquid flag is formed on the device: a host-side comparison would
        # be a CPU pass over n values and an unpinned copy
        p4.view(torch.int32)[:, 3].copy_((dpt == 1).to(torch.int32))
        v4.view(torch.int32)[:, 3] = torch.arange(n, dtype=torch.int32, device=dev)
        if self.cfg.droplets:
            self._drop_r.zero_()
        self._sort()
        self._fresh_sort = True
        self._vmax_valid = False

    def read_particles(self, pos_out=None, vel_out=None, sync=True):
        """Positions and velocities in the original order, copied into the given
        (pinned) host tensors when provided; returns (pos, vel).

        With contiguous host tensors given, each copy runs on the download
        stream in chunks of _CHUNK bytes, the positions' copy overlapping the
        reordering of the velocities; the caller's stream waits for both.  The
        chunks' events stay recorded, so that a set_particles from these same
        host buffers uploads each chunk as soon as its download has landed.

        sync=True (the default) returns only once the host tensors hold the
        values, as the reference's synchronous read does.  sync=False returns
        as soon as the copies are queued: the host must not read pos_out or
        vel_out before torch.cuda.synchronize() (or the caller's stream) says
        they have landed; handing them straight back to set_particles is safe,
        which is what lets a host round trip per step overlap its uploads with
        the downloads."""
        ids = self._ids().long()
        main = torch.cuda.current_stream(self.dev)
        out = []
        copied = False
        pending = []
        for src, dst in ((self._pos4, pos_out), (self._vel4, vel_out)):
            tmp = torch.empty((self.n_particles, 3), dtype=torch.float32, device=self.dev)
            tmp[ids] = src[:, :3]
            if dst is None:
                out.append(tmp.cpu())
            elif dst.device.type == "cpu" and dst.is_contiguous():
                down = self._copy_streams()[0]
                down.wait_stream(main)
                fd, ft = dst.view(-1), tmp.view(-1)
                step = self._CHUNK // 4
                with torch.cuda.stream(down):
                    for off in range(0, fd.numel(), step):
                        m = min(step, fd.numel() - off)
                        fd[off:off + m].copy_(ft[off:off + m], non_blocking=True)
                        lo = dst.data_ptr() + 4 * off
                        pending.append((lo, lo + 4 * m, down.record_event()))
                tmp.record_stream(down)
                copied = True
                out.append(dst)
            else:
                dst.copy_(tmp)
                out.append(dst)
        if copied:
            main.wait_stream(self._copy_streams()[0])
            if sync:
                self._copy_streams()[0].synchronize()
        self._pending_d2h = pending
        return tuple(out)

    _CHUNK = 1 << 25  # bytes per chunk of a host<->device particle copy

    def _copy_streams(self):
        """(download, upload) side streams of the host<->device particle copies."""
        if getattr(self, "_cstreams", None) is None:
            self._cstreams = (torch.cuda.Stream(device=self.dev), torch.cuda.Stream(device=self.dev))
        return self._cstreams

    def _upload(self, a, pending, stream):
        """Device copy of host array a, enqueued on `stream` (the current
        stream), chunk by chunk; a chunk whose host bytes overlap a pending
        download waits for that download's event."""
        d = torch.empty(a.shape, dtype=a.dtype, device=self.dev)
        if not pending or not a.is_contiguous():
            for _, _, ev in pending:
                stream.wait_event(ev)
            d.copy_(a, non_blocking=True)
            return d
        fa, fd = a.view(-1), d.view(-1)
        es = a.element_size()
        step = self._CHUNK // es
        for off in range(0, fa.numel(), step):
            m = min(step, fa.numel() - off)
            lo = a.data_ptr() + es * off
            hi = lo + es * m
            for b0, b1, ev in pending:
                if b0 < hi and lo < b1:
                    stream.wait_event(ev)
            fd[off:off + m].copy_(fa[off:off + m], non_blocking=True)
        return d

    def _alloc_particles(self, n):
        # each stream is a view of the first n rows of at least one row of
        # storage, so that an empty particle set still passes valid device
        # pointers (the library launches nothing for n = 0)
        dev = self.dev
        m = max(n, 1)

        def rows(*shape, dtype=torch.float32, zero=False):
            a = (torch.zeros if zero else torch.empty)((m,) + shape, dtype=dtype, device=dev)
            return a[:n]

        self._drop_r = rows(zero=True)
        self._drop_r_alt = rows()
        self._pos4 = rows(4)
        self._vel4 = rows(4)
        self._pos4_alt = rows(4)
        self._vel4_alt = rows(4)
        self._keys = rows(dtype=torch.int32)
        self._perm = rows(dtype=torch.int32)
        nc = self.res[0] * self.res[1] * self.res[2]
        self._cell_start = torch.zeros(nc + 1, dtype=torch.int32, device=dev)
        wsb = int(N.lib().pf_sort_workspace_bytes(C.byref(self._g), n))
        self._sort_ws = torch.empty(wsb, dtype=torch.uint8, device=dev)

    def _ids(self):
        return self._vel4.view(torch.int32)[:, 3]

    def _flags(self):
        return self._pos4.view(torch.int32)[:, 3]

    def _sort(self):
        """Counting sort of the particle streams by cell (new stage; the
        reference never reorders particles)."""
        n = self.n_particles
        N.call("pf_sort_particles", C.byref(self._g), n, N.sptr(self._pos4), N.sptr(self._vel4),
               N.sptr(self._pos4_alt), N.sptr(self._vel4_alt), N.sptr(self._keys), N.sptr(self._perm),
               self._cell_start.data_ptr(), self._sort_ws.data_ptr(), self._sort_ws.numel(), N.stream())
        self._pos4, self._pos4_alt = self._pos4_alt, self._pos4
        self._vel4, self._vel4_alt = self._vel4_alt, self._vel4
        if self.cfg.droplets:  # the droplet radius follows its particle
            N.call("pf_permute_f32", n, N.sptr(self._perm), N.sptr(self._drop_r), N.sptr(self._drop_r_alt),
                   N.stream())
            self._drop_r, self._drop_r_alt = self._drop_r_alt, self._drop_r

    # ------------------------------------------------------------------ timing
    def enable_stage_timing(self, on: bool = True):
        """Record a CUDA event at every stage boundary of ``step`` (no syncs)."""
        self._marks = [] if on else None

    def _mark(self, name):
        if self._marks is not None:
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            self._marks.append((name, e))

    def stage_times(self, reset=True):
        """Per-stage device time over the recorded steps: {stage: (launches, total_ms)}."""
        torch.cuda.synchronize(self.dev)
        out = {}
        m = self._marks or []
        for (name, e0), (_, e1) in zip(m[:-1], m[1:]):
            if name == "<end>":
                continue
            c, t = out.get(name, (0, 0.0))
            out[name] = (c + 1, t + e0.elapsed_time(e1))
        if reset and self._marks is not None:
            self._marks = []
        return out

    # ------------------------------------------------------------------ step
    def _particles_changed(self):
        """Particle positions, velocities or states were written outside the
        step: neither the last sort nor the last CFL speed describes them."""
        self._fresh_sort = False
        self._vmax_valid = False

    def dt_from_cfl(self) -> float:
        """CFL time step (pfflip/sim.py:157-166).  Right after a step the FLIP
        particles' max speed is already on the device (the step's last particle
        pass reduces it); otherwise one pf_particle_max_speed pass computes it."""
        cfg = self.cfg
        if self._vmax_valid:
            vmax = float(self._scal[2].item())
        else:
            N.call("pf_particle_max_speed", self.n_particles, N.sptr(self._pos4), N.sptr(self._vel4),
                   self._scal.data_ptr(), N.stream())
            vmax = float(self._scal[0].item())
        g = float(np.linalg.norm(cfg.gravity))
        vmax = max(vmax, math.sqrt(2.0 * g * cfg.dx) if g > 0 else 0.0, 1e-8)
        return float(np.clip(cfg.cfl * cfg.dx / vmax, cfg.dt_min, cfg.dt_max))

    def step(self, dt: float | None = None, verbose: bool = False) -> dict:
        if dt is None:
            dt = self.dt_from_cfl()
        t0 = time.perf_counter()
        mark = self._mark
        self._p2g(mark=mark)
        mark("phase_beta")
        self._phase_field_and_coefficients()
        mark("forces")
        self._add_forces(dt, save_vel_star=True)
        pcg_it, pcg_res = self._pressure_solve(dt, verbose=verbose, mark=mark)
        mark("project")
        self._project(dt)
        mark("divergence")
        self._divergence_async()
        if self.cfg.droplets:
            # the reference's order (pfflip/sim.py:182-185): droplet
            # conversions sit between G2P and advection, so the passes split
            mark("g2p_advect")
            self._g2p()
            mark("extrapolate")
            self._extrapolate_liquid_velocity()
            mark("droplets")
            self._droplets(dt)
            mark("g2p_advect")
            self._advect(dt)
        else:
            mark("extrapolate")
            self._extrapolate_liquid_velocity()
            mark("g2p_advect")
            self._g2p_advect(dt, do_g2p=True, do_advect=True)
        mark("<end>")
        div_after = float(self._scal[1].item())  # synchronises the stream
        wall = time.perf_counter() - t0
        self.time += dt
        self.step_index += 1
        rec = {
            "step": self.step_index,
            "t": self.time,
            "dt": dt,
            "pcg_iter": pcg_it,
            "pcg_res": pcg_res,
            "max_div": div_after,
            "droplets": self._droplet_count() if self.cfg.droplets else 0,
            "wall_s": wall,
        }
        self.stats.append(rec)
        return rec

    # ------------------------------------------------------------------ stages
    def _p2g(self, mark=None):
        """Sort, then eq. (3)-(6) splatting to faces and cells (pfflip/sim.py:205-236)."""
        cfg = self.cfg
        if mark:
            mark("sort")
        if self._fresh_sort:  # set_particles sorted these very particles
            self._fresh_sort = False
        else:
            self._sort()
        if mark:
            mark("p2g")
        N.call("pf_p2g", C.byref(self._g), self.n_particles, N.sptr(self._pos4), N.sptr(self._vel4),
               self._cell_start.data_ptr(), float(cfg.rho_l), float(cfg.rho_g), float(np.float32(cfg.r_p)),
               *(N.ptr(a) for a in self.mass), *(N.ptr(a) for a in self.mom), N.ptr(self.cell_mass),
               N.ptr(self.cell_wsum), N.stream())

    def _phase_field_and_coefficients(self):
        """u = P/m, eq. (7) phi, eq. (9) beta, walls and obstacles (pfflip/sim.py:229-268)."""
        cfg = self.cfg
        N.call("pf_phase_beta", C.byref(self._g), *(N.ptr(a) for a in self.mass), *(N.ptr(a) for a in self.mom),
               N.ptr(self.cell_mass), N.ptr(self.solid) if self.has_solids else None, float(1e-12 * self.rho_0l),
               float(self.rho_min), float(cfg.alpha_phi), float(self.rho_0l), float(cfg.rho_l), float(cfg.rho_g),
               *(N.ptr(a) for a in self.vel), *(N.ptr(a) for a in self.valid), N.ptr(self.phi_cell),
               N.ptr(self.is_liquid), *(N.ptr(a) for a in self.phi_face), *(N.ptr(a) for a in self.beta), N.stream())

    def _add_forces(self, dt: float, save_vel_star: bool = False):
        """Gravity and wall/obstacle zeroing (pfflip/sim.py:270-285); with
        save_vel_star the pre-force copy of pfflip/sim.py:176-177 is fused in."""
        g = self.cfg.gravity
        vs = [N.ptr(a) for a in self.vel_star] if save_vel_star else [None, None, None]
        N.call("pf_save_and_force", C.byref(self._g), *(N.ptr(a) for a in self.vel), *vs,
               N.ptr(self.solid) if self.has_solids else None, float(g[0]), float(g[1]), float(g[2]), float(dt),
               N.stream())

    def _pressure_solve(self, dt: float, verbose: bool = False, mark=None):
        cfg = self.cfg
        if mark:
            mark("rhs")
        N.call("pf_build_rhs", C.byref(self._g), *(N.ptr(a) for a in self.vel), N.ptr(self.cell_wsum),
               N.ptr(self.rhs), float(dt), float(self.rho_tilde_0), float(cfg.k_div), N.stream())
        if mark:
            mark("hierarchy")
        self.solver.build_hierarchy(*self.beta)
        if mark:
            mark("solve")
        return self.solver.solve(self.rhs, self.pressure, tol=cfg.pcg_tol, max_iter=cfg.pcg_max_iter,
                                 verbose=verbose)

    def _project(self, dt: float):
        N.call("pf_project", C.byref(self._g), N.ptr(self.pressure), *(N.ptr(a) for a in self.beta),
               *(N.ptr(a) for a in self.vel), float(dt), N.stream())

    def _divergence_async(self):
        N.call("pf_max_divergence", C.byref(self._g), *(N.ptr(a) for a in self.vel), self._scal.data_ptr() + 4,
               N.stream())

    def _max_divergence(self) -> float:
        self._divergence_async()
        return float(self._scal[1].item())

    def _extrapolate_liquid_velocity(self):
        N.call("pf_extrapolate", C.byref(self._g), *(N.ptr(a) for a in self.vel), N.ptr(self.is_liquid),
               int(self.cfg.extrap_cells), *(N.ptr(a) for a in self.vel_liq), *(N.ptr(a) for a in self._known),
               N.stream())

    def _bounds(self):
        eps = 1e-4 * self.cfg.dx
        lo = (C.c_float * 3)(eps, eps, eps)
        hi = (C.c_float * 3)(*[s - eps for s in self.cfg.domain_size])
        return lo, hi

    def _g2p_advect(self, dt, do_g2p, do_advect):
        self._particles_changed()
        lo, hi = self._bounds()
        cfg = self.cfg
        if self._g2p_ws is None:
            nb = int(N.lib().pf_g2p_workspace_bytes(C.byref(self._g)))
            self._g2p_ws = torch.empty(nb, dtype=torch.uint8, device=self.dev)
        N.call("pf_g2p_advect_packed", C.byref(self._g), self.n_particles, N.sptr(self._pos4),
               N.sptr(self._vel4), *(N.ptr(a) for a in self.vel), *(N.ptr(a) for a in self.vel_star),
               *(N.ptr(a) for a in self.vel_liq), N.ptr(self.solid) if self.has_solids else None,
               float(cfg.alpha_flip_liquid), float(cfg.alpha_flip_air), float(dt), lo, hi, int(do_g2p),
               int(do_advect), self._scal.data_ptr() + 8 if do_advect else None, self._g2p_ws.data_ptr(),
               self._g2p_ws.numel(), N.stream())
        # after an advection pass the particles are as the step leaves them
        self._vmax_valid = bool(do_advect)

    def _g2p(self):
        """eq. (11)-(12) FLIP/PIC update (pfflip/sim.py:316-327)."""
        self._g2p_advect(0.0, do_g2p=True, do_advect=False)

    def _advect(self, dt: float):
        """RK3 advection and wall reflection (pfflip/sim.py:408-424); needs
        ``_extrapolate_liquid_velocity`` first, as in the reference."""
        self._g2p_advect(dt, do_g2p=False, do_advect=True)

    def _droplets(self, dt: float):
        """Escaped particles -> droplets, droplet dynamics (pfflip/sim.py:343-392)."""
        self._particles_changed()
        cfg = self.cfg
        if not cfg.droplets or self.n_particles == 0:
            return
        mean_r = cfg.droplet_radius_mean * cfg.dx
        sigma = float(cfg.droplet_radius_spread)
        mu = float(np.log(mean_r) - 0.5 * sigma * sigma)  # pfflip/droplets.py:356-360
        r_min, r_max = 0.02 * cfg.dx, 2.0 * cfg.dx
        seed = (int(cfg.seed) + int(self.step_index)) & 0xFFFFFFFF
        g, n, st = C.byref(self._g), self.n_particles, N.stream()
        self._counters.zero_()
        N.call("pf_droplet_classify", g, n, N.sptr(self._pos4), N.sptr(self._vel4), N.sptr(self._drop_r),
               N.ptr(self.phi_cell), float(cfg.delta_phi), mu, sigma, float(r_min), float(r_max), seed,
               self._counters.data_ptr(), st)
        if cfg.spray_shear_threshold > 0.0:
            if self.shear is None:
                self.shear = DeviceArray(torch.zeros(self.res, dtype=torch.float32, device=self.dev))
            N.call("pf_velocity_gradient", g, *(N.ptr(a) for a in self.vel), N.ptr(self.shear), st)
            N.call("pf_spray_emit", g, n, N.sptr(self._pos4), N.sptr(self._vel4), N.sptr(self._drop_r),
                   N.ptr(self.phi_cell), N.ptr(self.shear), float(cfg.spray_shear_threshold),
                   float(cfg.spray_emission_rate), mu, sigma, float(r_min), float(r_max), seed,
                   self._counters.data_ptr(), st)
        lo, hi = self._bounds()
        grav = (C.c_float * 3)(*[float(x) for x in cfg.gravity])
        N.call("pf_droplet_advance", g, n, N.sptr(self._pos4), N.sptr(self._vel4), N.sptr(self._drop_r),
               *(N.ptr(a) for a in self.vel), float(dt), grav, float(cfg.rho_g), float(cfg.rho_l),
               float(cfg.droplet_drag_cd), float(cfg.evaporation_k * cfg.dx * cfg.dx), float(r_min), lo, hi,
               int(cfg.droplet_max_substeps), st)
        c = self._counters.cpu().numpy()
        for k, i in (("emitted", 0), ("bubbles", 1), ("merged", 2), ("spray", 3)):
            self.droplet_stats[k] += int(c[i])

    def _droplet_count(self) -> int:
        return int((((self._flags() >> N_PSTATE_SHIFT) & 3) == 1).sum().item())

    def rasterize_spray(self):
        """Droplet volume splatted into the float16 spray density field at
        spray_resolution_factor x the grid (pfflip/sim.py:394-401)."""
        if self.spray_density is None:
            self.spray_density = DeviceArray(torch.zeros(self.spray_res, dtype=torch.float16, device=self.dev))
        sx, sy, sz = self.spray_res
        N.call("pf_spray_rasterize", self.n_particles, N.sptr(self._pos4), N.sptr(self._drop_r),
               N.ptr(self.spray_density), sx, sy, sz, float(self.dx_spray), N.stream())
        return self.spray_density

    @property
    def dvel(self):
        """u - u* per axis (the reference's FLIP difference field)."""
        return [DeviceArray(as_tensor(a) - as_tensor(b)) for a, b in zip(self.vel, self.vel_star)]

    def state_counts(self):
        st = self.pstate.numpy()
        return {"flip": int((st == 0).sum()), "droplet": int((st == 1).sum()), "dead": int((st == 2).sum())}
