"""ctypes front end of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` import
this module, always as the checker (or the timed CPU baseline), never as part of
the product path.  It restates the reference's uniform-grid step:

* ``OracleMGPCG`` follows ``pfflip/poisson.py:240-409`` (``MGPCG``).
* ``OracleSim`` follows ``pfflip/sim.py:37-424`` (``Simulator``) stage by stage,
  with the same stage method names so a test can feed it the GPU state at the
  input of any one stage.

The arithmetic lives in ``pf_oracle.hpp`` (binary32 or binary64).  Parity is
pinned against the reference's own test vectors: see ``tests/golden/``.
"""

from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libpforacle.so")
_lib = None

f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        I64, I, D, VP = C.c_int64, C.c_int, C.c_double, C.c_void_p
        L.pfo_set_threads.argtypes = [I]
        L.pfo_get_threads.restype = I
        L.pfo_set_stencil.argtypes = [I]
        L.pfo_sort_by_cell.argtypes = [I64, f32p, C.c_float, I, I, I, i32p, i32p, i32p]
        for sfx, fp, R in (("f32", f32p, C.c_float), ("f64", f64p, C.c_double)):
            g = lambda n: getattr(L, f"pfo_{n}_{sfx}")  # noqa: E731
            g("p2g").argtypes = [I64, fp, fp, fp, fp, i32p, I, I, I, R] + [fp] * 8 + [I]
            g("face_velocity").argtypes = [fp, fp, fp, i32p, I64, R]
            g("cell_phase").argtypes = [fp, fp, i32p, I64, R, R, R]
            g("face_beta").argtypes = [fp, i32p, fp, fp, I, I, I, I, R, R, R, R, R]
            g("zero_solid_faces").argtypes = [fp, fp, I, I, I, I]
            g("zero_solid_obstacle_faces").argtypes = [i32p, fp, fp, I, I, I, I]
            g("add_gravity").argtypes = [fp, I64, R, R]
            g("build_rhs").argtypes = [fp, fp, fp, fp, fp, I, I, I, R, R, R, R]
            g("apply_pressure_gradient").argtypes = [fp, fp, fp, I, I, I, I, R, R]
            g("divergence_norm").argtypes = [fp, fp, fp, I, I, I, R]
            g("divergence_norm").restype = R
            g("seed_liquid_velocity").argtypes = [fp, i32p, fp, i32p, I, I, I, I]
            g("extrapolate_sweep").argtypes = [fp, i32p, fp, i32p, I, I, I]
            g("g2p").argtypes = [I64, fp, fp, i32p, i32p] + [fp] * 6 + [I, I, I, R, R, R]
            g("advect_reflect").argtypes = [I64, fp, fp, i32p, i32p] + [fp] * 6 + [I, I, I, R, R, fp, fp]
            g("push_out_of_solids").argtypes = [I64, fp, fp, i32p, i32p, I, I, I, R]
            U32 = C.c_uint32
            g("droplet_classify").argtypes = [I64, fp, i32p, i32p, fp, fp, I, I, I, R, R, R, R, R, R, U32, i32p]
            g("velocity_gradient").argtypes = [fp, fp, fp, fp, I, I, I, R]
            g("spray_emit").argtypes = [I64, fp, i32p, i32p, fp, fp, fp, I, I, I, R, R, R, R, R, R, R, U32, i32p]
            g("droplet_advance").argtypes = [I64, fp, fp, i32p, fp, fp, fp, fp, I, I, I, R, R, fp, R, R, R, R, R,
                                             fp, fp, I]
            g("spray_rasterize").argtypes = [I64, fp, i32p, fp, fp, I, I, I, R]
            g("particle_max_speed").argtypes = [I64, fp, i32p]
            g("particle_max_speed").restype = R
            g("apply_A").argtypes = [fp] * 6 + [I, I, I]
            g("mg_create").argtypes = [I, I, I, R, I, I, I, I]
            g("mg_create").restype = VP
            g("mg_destroy").argtypes = [VP]
            g("mg_nlev").argtypes = [VP]
            g("mg_nlev").restype = I
            g("mg_level_dims").argtypes = [VP, I, i32p]
            g("mg_level_io").argtypes = [VP, I, I, fp, I]
            g("mg_build").argtypes = [VP, fp, fp, fp]
            g("mg_precondition").argtypes = [VP, fp, fp]
            g("mg_smooth").argtypes = [VP, I, I, I]
            g("mg_solve").argtypes = [VP, fp, fp, D, I, C.POINTER(D), f64p, I]
            g("mg_solve").restype = I
        _lib = L
    return _lib


STENCIL = {"reference": 0, "flux": 1}


def set_stencil(form: str):
    """Operator row form used by every following oracle call ("reference" or "flux")."""
    lib().pfo_set_stencil(STENCIL[form])


def set_threads(n: int):
    lib().pfo_set_threads(int(n))


def get_threads() -> int:
    return int(lib().pfo_get_threads())


def _sfx(dtype):
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


def _fn(name, dtype):
    return getattr(lib(), f"pfo_{name}_{_sfx(dtype)}")


def face_shapes(res):
    nx, ny, nz = res
    return ((nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1))


# ----------------------------------------------------------------- sorting
def sort_by_cell(pos: np.ndarray, dx: float, res):
    """Stable counting sort by cell key; returns (keys, perm, cell_start)."""
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    n = len(pos)
    nx, ny, nz = res
    keys = np.empty(n, np.int32)
    perm = np.empty(n, np.int32)
    start = np.empty(nx * ny * nz + 1, np.int32)
    lib().pfo_sort_by_cell(n, pos, np.float32(dx), nx, ny, nz, keys, perm, start)
    return keys, perm, start


def cell_keys_numpy(pos: np.ndarray, dx: float, res):
    """Same keys in plain numpy (binary32 division, floor, clamp)."""
    pos = np.asarray(pos, np.float32).reshape(-1, 3)
    q = np.floor(pos / np.float32(dx)).astype(np.int64)
    for a in range(3):
        q[:, a] = np.clip(q[:, a], 0, res[a] - 1)
    return ((q[:, 0] * res[1] + q[:, 1]) * res[2] + q[:, 2]).astype(np.int32)


# ----------------------------------------------------------------- solver
def apply_A(p, bx, by, bz, diag, dtype=np.float32, stencil="reference"):
    set_stencil(stencil)
    dt = np.dtype(dtype)
    res = p.shape
    out = np.empty(res, dt)
    arrs = [np.ascontiguousarray(a, dt) for a in (p, bx, by, bz, diag)]
    _fn("apply_A", dt)(*arrs, out, *res)
    return out


def compute_diag(bx, by, bz):
    return bx[:-1] + bx[1:] + by[:, :-1] + by[:, 1:] + bz[:, :, :-1] + bz[:, :, 1:]


class OracleMGPCG:
    """``pfflip/poisson.py:240-409`` in binary32 (default) or binary64."""

    def __init__(self, res, *, omega=6.0 / 7.0, pre=2, post=2, coarsest=60, min_dim=4, dtype=np.float32,
                 stencil="reference"):
        self.dtype = np.dtype(dtype)
        self.stencil = stencil
        self.res = tuple(int(r) for r in res)
        self._h = _fn("mg_create", self.dtype)(*self.res, omega, pre, post, coarsest, min_dim)
        self.nlev = int(_fn("mg_nlev", self.dtype)(self._h))

    def __del__(self):
        try:
            if self._h:
                _fn("mg_destroy", self.dtype)(self._h)
        except Exception:
            pass

    def level_res(self, lv):
        d = np.empty(3, np.int32)
        _fn("mg_level_dims", self.dtype)(self._h, lv, d)
        return tuple(int(x) for x in d)

    def level_array(self, lv, which):
        names = ["bx", "by", "bz", "diag", "p", "b", "r"]
        w = names.index(which)
        r = self.level_res(lv)
        shape = face_shapes(r)[w] if w < 3 else r
        out = np.empty(shape, self.dtype)
        _fn("mg_level_io", self.dtype)(self._h, lv, w, out, 0)
        return out

    def set_level_array(self, lv, which, arr):
        names = ["bx", "by", "bz", "diag", "p", "b", "r"]
        a = np.ascontiguousarray(arr, self.dtype)
        _fn("mg_level_io", self.dtype)(self._h, lv, names.index(which), a, 1)

    def build_hierarchy(self, bx, by, bz):
        c = lambda a: np.ascontiguousarray(a, self.dtype)  # noqa: E731
        _fn("mg_build", self.dtype)(self._h, c(bx), c(by), c(bz))

    def precondition(self, r):
        set_stencil(self.stencil)
        z = np.empty(self.res, self.dtype)
        _fn("mg_precondition", self.dtype)(self._h, np.ascontiguousarray(r, self.dtype), z)
        return z

    def smooth(self, lv, nsweeps, reverse=False):
        set_stencil(self.stencil)
        _fn("mg_smooth", self.dtype)(self._h, lv, nsweeps, int(reverse))

    def solve(self, b, *, tol=1e-4, max_iter=200, return_history=False):
        set_stencil(self.stencil)
        x = np.empty(self.res, self.dtype)
        rel = C.c_double(0.0)
        hist = np.zeros(max(max_iter, 1), np.float64)
        it = _fn("mg_solve", self.dtype)(
            self._h, np.ascontiguousarray(b, self.dtype), x, float(tol), int(max_iter), C.byref(rel), hist, len(hist)
        )
        if return_history:
            return x, int(it), float(rel.value), hist[: max(int(it), 0)].copy()
        return x, int(it), float(rel.value)


def fp64_reference_solve(bx, by, bz, b, *, tol=1e-12, max_iter=400, pre=3, post=3, coarsest=60, min_dim=4):
    """The binary64 oracle: the same MG-preconditioned flexible CG, run in double
    (flux-form rows) to a 1e-12 relative inf-norm residual.  Returns the
    zero-mean solution."""
    res = b.shape
    s = OracleMGPCG(res, pre=pre, post=post, coarsest=coarsest, min_dim=min_dim, dtype=np.float64,
                    stencil="flux")
    s.build_hierarchy(bx, by, bz)
    x, it, rel = s.solve(np.asarray(b, np.float64), tol=tol, max_iter=max_iter)
    return x, it, rel


# ----------------------------------------------------------------- simulator
def rho_tilde_0(dx: float, r: float, ppc: int) -> float:
    """Kernel weight sum of a perfect lattice, following ``pfflip/sim.py:119-140``."""
    per_axis = round(ppc ** (1.0 / 3.0))
    step = dx / per_axis
    R = int(math.ceil(r / step)) + 1
    acc = 0.0
    for a in range(-R, R + 1):
        for b in range(-R, R + 1):
            for c in range(-R, R + 1):
                d2 = ((a + 0.5) ** 2 + (b + 0.5) ** 2 + (c + 0.5) ** 2) * step * step
                t = max(1.0 - d2 / (r * r), 0.0)
                acc += t * t * t
    return acc


class OracleSim:
    """``pfflip/sim.py:37-424`` on the CPU oracle.  Fields are numpy arrays with the
    reference's shapes; particle arrays are AoS (n,3).  The droplet stage is not
    part of the restated path and is never run."""

    def __init__(self, cfg, dtype=np.float32, nthreads=1, stencil=None):
        self.cfg = cfg
        self.R = np.dtype(dtype)
        R = self.R
        self.res = tuple(cfg.res)
        self.nthreads = int(nthreads)
        self.face_shapes = face_shapes(self.res)
        z = lambda s: np.zeros(s, R)  # noqa: E731
        zi = lambda s: np.zeros(s, np.int32)  # noqa: E731
        fs = self.face_shapes
        self.vel = [z(s) for s in fs]
        self.vel_star = [z(s) for s in fs]
        self.vel_liq = [z(s) for s in fs]
        self.dvel = [z(s) for s in fs]
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
        self.solver = OracleMGPCG(
            self.res, omega=cfg.mg_omega, pre=cfg.mg_pre_sweeps, post=cfg.mg_post_sweeps,
            coarsest=cfg.mg_coarsest_sweeps, min_dim=cfg.mg_min_dim, dtype=R,
            stencil=stencil or getattr(cfg, "stencil", "reference"),
        )
        self.rho_tilde_0 = rho_tilde_0(cfg.dx, cfg.r_p, cfg.ppc)
        self.rho_0l = self.rho_tilde_0 * cfg.rho_l
        self.rho_min = cfg.eta_phi * cfg.rho_g * self.rho_tilde_0
        self.has_solids = False
        self.time = 0.0
        self.step_index = 0
        self.stats = []
        self.n_particles = 0
        self.droplet_stats = {"emitted": 0, "bubbles": 0, "merged": 0, "spray": 0}
        f = max(1, int(cfg.spray_resolution_factor))
        self.spray_res = tuple(n * f for n in self.res)
        self.dx_spray = cfg.dx / f

    def _c(self, x):
        return self.R.type(x)

    def set_solids(self, mask):
        self.solid = np.ascontiguousarray(mask, np.int32)
        self.has_solids = bool(np.any(mask))

    def set_particles(self, pos, vel, ptype, pstate=None):
        cfg, R = self.cfg, self.R
        n = len(pos)
        self.n_particles = n
        self.px = np.ascontiguousarray(pos, R).reshape(n, 3).copy()
        self.pv = np.ascontiguousarray(vel, R).reshape(n, 3).copy()
        self.ptype = np.ascontiguousarray(ptype, np.int32).copy()
        self.pmass = np.where(self.ptype == 1, cfg.rho_l, cfg.rho_g).astype(R)
        self.prad = np.full(n, cfg.r_p, R)
        self.pstate = np.zeros(n, np.int32) if pstate is None else np.ascontiguousarray(pstate, np.int32).copy()
        self.pdrop_r = np.zeros(n, R)

    # ----------------------------------------------------------- stages
    def _p2g(self):
        cfg = self.cfg
        nx, ny, nz = self.res
        _fn("p2g", self.R)(
            self.n_particles, self.px, self.pv, self.pmass, self.prad, self.pstate, nx, ny, nz, self._c(cfg.dx),
            *self.mass, *self.mom, self.cell_mass, self.cell_wsum, self.nthreads,
        )
        eps = self._c(1e-12 * self.rho_0l)
        for ax in range(3):
            _fn("face_velocity", self.R)(self.mass[ax], self.mom[ax], self.vel[ax], self.valid[ax],
                                         self.mass[ax].size, eps)

    def _phase_field_and_coefficients(self):
        cfg, c = self.cfg, self._c
        nx, ny, nz = self.res
        _fn("cell_phase", self.R)(self.cell_mass, self.phi_cell, self.is_liquid, self.cell_mass.size,
                                  c(self.rho_min), c(cfg.alpha_phi), c(self.rho_0l))
        for ax in range(3):
            _fn("face_beta", self.R)(self.mass[ax], self.is_liquid, self.phi_face[ax], self.beta[ax], nx, ny, nz,
                                     ax, c(self.rho_min), c(cfg.alpha_phi), c(self.rho_0l), c(cfg.rho_l),
                                     c(cfg.rho_g))
            _fn("zero_solid_faces", self.R)(self.beta[ax], self.vel[ax], nx, ny, nz, ax)
            if self.has_solids:
                _fn("zero_solid_obstacle_faces", self.R)(self.solid, self.beta[ax], self.vel[ax], nx, ny, nz, ax)

    def _save_vel_star(self):
        for ax in range(3):
            self.vel_star[ax][...] = self.vel[ax]

    def _add_forces(self, dt):
        nx, ny, nz = self.res
        for ax in range(3):
            g = self.cfg.gravity[ax]
            if g != 0.0:
                _fn("add_gravity", self.R)(self.vel[ax], self.vel[ax].size, self._c(g), self._c(dt))
            _fn("zero_solid_faces", self.R)(self.beta[ax], self.vel[ax], nx, ny, nz, ax)
            if self.has_solids:
                _fn("zero_solid_obstacle_faces", self.R)(self.solid, self.beta[ax], self.vel[ax], nx, ny, nz, ax)

    def _build_rhs(self, dt):
        cfg, c = self.cfg, self._c
        _fn("build_rhs", self.R)(*self.vel, self.cell_wsum, self.rhs, *self.res, c(cfg.dx), c(dt),
                                 c(self.rho_tilde_0), c(cfg.k_div))
        return self.rhs

    def _pressure_solve(self, dt, tol=None):
        cfg = self.cfg
        self._build_rhs(dt)
        self.solver.build_hierarchy(*self.beta)
        x, it, rel = self.solver.solve(self.rhs, tol=cfg.pcg_tol if tol is None else tol,
                                       max_iter=cfg.pcg_max_iter)
        self.pressure[...] = x
        return it, rel

    def _project(self, dt):
        c = self._c
        for ax in range(3):
            _fn("apply_pressure_gradient", self.R)(self.pressure, self.beta[ax], self.vel[ax], *self.res, ax,
                                                   c(self.cfg.dx), c(dt))

    def _max_divergence(self):
        return float(_fn("divergence_norm", self.R)(*self.vel, *self.res, self._c(self.cfg.dx)))

    def _g2p(self):
        cfg, c = self.cfg, self._c
        for ax in range(3):
            self.dvel[ax] = (self.vel[ax] - self.vel_star[ax]).astype(self.R)
        _fn("g2p", self.R)(self.n_particles, self.px, self.pv, self.ptype, self.pstate, *self.vel, *self.dvel,
                           *self.res, c(cfg.dx), c(cfg.alpha_flip_liquid), c(cfg.alpha_flip_air))

    def _extrapolate_liquid_velocity(self):
        for ax in range(3):
            _fn("seed_liquid_velocity", self.R)(self.vel[ax], self.is_liquid, self.vel_liq[ax], self._known[ax],
                                                *self.res, ax)
        for _ in range(self.cfg.extrap_cells):
            for ax in range(3):
                out = np.empty_like(self.vel_liq[ax])
                kout = np.empty_like(self._known[ax])
                _fn("extrapolate_sweep", self.R)(self.vel_liq[ax], self._known[ax], out, kout,
                                                 *self.vel_liq[ax].shape)
                self.vel_liq[ax], self._known[ax] = out, kout

    def _advect(self, dt):
        cfg = self.cfg
        eps = 1e-4 * cfg.dx
        lo = np.full(3, eps, self.R)
        hi = np.array([s - eps for s in cfg.domain_size], self.R)
        _fn("advect_reflect", self.R)(self.n_particles, self.px, self.pv, self.ptype, self.pstate, *self.vel,
                                      *self.vel_liq, *self.res, self._c(dt), self._c(cfg.dx), lo, hi)
        if self.has_solids:
            _fn("push_out_of_solids", self.R)(self.n_particles, self.px, self.pv, self.pstate, self.solid,
                                              *self.res, self._c(cfg.dx))

    def _droplets(self, dt):
        """``pfflip/sim.py:343-392``: classification, optional shear spray, droplet dynamics."""
        cfg, c, R = self.cfg, self._c, self.R
        if not cfg.droplets or self.n_particles == 0:
            return
        sigma = float(cfg.droplet_radius_spread)
        mu = float(np.log(cfg.droplet_radius_mean * cfg.dx) - 0.5 * sigma * sigma)
        r_min, r_max = 0.02 * cfg.dx, 2.0 * cfg.dx
        seed = (int(cfg.seed) + int(self.step_index)) & 0xFFFFFFFF
        counters = np.zeros(4, np.int32)
        nx, ny, nz = self.res
        _fn("droplet_classify", R)(self.n_particles, self.px, self.ptype, self.pstate, self.pdrop_r, self.phi_cell,
                                   nx, ny, nz, c(cfg.dx), c(cfg.delta_phi), c(mu), c(sigma), c(r_min), c(r_max),
                                   seed, counters)
        if cfg.spray_shear_threshold > 0.0:
            self.shear = np.zeros(self.res, R)
            _fn("velocity_gradient", R)(*self.vel, self.shear, nx, ny, nz, c(cfg.dx))
            _fn("spray_emit", R)(self.n_particles, self.px, self.ptype, self.pstate, self.pdrop_r, self.phi_cell,
                                 self.shear, nx, ny, nz, c(cfg.dx), c(cfg.spray_shear_threshold),
                                 c(cfg.spray_emission_rate), c(mu), c(sigma), c(r_min), c(r_max), seed, counters)
        eps = 1e-4 * cfg.dx
        lo = np.full(3, eps, R)
        hi = np.array([s - eps for s in cfg.domain_size], R)
        _fn("droplet_advance", R)(self.n_particles, self.px, self.pv, self.pstate, self.pdrop_r, *self.vel, nx, ny,
                                  nz, c(dt), c(cfg.dx), np.asarray(cfg.gravity, R), c(cfg.rho_g), c(cfg.rho_l),
                                  c(cfg.droplet_drag_cd), c(cfg.evaporation_k * cfg.dx * cfg.dx), c(r_min), lo, hi,
                                  int(cfg.droplet_max_substeps))
        for k, i in (("emitted", 0), ("bubbles", 1), ("merged", 2), ("spray", 3)):
            self.droplet_stats[k] += int(counters[i])

    def rasterize_spray(self):
        """``pfflip/sim.py:394-401`` (accumulated in the oracle's precision)."""
        out = np.zeros(self.spray_res, self.R)
        _fn("spray_rasterize", self.R)(self.n_particles, self.px, self.pstate, self.pdrop_r, out, *self.spray_res,
                                       self._c(self.dx_spray))
        return out

    def dt_from_cfl(self):
        cfg = self.cfg
        vmax = float(_fn("particle_max_speed", self.R)(self.n_particles, self.pv, self.pstate))
        g = float(np.linalg.norm(cfg.gravity))
        vmax = max(vmax, math.sqrt(2.0 * g * cfg.dx) if g > 0 else 0.0, 1e-8)
        return float(np.clip(cfg.cfl * cfg.dx / vmax, cfg.dt_min, cfg.dt_max))

    def step(self, dt=None):
        if dt is None:
            dt = self.dt_from_cfl()
        self._p2g()
        self._phase_field_and_coefficients()
        self._save_vel_star()
        self._add_forces(dt)
        it, rel = self._pressure_solve(dt)
        self._project(dt)
        div = self._max_divergence()
        self._g2p()
        self._extrapolate_liquid_velocity()
        self._droplets(dt)
        self._advect(dt)
        self.time += dt
        self.step_index += 1
        rec = {"step": self.step_index, "t": self.time, "dt": dt, "pcg_iter": it, "pcg_res": rel,
               "max_div": div, "droplets": int((self.pstate == 1).sum()) if self.cfg.droplets else 0}
        self.stats.append(rec)
        return rec


def rt_interface_variance(cfg, pos, ptype, dt, steps, nthreads=1):
    """The Rayleigh-Taylor gradient's loss on the binary64 oracle (solve to
    1e-12): run ``steps`` steps from rest at ``pos``, then the variance over
    the (x, z) columns of the light-phase height h = dx sum_y (1 - phi)."""
    import dataclasses

    c64 = dataclasses.replace(cfg, pcg_tol=1e-12, pcg_max_iter=1000)
    sim = OracleSim(c64, dtype=np.float64, nthreads=nthreads, stencil="flux")
    sim.set_particles(np.asarray(pos, np.float64), np.zeros((len(pos), 3)), ptype)
    for _ in range(steps):
        sim.step(dt)
    sim._p2g()
    sim._phase_field_and_coefficients()
    h = (1.0 - sim.phi_cell).sum(axis=1) * cfg.dx
    return float(((h - h.mean()) ** 2).mean())


def stable_central_difference(loss, eps_list=(1e-6, 3e-7, 1e-7, 3e-8, 1e-8), rtol=2e-4):
    """Central difference (loss(+e) - loss(-e)) / 2e of a scalar function of one
    step size e, taken away from the function's jumps and kinks: the first two
    consecutive step sizes of ``eps_list`` whose differences agree to ``rtol``
    give the value (the smaller step's).  Returns (value, eps, all differences)
    or (None, None, all differences) when no two agree, i.e. a jump of the
    loss lies within the largest step of the point."""
    fds = []
    for e in eps_list:
        fds.append((loss(e) - loss(-e)) / (2.0 * e))
        if len(fds) >= 2 and abs(fds[-1] - fds[-2]) <= rtol * max(abs(fds[-1]), 1e-300):
            return fds[-1], e, fds
    return None, None, fds
