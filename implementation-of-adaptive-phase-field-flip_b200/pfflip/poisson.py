"""Variable-coefficient pressure Poisson solver on the GPU.

``MGPCG`` keeps the constructor, methods and attributes of the reference's
``pfflip.poisson.MGPCG`` (``pfflip/poisson.py:240-409``): unsmoothed aggregation
Galerkin multigrid with a red-black weighted Gauss-Seidel smoother (ω = 6/7)
preconditioning a flexible Polak-Ribière CG, the constant null space removed
from b, z and x, stopping on max|r| / max|b| < tol.  All work runs in
libpfflip.so (sm_100a); this class owns the device buffers and the plan.

``apply_A`` is a launchable stand-in for the reference kernel of that name
(``pfflip/poisson.py:78-88``): ``launch(apply_A, dim, inputs=[p, bx, by, bz,
diag, out])`` or ``apply_A(p, bx, by, bz, diag, out)``.

Additions: ``stencil`` selects the operator-row arithmetic: "reference" is the
reference's written form diag*p_i - Σβ p_nbr; "flux" (default) is Σβ (p_i - p_nbr),
equal in exact arithmetic but free of the cancellation that makes the
reference form stall at an inf-norm residual of 1e-6..1e-5 in binary32 on
1000:1 problems.  ``precision`` ("fp32" | "fp16" | "bf16") selects the storage
of the multigrid hierarchy, ``use_graphs`` replays each CG iteration as a CUDA
graph.
"""

from __future__ import annotations

import ctypes as C
import math
import warnings

import torch

from . import _native as N
from ._arrays import DeviceArray, as_tensor

_LP_DTYPE = {"fp16": torch.float16, "bf16": torch.bfloat16}


class _Level:
    """Per-level arrays (the reference's ``_Level``, pfflip/poisson.py:226-237)."""

    def __init__(self, res, device, precision):
        nx, ny, nz = res
        self.res = (nx, ny, nz)
        z = lambda shape: DeviceArray.zeros(shape, torch.float32, device)  # noqa: E731
        self.bx = z((nx + 1, ny, nz))
        self.by = z((nx, ny + 1, nz))
        self.bz = z((nx, ny, nz + 1))
        self.diag = z((nx, ny, nz))
        self.p = z((nx, ny, nz))
        self.b = z((nx, ny, nz))
        self.r = z((nx, ny, nz))
        self.p_alt = z((nx, ny, nz))
        # z-faces with rows padded to a multiple of 8 floats for TMA staging
        self.bz_pitch = (nz + 1 + 7) // 8 * 8
        self.bz_pad = z((nx, ny, self.bz_pitch)) if nz % 4 == 0 else None
        self.lp = None
        if precision in _LP_DTYPE:
            dt = _LP_DTYPE[precision]
            mk = lambda shape: DeviceArray.zeros(shape, dt, device)  # noqa: E731
            self.lp = {
                "bx": mk((nx + 1, ny, nz)), "by": mk((nx, ny + 1, nz)), "bz": mk((nx, ny, nz + 1)),
                "p": mk((nx, ny, nz)), "p_alt": mk((nx, ny, nz)), "b": mk((nx, ny, nz)),
            }

    def desc(self) -> N.pf_mg_level:
        d = N.pf_mg_level()
        d.nx, d.ny, d.nz = self.res
        d.bx, d.by, d.bz, d.diag = (N.ptr(a) for a in (self.bx, self.by, self.bz, self.diag))
        d.p, d.p_alt, d.b, d.r = (N.ptr(a) for a in (self.p, self.p_alt, self.b, self.r))
        if self.bz_pad is not None:
            d.bz_pad, d.bz_pitch = N.ptr(self.bz_pad), self.bz_pitch
        if self.lp:
            lp = self.lp
            d.bx_lp, d.by_lp, d.bz_lp = N.ptr(lp["bx"]), N.ptr(lp["by"]), N.ptr(lp["bz"])
            d.p_lp, d.p_lp_alt, d.b_lp = N.ptr(lp["p"]), N.ptr(lp["p_alt"]), N.ptr(lp["b"])
        return d


def level_dims(res, min_dim=4):
    """Level resolutions of the reference's rule (pfflip/poisson.py:256-263)."""
    out = []
    r = tuple(int(n) for n in res)
    while True:
        out.append(r)
        if min(r) // 2 < min_dim or any(n % 2 for n in r):
            break
        r = tuple(n // 2 for n in r)
    return out


def default_coef_scale(rho_l=1000.0, rho_g=1.0):
    """Power of two that centres beta = 1/rho in [1/rho_l, 1/rho_g] around 1."""
    return float(2.0 ** round(0.5 * math.log2(rho_l * rho_g)))


class MGPCG:
    """Multigrid-preconditioned flexible conjugate gradient (reference signature)."""

    def __init__(self, res, device="cuda:0", *, omega=6.0 / 7.0, pre=2, post=2, coarsest=60, min_dim=4,
                 precision="fp32", stencil="flux", coef_scale=None, use_graphs=True):
        self.device = N.require_cuda(device)
        if precision not in N.PF_PREC:
            raise ValueError(f"precision must be one of {sorted(N.PF_PREC)}")
        if stencil not in N.PF_STENCIL:
            raise ValueError(f"stencil must be one of {sorted(N.PF_STENCIL)}")
        self.stencil = stencil
        self.omega = omega
        self.pre = pre
        self.post = post
        self.coarsest = coarsest
        self.precision = precision
        self.use_graphs = bool(use_graphs)
        self.coef_scale = float(coef_scale) if coef_scale is not None else default_coef_scale()
        self.levels = [_Level(r, self.device, precision) for r in level_dims(res, min_dim)]
        self.nlev = len(self.levels)
        self.res = tuple(int(n) for n in res)
        self.ncells = self.res[0] * self.res[1] * self.res[2]
        z = lambda: DeviceArray.zeros(self.res, torch.float32, self.device)  # noqa: E731
        self.rhs, self.res_v, self.z, self.q, self.Ap, self.r_prev, self.x = z(), z(), z(), z(), z(), z(), z()
        self._state = torch.zeros(N.PF_MG_STATE_BYTES, dtype=torch.uint8, device=self.device)
        self._partials = torch.zeros(int(N.lib().pf_mg_partials_count()), dtype=torch.float64, device=self.device)
        self._counters = torch.zeros(N.PF_MG_COUNTERS, dtype=torch.int32, device=self.device)
        d = N.pf_mg_desc()
        d.nlev = self.nlev
        for i, L in enumerate(self.levels):
            d.lev[i] = L.desc()
        d.omega, d.pre, d.post, d.coarsest = float(omega), int(pre), int(post), int(coarsest)
        d.precision = N.PF_PREC[precision]
        d.stencil = N.PF_STENCIL[stencil]
        d.coef_scale = self.coef_scale
        d.rhs, d.res_v, d.res_alt, d.z = N.ptr(self.rhs), N.ptr(self.res_v), N.ptr(self.r_prev), N.ptr(self.z)
        d.q, d.Ap, d.x = N.ptr(self.q), N.ptr(self.Ap), N.ptr(self.x)
        d.state, d.partials, d.counters = self._state.data_ptr(), self._partials.data_ptr(), self._counters.data_ptr()
        nop = int(N.lib().pf_mg_bottom_op_floats(C.byref(d)))  # dense operator of the smallest levels (or 0)
        self._bottom_op = torch.zeros(max(nop, 1), dtype=torch.float32, device=self.device)
        d.bottom_op = self._bottom_op.data_ptr() if nop > 0 else None
        self._desc = d
        h = C.c_void_p()
        N.check(N.lib().pf_mg_plan_create(C.byref(d), C.byref(h)), "pf_mg_plan_create")
        self._plan = h
        self.last_status = N.PF_OK

    def __del__(self):
        try:
            if getattr(self, "_plan", None) and self._plan.value:
                torch.cuda.synchronize(self.device)
                N.lib().pf_mg_plan_destroy(self._plan)
                self._plan = C.c_void_p()
        except Exception:
            pass

    # ------------------------------------------------------------ hierarchy
    def build_hierarchy(self, bx, by, bz):
        """Level-0 faces = (bx, by, bz); diag and Galerkin-coarsened faces below."""
        N.call("pf_mg_build_hierarchy", self._plan, N.ptr(as_tensor(bx)), N.ptr(as_tensor(by)),
               N.ptr(as_tensor(bz)), N.stream())

    def _smooth(self, L, nsweeps, reverse=False):
        lv = self.levels.index(L) if isinstance(L, _Level) else int(L)
        N.call("pf_mg_smooth", self._plan, lv, int(nsweeps), int(bool(reverse)), N.stream())

    def precondition(self, r_in, z_out):
        """``z = M^-1 r``: one V-cycle, mean removed (pfflip/poisson.py:345-352)."""
        N.call("pf_mg_precondition", self._plan, N.ptr(as_tensor(r_in)), N.ptr(as_tensor(z_out)), N.stream())

    def bottom_info(self):
        """``(first_level, cluster_levels, dense)`` of the kernel that runs the
        coarse end of the V-cycle: cluster_levels > 0 for the CTA-cluster
        kernel, 0 for the single-CTA one; dense = 1 when the levels below the
        cluster's slabs run as a dense operator (diagnostics; no reference
        counterpart)."""
        first, nd, dense = C.c_int32(0), C.c_int32(0), C.c_int32(0)
        N.call("pf_mg_bottom_info", self._plan, C.byref(first), C.byref(nd), C.byref(dense))
        return int(first.value), int(nd.value), int(dense.value)

    # ------------------------------------------------------------ solve
    def solve(self, b, p_out, *, tol=1e-4, max_iter=200, verbose=False):
        """Flexible PCG with Polak-Ribière beta; returns ``(iterations, relative_residual)``.

        As in the reference a missed tolerance is not an error; a non-finite
        residual stops the iteration early and warns."""
        it = C.c_int32(0)
        rel = C.c_double(0.0)
        rc = N.lib().pf_mg_solve(self._plan, N.ptr(as_tensor(b)), N.ptr(as_tensor(p_out)), float(tol),
                                 int(max_iter), int(self.use_graphs), int(bool(verbose)), C.byref(it),
                                 C.byref(rel), N.stream())
        N.check(rc, "pf_mg_solve", ok=(N.PF_OK, N.PF_ERR_NOT_CONVERGED, N.PF_ERR_NONFINITE))
        self.last_status = rc
        if rc == N.PF_ERR_NONFINITE:
            warnings.warn(f"MG-PCG: {N.last_error()}", RuntimeWarning, stacklevel=2)
        return int(it.value), float(rel.value)


def apply_A(p, bx, by, bz, diag, out, stencil="reference"):
    """``out = A p`` (pfflip/poisson.py:54-88); the default row form is the
    reference's ``diag*p - Σβ p_nbr`` with the given diag."""
    t = as_tensor(p)
    nx, ny, nz = t.shape
    g = N.grid((nx, ny, nz), 1.0)
    N.call("pf_apply_A", C.byref(g), N.ptr(t), N.ptr(as_tensor(bx)), N.ptr(as_tensor(by)), N.ptr(as_tensor(bz)),
           N.ptr(as_tensor(diag)) if diag is not None else None, N.ptr(as_tensor(out)), N.PF_STENCIL[stencil],
           N.stream())
    return out
