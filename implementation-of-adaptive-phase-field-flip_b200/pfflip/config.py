"""Simulation parameters of the uniform-grid PF-FLIP step.

Field names, meanings and default values are those of the reference's
``Config`` dataclass (``pfflip/config.py:15-135``), so reference scripts and
tests construct it unchanged.  Three fields are added at the end; their
defaults give the reference's plain-FP32 behaviour.
"""

from __future__ import annotations

import math
from dataclasses import dataclass


@dataclass
class Config:
    # grid: cell counts, spacing, particles per cell at seeding (a perfect cube)
    res: tuple[int, int, int] = (64, 64, 64)
    dx: float = 1.0
    ppc: int = 8

    # physics: liquid density, rho_l / rho_g, body force
    rho_l: float = 1000.0
    density_ratio: float = 1000.0
    gravity: tuple[float, float, float] = (0.0, -9.81, 0.0)

    # eq. (7) stiffness knob
    alpha_phi: float = 1.0

    # eq. (12) FLIP/PIC blend per phase
    alpha_flip_liquid: float = 0.985
    alpha_flip_air: float = 0.96

    # time stepping
    cfl: float = 1.0
    dt_max: float = 1.0 / 24.0
    dt_min: float = 1e-6

    # c_div volume correction strength (0 disables it)
    k_div: float = 0.0

    # pressure solve: inf-norm relative tolerance, iteration cap, V-cycle shape
    pcg_tol: float = 1e-4
    pcg_max_iter: int = 200
    mg_pre_sweeps: int = 3
    mg_post_sweeps: int = 3
    mg_coarsest_sweeps: int = 60
    mg_omega: float = 6.0 / 7.0
    mg_min_dim: int = 4

    # liquid velocity extrapolation depth in cells
    extrap_cells: int = 3

    # escaped-particle / droplet / spray parameters (pfflip/config.py, paper 3.4, 7)
    droplets: bool = True
    delta_phi: float = 0.2
    droplet_radius_mean: float = 0.25
    droplet_radius_spread: float = 0.5
    droplet_drag_cd: float = 0.5
    evaporation_k: float = 0.0
    spray_shear_threshold: float = 0.0
    spray_emission_rate: float = 0.02
    spray_resolution_factor: int = 2
    droplet_max_substeps: int = 8

    # runtime
    device: str = "cuda:0"
    seed: int = 42

    # ---- additions of this implementation -------------------------------
    precision: str = "fp32"
    """Multigrid hierarchy storage: "fp32" (the reference's arithmetic), "fp16"
    or "bf16" (16-bit storage of smoother/transfer fields, FP32 arithmetic, FP32
    outer CG with FP64 reductions, FP64 coarsest solve)."""

    stencil: str = "flux"
    """Operator-row arithmetic of the pressure solve: "flux" = Σβ(p_i - p_nbr)
    (reaches a 1e-7 inf-norm residual in FP32) or "reference" = diag*p_i - Σβ p_nbr,
    the reference's written form (stalls near 1e-6..1e-5 at 1000:1)."""

    cuda_graphs: bool = True
    """Replay each flexible-CG iteration as one captured CUDA graph."""

    # ------------------------------------------------------------- derived
    @property
    def rho_g(self) -> float:
        return self.rho_l / self.density_ratio

    @property
    def r_p(self) -> float:
        return self.dx

    @property
    def eta_phi(self) -> float:
        return math.log(self.density_ratio)

    @property
    def domain_size(self) -> tuple[float, float, float]:
        return (self.res[0] * self.dx, self.res[1] * self.dx, self.res[2] * self.dx)
