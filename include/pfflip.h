/*
 * pfflip.h — C ABI of the B200 (sm_100a) uniform-grid PF-FLIP step.
 *
 * One shared library, libpfflip.so, exports every entry point below.  All
 * arguments are plain pointers and sizes; no framework types cross the ABI.
 *
 * Ownership.  The caller owns every buffer (device memory for fields and
 * particles, host memory only where stated).  The library never allocates
 * device memory: scratch space comes in through caller-sized workspaces whose
 * sizes the *_workspace_bytes / *_count queries return.  Pointers are borrowed
 * for the duration of the call (a pf_mg_plan borrows them until it is
 * destroyed).
 *
 * Streams.  `stream` is a cudaStream_t passed as void* (NULL = legacy default
 * stream).  Every call only enqueues work on that stream and returns, except
 * where a host result is documented (pf_mg_solve, pf_read_*), which synchronise
 * that stream.
 *
 * Errors.  Every call returns PF_OK (0) or a PF_ERR_* code; pf_last_error()
 * returns a message for the calling thread's last failure and
 * pf_last_cuda_error() the CUDA error code behind a PF_ERR_CUDA.
 *
 * Layouts (those of the reference, pfflip/kernels.py:1-12):
 *   cell arrays       (nx, ny, nz)      C order, index (i*ny + j)*nz + k
 *   face arrays, x    (nx+1, ny, nz)    the face with index i sits at x = i*dx
 *   face arrays, y    (nx, ny+1, nz)
 *   face arrays, z    (nx, ny, nz+1)
 *   particles         two float4 streams, 16-byte aligned, sorted by cell:
 *       pos4[p] = (x, y, z, flags)   flags: int32 bits, bit 0 = liquid
 *                                    (ptype == 1), bits 1-2 = pstate
 *       vel4[p] = (u, v, w, id)      id: int32 bits, the particle's index in
 *                                    the caller's original order
 */
#ifndef PFFLIP_H
#define PFFLIP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PF_OK 0
#define PF_ERR_ARG 1           /* invalid argument (null pointer, bad size, misalignment) */
#define PF_ERR_CUDA 2          /* a CUDA runtime call failed; see pf_last_cuda_error() */
#define PF_ERR_NONFINITE 3     /* a NaN/Inf appeared in the CG residual */
#define PF_ERR_NOT_CONVERGED 4 /* tolerance not met within max_iter (results still valid) */
#define PF_ERR_WORKSPACE 5     /* workspace too small */
#define PF_ERR_UNSUPPORTED 6   /* option not supported by this library */

#define PF_FLAG_LIQUID 1u
#define PF_PSTATE_SHIFT 1

#define PF_MG_MAX_LEVELS 16

/* operator row form: the reference's written form diag*p_i - sum beta*p_nbr
 * (pfflip/poisson.py:69-75), or the flux form sum beta*(p_i - p_nbr), equal in
 * exact arithmetic but free of the cancellation that stalls the reference form
 * at an inf-norm residual near 1e-6..1e-5 in binary32 */
#define PF_STENCIL_REFERENCE 0
#define PF_STENCIL_FLUX 1

#define PF_PREC_FP32 0
#define PF_PREC_FP16 1
#define PF_PREC_BF16 2

typedef struct pf_grid {
  int32_t nx, ny, nz;
  float dx;
} pf_grid;

/* ------------------------------------------------------------------ misc */
const char* pf_version(void);
const char* pf_last_error(void);
int pf_last_cuda_error(void);
/* number of kernel launches this library has issued from this process (all
 * threads, captured graph replays counted once per launched node) */
uint64_t pf_launch_count(void);

/* ------------------------------------------------------------- particles */
/* Counting sort by cell key.  No reference counterpart: the reference never
 * reorders particles (pfflip/scenes.py:23-29 order is kept; pfflip/droplets.py:22-24).
 * key(p) = (i*ny + j)*nz + k with i = clamp(floor(x/dx), 0, nx-1) computed in
 * binary32 with IEEE division (likewise j, k); the sort is stable, so perm and
 * keys equal a stable CPU argsort of the same keys.
 *   in : pos4_in, vel4_in (n particles, any order)
 *   out: pos4_out, vel4_out (sorted), keys_out[n] (sorted keys), perm_out[n]
 *        (perm_out[t] = input slot of the t-th sorted particle), cell_start
 *        [nx*ny*nz + 1] (particles of cell c are [cell_start[c], cell_start[c+1]))
 *   every output and the workspace must be disjoint from every other buffer
 *   of the call (PF_ERR_ARG on any overlap); the workspace
 *   (pf_sort_workspace_bytes) is 16-byte aligned. */
size_t pf_sort_workspace_bytes(const pf_grid* g, int64_t n);
int pf_sort_particles(const pf_grid* g, int64_t n, const float* pos4_in, const float* vel4_in, float* pos4_out,
                      float* vel4_out, int32_t* keys_out, int32_t* perm_out, int32_t* cell_start, void* workspace,
                      size_t workspace_bytes, void* stream);

/* The same sort without a caller workspace; no counterpart in the reference.
 * For hosts that cannot hand over device scratch (all device memory fixed at
 * start-up, or a step that must not allocate).  Arguments, outputs and
 * results are those of pf_sort_particles.  The call allocates nothing:
 * per-particle scratch lives in pos4_out for the whole call (until the final
 * gather writes the sorted positions there), and the scan's tile sums sit in
 * a static device array of the library (131,328 bytes), which limits the grid
 * to PF_SORT_STATIC_MAX_CELLS cells; larger grids return PF_ERR_ARG.  Every
 * output must be disjoint from every other buffer of the call (checked:
 * PF_ERR_ARG on any overlap).  cell_start is cleared on the stream each call;
 * nothing else needs to start at zero.  The first call on a device, and the
 * first after the current context changes (cudaDeviceReset, or another
 * context made current), looks up the array's address in that context
 * (cudaGetSymbolAddress): make it before any stream capture.  All calls on a
 * device share the array, so calls whose executions overlap (different
 * streams or host threads) race: order them. */
#define PF_SORT_STATIC_MAX_CELLS 134217728LL /* 512^3 */
int pf_sort_particles_static(const pf_grid* g, int64_t n, const float* pos4_in, const float* vel4_in,
                             float* pos4_out, float* vel4_out, int32_t* keys_out, int32_t* perm_out,
                             int32_t* cell_start, void* stream);

/* P2G: replaces pfflip/kernels.py:100-158 (p2g_face, x3 axes) and :161-209
 * (p2g_cell) as launched by pfflip/sim.py:205-228, including the zeroing of the
 * 8 accumulators.  Eq. (6) weights with support radius r_p; particle mass is
 * rho_l for liquid, rho_g for air; particles with pstate != 0 are skipped.
 * Requires cell_start of the sort above (pos4/vel4 in sorted order). */
int pf_p2g(const pf_grid* g, int64_t n, const float* pos4, const float* vel4, const int32_t* cell_start, float rho_l,
           float rho_g, float r_p, float* mass_x, float* mass_y, float* mass_z, float* mom_x, float* mom_y,
           float* mom_z, float* cell_mass, float* cell_wsum, void* stream);

/* Face velocities, phase field and Poisson coefficients in one pass; replaces
 * pfflip/kernels.py:212-228 (face_velocity_from_momentum), :244-255
 * (cell_phase), :258-311 (face_beta), :314-326 (zero_solid_faces) and
 * :601-627 (zero_solid_obstacle_faces), as sequenced by pfflip/sim.py:229-268.
 *   u_a = P_a/m_a where m_a > mass_eps else 0; phi_cell by eq. (7); is_liquid =
 *   phi >= 0.5; face phi 1/0 between equal tags, eq. (7) of the face mass
 *   otherwise; beta = 1/((1-phi) rho_g + phi rho_l); beta = u = 0 on domain
 *   boundary faces and on faces touching a solid cell (solid may be NULL).
 * valid_* and phi_face_* may be NULL (not written). */
int pf_phase_beta(const pf_grid* g, const float* mass_x, const float* mass_y, const float* mass_z,
                  const float* mom_x, const float* mom_y, const float* mom_z, const float* cell_mass,
                  const int32_t* solid, float mass_eps, float rho_min, float alpha_phi, float rho_0l, float rho_l,
                  float rho_g, float* vel_x, float* vel_y, float* vel_z, int32_t* valid_x, int32_t* valid_y,
                  int32_t* valid_z, float* phi_cell, int32_t* is_liquid, float* phi_face_x, float* phi_face_y,
                  float* phi_face_z, float* beta_x, float* beta_y, float* beta_z, void* stream);

/* vel_star = vel (any of vel_star_* may be NULL to skip the copy), then
 * vel += g*dt on every face of each axis with g != 0, then vel = 0 on domain
 * boundary faces and faces touching a solid cell.  Replaces the copy at
 * pfflip/sim.py:176-177 and _add_forces, pfflip/sim.py:270-285
 * (pfflip/kernels.py:332-335 add_gravity, :314-326, :601-627). */
int pf_save_and_force(const pf_grid* g, float* vel_x, float* vel_y, float* vel_z, float* vel_star_x,
                      float* vel_star_y, float* vel_star_z, const int32_t* solid, float gx, float gy, float gz,
                      float dt, void* stream);

/* b = -(dx/dt) div u  [- dx^2 k_div max((wsum-rho_0)/rho_0, 0)/dt]; replaces
 * pfflip/kernels.py:338-363 (build_rhs).  cell_wsum may be NULL when k_div == 0. */
int pf_build_rhs(const pf_grid* g, const float* vel_x, const float* vel_y, const float* vel_z,
                 const float* cell_wsum, float* b, float dt, float rho_0, float k_div, void* stream);

/* u -= dt beta (p_i - p_{i-1}) / dx on interior faces with beta != 0;
 * replaces pfflip/kernels.py:366-387 (apply_pressure_gradient, x3 axes). */
int pf_project(const pf_grid* g, const float* p, const float* beta_x, const float* beta_y, const float* beta_z,
               float* vel_x, float* vel_y, float* vel_z, float dt, void* stream);

/* max |div u| / dx written to the device float *out; replaces
 * pfflip/kernels.py:390-400 (divergence_norm) used by pfflip/sim.py:310-314. */
int pf_max_divergence(const pf_grid* g, const float* vel_x, const float* vel_y, const float* vel_z, float* out,
                      void* stream);

/* Liquid velocity extrapolation: seed faces touching a liquid cell, then
 * `sweeps` Jacobi sweeps of the mean of known axial neighbours within each
 * face array.  Replaces pfflip/kernels.py:406-425 (seed_liquid_velocity) and
 * :428-462 (extrapolate_sweep) as run by pfflip/sim.py:329-341.  known_* may
 * be NULL: the same velocities then come from one shared-memory pass per tile
 * over all sweeps, which is slower on large grids (0.47 against 0.16 ms at
 * 128^3), so pass the known arrays where speed matters.  sweeps must be <= 4. */
int pf_extrapolate(const pf_grid* g, const float* vel_x, const float* vel_y, const float* vel_z,
                   const int32_t* is_liquid, int32_t sweeps, float* vel_liq_x, float* vel_liq_y, float* vel_liq_z,
                   int32_t* known_x, int32_t* known_y, int32_t* known_z, void* stream);

/* Grid-to-particle transfer and advection in one particle pass.
 *   do_g2p:    v = alpha (v + I(u - u*)) + (1 - alpha) I(u), alpha per phase;
 *              replaces pfflip/kernels.py:468-502 (g2p, field_difference).
 *   do_advect: Ralston RK3 through vel_liq (liquid) or vel (air), clamp to
 *              [lo, hi], then wall reflection; replaces pfflip/kernels.py:508-549
 *              (advect_rk3) and :567-595 (reflect_at_walls); with a non-NULL
 *              solid mask also :630-679 (push_out_of_solids).
 * Particles with pstate != 0 are not transferred or advected; pstate == 2 is
 * not reflected (as in the reference). */
int pf_g2p_advect(const pf_grid* g, int64_t n, float* pos4, float* vel4, const float* vel_x, const float* vel_y,
                  const float* vel_z, const float* vstar_x, const float* vstar_y, const float* vstar_z,
                  const float* vliq_x, const float* vliq_y, const float* vliq_z, const int32_t* solid,
                  float alpha_liquid, float alpha_air, float dt, const float lo[3], const float hi[3],
                  int32_t do_g2p, int32_t do_advect, void* stream);

/* The same pass reading the face fields through (j, k) quads built in the
 * caller's workspace (pf_g2p_workspace_bytes, 256-byte aligned): per face of
 * u, u* and vel_liq, (v[j][k], v[j][k+1], v[j+1][k], v[j+1][k+1]).  A
 * trilinear sample then takes two 16-byte loads instead of eight gathers;
 * every tap value is the one pf_g2p_advect reads (sums within rounding).
 * max_speed (device float, may be NULL): cleared on the stream, then set to
 * the largest |v| over the FLIP particles (pstate 0) as this pass leaves
 * them: the value pf_particle_max_speed would return right after the pass
 * (pfflip/kernels.py:552-564 as called by pfflip/sim.py:157-166), so the next
 * step's CFL dt needs no separate particle pass.
 * Same arguments and results otherwise. */
size_t pf_g2p_workspace_bytes(const pf_grid* g);
int pf_g2p_advect_packed(const pf_grid* g, int64_t n, float* pos4, float* vel4, const float* vel_x,
                         const float* vel_y, const float* vel_z, const float* vstar_x, const float* vstar_y,
                         const float* vstar_z, const float* vliq_x, const float* vliq_y, const float* vliq_z,
                         const int32_t* solid, float alpha_liquid, float alpha_air, float dt, const float lo[3],
                         const float hi[3], int32_t do_g2p, int32_t do_advect, float* max_speed, void* workspace,
                         size_t workspace_bytes, void* stream);

/* max |v| over particles with pstate == 0, written to the device float *out;
 * replaces pfflip/kernels.py:552-564 (particle_max_speed). */
int pf_particle_max_speed(int64_t n, const float* pos4, const float* vel4, float* out, void* stream);

/* ------------------------------------------------------------- droplets */
/* Escaped particles, droplets and spray; pfflip/droplets.py as run by
 * pfflip/sim.py:343-401.  A particle's state is bits 1-2 of its flags
 * (0 FLIP, 1 droplet, 2 dead); drop_r[n] is the droplet radius, in the order
 * of pos4/vel4 (after a sort, permute it with pf_permute_f32 and perm_out).
 * counters[4] accumulate (emitted, bubbles deleted, merged back, spray); the
 * caller zeroes them.  Random numbers (radii, spray emission) come from a
 * PCG-hash stream keyed by (seed, particle id = vel4.w), not from the
 * reference's Warp stream: radii follow the same log-normal law
 * exp(r_mu + r_sigma N(0,1)) clamped to [r_min, r_max], with other values. */

/* classify_escaped (pfflip/droplets.py:67-106): liquid FLIP particles where
 * the trilinear cell phi < 1/2 - delta_phi become droplets; air FLIP particles
 * where phi > 1/2 + delta_phi die (bubbles); droplets where phi > 1/2 +
 * delta_phi merge back. */
int pf_droplet_classify(const pf_grid* g, int64_t n, float* pos4, const float* vel4, float* drop_r,
                        const float* phi_cell, float delta_phi, float r_mu, float r_sigma, float r_min, float r_max,
                        uint32_t seed, int32_t* counters, void* stream);

/* velocity_gradient_magnitude (pfflip/droplets.py:153-194): |grad u| at cell
 * centres from the MAC faces. */
int pf_velocity_gradient(const pf_grid* g, const float* vel_x, const float* vel_y, const float* vel_z, float* out,
                         void* stream);

/* emit_spray_in_shear (pfflip/droplets.py:112-150): liquid FLIP particles of
 * the interfacial band (0.1 <= phi <= 0.9) with shear >= threshold become
 * droplets with probability rate. */
int pf_spray_emit(const pf_grid* g, int64_t n, float* pos4, const float* vel4, float* drop_r, const float* phi_cell,
                  const float* shear, float threshold, float rate, float r_mu, float r_sigma, float r_min, float r_max,
                  uint32_t seed, int32_t* counters, void* stream);

/* advance_droplets (pfflip/droplets.py:211-279): per-droplet sub-steps
 * min(int(|v| dt / (dx/2)) + 1, max_substeps), gravity + sphere drag through
 * the face velocities, evaporation dr/dt = -evap_k/r by RK2; droplets that
 * leave [lo, hi] or shrink to r_min die. */
int pf_droplet_advance(const pf_grid* g, int64_t n, float* pos4, float* vel4, float* drop_r, const float* vel_x,
                       const float* vel_y, const float* vel_z, float dt, const float gravity[3], float rho_g,
                       float rho_l, float drag_cd, float evap_k, float r_min, const float lo[3], const float hi[3],
                       int32_t max_substeps, void* stream);

/* rasterize_spray (pfflip/droplets.py:309-353): droplet volume splatted into
 * a float16 grid (sx, sy, sz) of spacing dx_spray, zeroed first. */
int pf_spray_rasterize(int64_t n, const float* pos4, const float* drop_r, void* density_f16, int32_t sx, int32_t sy,
                       int32_t sz, float dx_spray, void* stream);

/* out[t] = in[perm[t]]: a per-particle float follows the sort. */
int pf_permute_f32(int64_t n, const int32_t* perm, const float* in, float* out, void* stream);

/* --------------------------------------------------------------- Poisson */
/* (Ap)_i = sum_f beta_f (p_i - p_nbr) with clamped neighbour indices;
 * replaces pfflip/poisson.py:54-88 (apply_A).  stencil = PF_STENCIL_REFERENCE
 * evaluates diag*p_i - sum beta p_nbr with diag = the given array (or, when
 * diag is NULL, the 6-face sum formed in compute_diag's order);
 * PF_STENCIL_FLUX evaluates sum beta (p_i - p_nbr) and ignores diag. */
int pf_apply_A(const pf_grid* g, const float* p, const float* bx, const float* by, const float* bz,
               const float* diag, float* out, int32_t stencil, void* stream);

/* One multigrid level.  fp32 arrays always; *_lp arrays are the 16-bit
 * storage used when precision != PF_PREC_FP32 (NULL otherwise).
 * The solver requires beta = 0 on the domain boundary faces, which the
 * reference's simulator always produces (pfflip/kernels.py:314-326); the
 * smoother then never reads outside the level. */
typedef struct pf_mg_level {
  int32_t nx, ny, nz;
  float *bx, *by, *bz, *diag; /* coefficients; diag kept for the reference's attribute */
  float *p, *p_alt;           /* solution and its ping-pong partner */
  float *b, *r;               /* right-hand side, residual */
  void *bx_lp, *by_lp, *bz_lp;
  void *p_lp, *p_lp_alt, *b_lp;
  /* optional copy of bz with rows padded to bz_pitch floats (bz_pitch a multiple
   * of 8, >= nz+1), filled by pf_mg_build_hierarchy: lets the fp32 smoother
   * stage z-faces with TMA, whose row pitch must be a multiple of 16 bytes.
   * NULL: that level's smoother stages through registers. */
  float* bz_pad;
  int32_t bz_pitch;
} pf_mg_level;

/* Multigrid-preconditioned flexible CG; mirrors pfflip/poisson.py:240-274
 * (MGPCG.__init__).  All pointers are device memory owned by the caller:
 *   rhs, res_v, res_alt, z, q, Ap, x: finest-level vectors (nx*ny*nz floats);
 *             x accumulates the iterate, the caller's output is written at the end
 *   state:    PF_MG_STATE_BYTES bytes
 *   partials: pf_mg_partials_count() doubles
 *   counters: PF_MG_COUNTERS uint32 (zeroed by the caller once) */
#define PF_MG_STATE_BYTES 512
#define PF_MG_COUNTERS 32
typedef struct pf_mg_desc {
  int32_t nlev;
  pf_mg_level lev[PF_MG_MAX_LEVELS];
  float omega;
  int32_t pre, post, coarsest;
  int32_t precision;   /* PF_PREC_* */
  int32_t stencil;     /* PF_STENCIL_* for every operator row (CG, smoother, residual) */
  float coef_scale;    /* 16-bit storage: beta is stored times coef_scale (power of two) */
  float *rhs, *res_v, *res_alt, *z, *q, *Ap, *x;
  void* state;
  double* partials;
  uint32_t* counters;
  /* optional (NULL = off): pf_mg_bottom_op_floats(desc) floats for the dense
   * operator of the V-cycle's smallest levels, rebuilt by every
   * pf_mg_build_hierarchy (see pf_mg_bottom_info) */
  float* bottom_op;
} pf_mg_desc;

typedef struct pf_mg_plan pf_mg_plan;

int64_t pf_mg_partials_count(void);
/* Level count of the reference's hierarchy rule (pfflip/poisson.py:256-263):
 * halve while min(res)//2 >= min_dim and every dimension is even; writes the
 * level dimensions (3 ints per level) into dims_out (may be NULL). */
int32_t pf_mg_level_count(int32_t nx, int32_t ny, int32_t nz, int32_t min_dim, int32_t* dims_out);
int pf_mg_plan_create(const pf_mg_desc* desc, pf_mg_plan** out);
int pf_mg_plan_destroy(pf_mg_plan* plan);
/* Which kernel runs the coarse end of the plan's V-cycle (no reference
 * counterpart; diagnostics).  *first_level: the finest level it covers (nlev:
 * none); *cluster_levels: > 0 when it is the cluster kernel (one cluster of
 * 8 CTAs; that many levels from first_level split into slabs across the CTAs),
 * 0 for the single-CTA kernel; *dense: 1 when the levels below the slabs are
 * applied as a dense operator (desc->bottom_op), 0 when CTA 0 sweeps them.
 * The cluster kernel is used whenever the levels allow it; the environment
 * variable PFFLIP_MG_BOTTOM, read at plan creation, selects "cta" (single-CTA
 * kernel) or "cluster" (cluster kernel without the dense operator). */
int pf_mg_bottom_info(const pf_mg_plan* plan, int32_t* first_level, int32_t* cluster_levels, int32_t* dense);
/* Floats desc->bottom_op must hold for the plan that desc would create (0: the
 * dense bottom does not apply to these levels).  The dense operator is the
 * exact linear map of the V-cycle below the cluster's slabs (pre-smoothing,
 * restriction, coarsest sweeps with mean removal, prolongation,
 * post-smoothing), built column by column from unit right-hand sides. */
int64_t pf_mg_bottom_op_floats(const pf_mg_desc* desc);
/* pfflip/poisson.py:295-309 build_hierarchy: level-0 faces = (bx, by, bz),
 * per level diag = sum of 6 faces, coarse face = sum of the 2x2 fine faces in
 * plane 2I.  Also fills the 16-bit copies in mixed precision. */
int pf_mg_build_hierarchy(pf_mg_plan* plan, const float* bx, const float* by, const float* bz, void* stream);
/* pfflip/poisson.py:345-352 precondition: z = one V-cycle applied to r, mean removed. */
int pf_mg_precondition(pf_mg_plan* plan, const float* r, float* z, void* stream);
/* Level smoother (pfflip/poisson.py:312-321): `nsweeps` red-black sweeps on
 * level lv in place on lev[lv].p (reverse: black first). */
int pf_mg_smooth(pf_mg_plan* plan, int32_t lv, int32_t nsweeps, int32_t reverse, void* stream);
/* pfflip/poisson.py:355-409 solve.  Synchronises `stream`; writes the
 * iteration count and the final inf-norm relative residual to host memory.
 * use_graphs: replay each CG iteration as a captured CUDA graph.
 * verbose: print the residual of every iteration to stdout.
 * Returns PF_OK, PF_ERR_NOT_CONVERGED (results valid) or an error. */
int pf_mg_solve(pf_mg_plan* plan, const float* b, float* x, float tol, int32_t max_iter, int32_t use_graphs,
                int32_t verbose, int32_t* iters_out, double* rel_out, void* stream);

/* --------------------------------------------------------------- adjoint */
/* Reverse-mode counterparts of the step's stages.  The reference step
 * (pfflip/sim.py:168-202) is not differentiable, so none of these replaces a
 * reference entry point; each is the vector-Jacobian product of the forward
 * stage cited.  Discrete decisions (sort order, liquid tags, extrapolation
 * masks, wall clamps, the valid-face test) are held fixed.  Particle
 * adjoints are float4 streams (x, y, z, unused) in the order of pos4/vel4.
 * The adjoint of the pressure solve is an MG-PCG solve by the caller:
 * lam = pf_mg_solve(plan built for the same beta, b = p_bar).  Order of use
 * for one step, in reverse:
 *   pf_adj_g2p_advect -> pf_adj_extrapolate -> pf_adj_project -> pf_mg_solve
 *   -> pf_adj_face_sources -> pf_adj_p2g -> pf_adj_unsort.
 * Face-grid adjoint outputs marked "accumulate" must be zeroed by the caller. */

/* G2P + Ralston RK3 + wall reflection (pfflip/kernels.py:468-549, :567-595).
 * pos4/vel4: the particles at the start of the step (sorted order); vel_*:
 * the projected field u, vstar_*: u*, vliq_*: the extrapolated field.
 * gpos4_in/gvel4_in: adjoints of the particles after the step.  Writes
 * gpos4_out/gvel4_out (adjoints at the start of the step, G2P/advection part)
 * and accumulates into gvel_* (u), gvstar_* (u*) and gvliq_* (extrapolated). */
int pf_adj_g2p_advect(const pf_grid* g, int64_t n, const float* pos4, const float* vel4, const float* vel_x,
                      const float* vel_y, const float* vel_z, const float* vstar_x, const float* vstar_y,
                      const float* vstar_z, const float* vliq_x, const float* vliq_y, const float* vliq_z,
                      float alpha_liquid, float alpha_air, float dt, const float lo[3], const float hi[3],
                      int32_t do_g2p, int32_t do_advect, const float* gpos4_in, const float* gvel4_in,
                      float* gpos4_out, float* gvel4_out, float* gvel_x, float* gvel_y, float* gvel_z,
                      float* gvstar_x, float* gvstar_y, float* gvstar_z, float* gvliq_x, float* gvliq_y,
                      float* gvliq_z, void* stream);

/* Transpose of the liquid extrapolation (pfflip/kernels.py:406-462) with
 * `sweeps` Jacobi sweeps.  gliq_*: adjoint of the extrapolated field (used as
 * scratch, destroyed); tmp_*: face-sized float scratch; level_*, level_tmp_*:
 * face-sized byte scratch.  Accumulates into gvel_*. */
int pf_adj_extrapolate(const pf_grid* g, const int32_t* is_liquid, int32_t sweeps, float* gliq_x, float* gliq_y,
                       float* gliq_z, float* tmp_x, float* tmp_y, float* tmp_z, uint8_t* level_x, uint8_t* level_y,
                       uint8_t* level_z, uint8_t* level_tmp_x, uint8_t* level_tmp_y, uint8_t* level_tmp_z,
                       float* gvel_x, float* gvel_y, float* gvel_z, void* stream);

/* Projection u -= dt*beta*(p_i - p_{i-1})/dx (pfflip/kernels.py:366-387):
 * writes gp (cells, the right-hand side of the adjoint solve) and gbeta_*
 * (faces) from the adjoint gvel_* of the projected field. */
int pf_adj_project(const pf_grid* g, const float* p, const float* beta_x, const float* beta_y, const float* beta_z,
                   const float* gvel_x, const float* gvel_y, const float* gvel_z, float dt, float* gp,
                   float* gbeta_x, float* gbeta_y, float* gbeta_z, void* stream);

/* Face sources of the solve, from the adjoint solution lam: the divergence
 * right-hand side (pfflip/kernels.py:338-363, k_div = 0), gravity and wall
 * zeroing (:332-335, :314-326), the u* copy (pfflip/sim.py:176-177), eq. (9)
 * beta with eq. (7) at mixed faces (pfflip/kernels.py:258-311), the
 * operator's beta sensitivity -(lam_i - lam_j)(p_i - p_j), and u = P/m
 * (:212-228).  gvel_*: adjoint of u after projection (all contributions),
 * gvstar_*: adjoint of u*, gbeta_*: from pf_adj_project.  Writes the
 * adjoints of the P2G face accumulators, gmass_* and gmom_*. */
int pf_adj_face_sources(const pf_grid* g, const float* p, const float* lam, const float* beta_x, const float* beta_y,
                        const float* beta_z, const float* mass_x, const float* mass_y, const float* mass_z,
                        const float* mom_x, const float* mom_y, const float* mom_z, const int32_t* is_liquid,
                        float mass_eps, float rho_min, float alpha_phi, float rho_0l, float rho_l, float rho_g,
                        float dt, const float* gvel_x, const float* gvel_y, const float* gvel_z,
                        const float* gvstar_x, const float* gvstar_y, const float* gvstar_z, const float* gbeta_x,
                        const float* gbeta_y, const float* gbeta_z, float* gmass_x, float* gmass_y, float* gmass_z,
                        float* gmom_x, float* gmom_y, float* gmom_z, void* stream);

/* P2G splat, eq. (6) (pfflip/kernels.py:100-209): a per-particle gather of
 * the face mass/momentum adjoints (all six, or all NULL) and of the cell-mass
 * adjoint (gcell_mass, may be NULL).  Accumulates into gpos4/gvel4. */
int pf_adj_p2g(const pf_grid* g, int64_t n, const float* pos4, const float* vel4, float rho_l, float rho_g, float r_p,
               const float* gmass_x, const float* gmass_y, const float* gmass_z, const float* gmom_x,
               const float* gmom_y, const float* gmom_z, const float* gcell_mass, float* gpos4, float* gvel4,
               void* stream);

/* eq. (7) on cells (pfflip/kernels.py:234-255): gcell_mass = dphi/dm * gphi,
 * zero on the clamped pieces. */
int pf_adj_phase_cell(const pf_grid* g, const float* cell_mass, const float* gphi, float rho_min, float alpha_phi,
                      float rho_0l, float* gcell_mass, void* stream);

/* Adjoint of the sort's gather: out[perm[t]] = in[t] for both streams. */
int pf_adj_unsort(int64_t n, const int32_t* perm, const float* gpos4_sorted, const float* gvel4_sorted,
                  float* gpos4_out, float* gvel4_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PFFLIP_H */
