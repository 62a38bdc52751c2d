// extern "C" entry points of the CPU oracle (test infrastructure only; see
// pf_oracle.hpp).  Each function is instantiated for binary32 (_f32) and
// binary64 (_f64).  Pointers are host arrays in the reference's layouts.
#include "pf_oracle.hpp"

using namespace pfo;

extern "C" {

void pfo_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}

int pfo_get_threads(void) { return nthreads_default(); }

void pfo_set_stencil(int form) { g_stencil = form; }

void pfo_sort_by_cell(int64_t n, const float* pos, float dx, int nx, int ny, int nz, int32_t* keys, int32_t* perm,
                      int32_t* cell_start) {
  sort_by_cell(n, pos, dx, nx, ny, nz, keys, perm, cell_start);
}

#define PFO_DEFINE(R, SFX)                                                                                        \
  void pfo_p2g_##SFX(int64_t n, const R* px, const R* pv, const R* pmass, const R* prad, const int32_t* pstate,    \
                     int nx, int ny, int nz, R dx, R* m0, R* m1, R* m2, R* q0, R* q1, R* q2, R* cmass, R* cwsum,   \
                     int nthr) {                                                                                  \
    P2GArgs<R> a{n, px, pv, pmass, prad, pstate, nx, ny, nz, dx};                                                 \
    R* mass[3] = {m0, m1, m2};                                                                                    \
    R* mom[3] = {q0, q1, q2};                                                                                     \
    p2g(a, mass, mom, cmass, cwsum, nthr);                                                                        \
  }                                                                                                               \
  void pfo_face_velocity_##SFX(const R* mass, const R* mom, R* vel, int32_t* valid, int64_t n, R eps) {           \
    face_velocity_from_momentum(mass, mom, vel, valid, n, eps);                                                   \
  }                                                                                                               \
  void pfo_cell_phase_##SFX(const R* cmass, R* phi, int32_t* liq, int64_t n, R rho_min, R alpha_phi, R rho_0l) { \
    cell_phase(cmass, phi, liq, n, rho_min, alpha_phi, rho_0l);                                                   \
  }                                                                                                               \
  void pfo_face_beta_##SFX(const R* mass, const int32_t* liq, R* phi_face, R* beta, int nx, int ny, int nz,       \
                           int axis, R rho_min, R alpha_phi, R rho_0l, R rho_l, R rho_g) {                        \
    face_beta(mass, liq, phi_face, beta, nx, ny, nz, axis, rho_min, alpha_phi, rho_0l, rho_l, rho_g);             \
  }                                                                                                               \
  void pfo_zero_solid_faces_##SFX(R* beta, R* vel, int nx, int ny, int nz, int axis) {                            \
    zero_solid_faces(beta, vel, nx, ny, nz, axis);                                                                \
  }                                                                                                               \
  void pfo_zero_solid_obstacle_faces_##SFX(const int32_t* solid, R* beta, R* vel, int nx, int ny, int nz,         \
                                           int axis) {                                                            \
    zero_solid_obstacle_faces(solid, beta, vel, nx, ny, nz, axis);                                                \
  }                                                                                                               \
  void pfo_add_gravity_##SFX(R* vel, int64_t n, R g, R dt) { add_gravity(vel, n, g, dt); }                        \
  void pfo_build_rhs_##SFX(const R* u, const R* v, const R* w, const R* cwsum, R* b, int nx, int ny, int nz,      \
                           R dx, R dt, R rho_0, R k_div) {                                                        \
    build_rhs(u, v, w, cwsum, b, nx, ny, nz, dx, dt, rho_0, k_div);                                               \
  }                                                                                                               \
  void pfo_apply_pressure_gradient_##SFX(const R* p, const R* beta, R* vel, int nx, int ny, int nz, int axis,     \
                                         R dx, R dt) {                                                            \
    apply_pressure_gradient(p, beta, vel, nx, ny, nz, axis, dx, dt);                                              \
  }                                                                                                               \
  R pfo_divergence_norm_##SFX(const R* u, const R* v, const R* w, int nx, int ny, int nz, R dx) {                 \
    return divergence_norm(u, v, w, nx, ny, nz, dx);                                                              \
  }                                                                                                               \
  void pfo_seed_liquid_velocity_##SFX(const R* vel, const int32_t* liq, R* vel_l, int32_t* known, int nx,         \
                                      int ny, int nz, int axis) {                                                 \
    seed_liquid_velocity(vel, liq, vel_l, known, nx, ny, nz, axis);                                               \
  }                                                                                                               \
  void pfo_extrapolate_sweep_##SFX(const R* vel_l, const int32_t* known, R* vel_out, int32_t* known_out, int n0,  \
                                   int n1, int n2) {                                                              \
    extrapolate_sweep(vel_l, known, vel_out, known_out, Dims{n0, n1, n2});                                        \
  }                                                                                                               \
  void pfo_g2p_##SFX(int64_t n, const R* px, R* pv, const int32_t* ptype, const int32_t* pstate, const R* u0,     \
                     const R* u1, const R* u2, const R* d0, const R* d1, const R* d2, int nx, int ny, int nz,     \
                     R dx, R a_liq, R a_air) {                                                                    \
    const R* u[3] = {u0, u1, u2};                                                                                 \
    const R* du[3] = {d0, d1, d2};                                                                                \
    g2p(n, px, pv, ptype, pstate, u, du, nx, ny, nz, dx, a_liq, a_air);                                           \
  }                                                                                                               \
  void pfo_advect_reflect_##SFX(int64_t n, R* px, R* pv, const int32_t* ptype, const int32_t* pstate,             \
                                const R* u0, const R* u1, const R* u2, const R* l0, const R* l1, const R* l2,     \
                                int nx, int ny, int nz, R dt, R dx, const R* lo, const R* hi) {                   \
    const R* u[3] = {u0, u1, u2};                                                                                 \
    const R* ul[3] = {l0, l1, l2};                                                                                \
    advect_reflect(n, px, pv, ptype, pstate, u, ul, nx, ny, nz, dt, dx, lo, hi);                                  \
  }                                                                                                               \
  void pfo_push_out_of_solids_##SFX(int64_t n, R* px, R* pv, const int32_t* pstate, const int32_t* solid,         \
                                    int nx, int ny, int nz, R dx) {                                               \
    push_out_of_solids(n, px, pv, pstate, solid, nx, ny, nz, dx);                                                 \
  }                                                                                                               \
  void pfo_droplet_classify_##SFX(int64_t n, const R* px, const int32_t* ptype, int32_t* pstate, R* pdrop_r,     \
                                  const R* phi, int nx, int ny, int nz, R dx, R delta_phi, R mu, R sigma, R rmin, \
                                  R rmax, uint32_t seed, int32_t* counters) {                                     \
    droplet_classify(n, px, ptype, pstate, pdrop_r, phi, nx, ny, nz, dx, delta_phi, mu, sigma, rmin, rmax, seed,  \
                     counters);                                                                                   \
  }                                                                                                               \
  void pfo_velocity_gradient_##SFX(const R* u, const R* v, const R* w, R* out, int nx, int ny, int nz, R dx) {    \
    velocity_gradient(u, v, w, out, nx, ny, nz, dx);                                                              \
  }                                                                                                               \
  void pfo_spray_emit_##SFX(int64_t n, const R* px, const int32_t* ptype, int32_t* pstate, R* pdrop_r,            \
                            const R* phi, const R* shear, int nx, int ny, int nz, R dx, R threshold, R rate,      \
                            R mu, R sigma, R rmin, R rmax, uint32_t seed, int32_t* counters) {                    \
    spray_emit(n, px, ptype, pstate, pdrop_r, phi, shear, nx, ny, nz, dx, threshold, rate, mu, sigma, rmin, rmax, \
               seed, counters);                                                                                   \
  }                                                                                                               \
  void pfo_droplet_advance_##SFX(int64_t n, R* px, R* pv, int32_t* pstate, R* pdrop_r, const R* u0, const R* u1,  \
                                 const R* u2, int nx, int ny, int nz, R dt, R dx, const R* grav, R rho_g,         \
                                 R rho_l, R cd, R evap_k, R rmin, const R* lo, const R* hi, int max_sub) {        \
    const R* u[3] = {u0, u1, u2};                                                                                 \
    droplet_advance(n, px, pv, pstate, pdrop_r, u, nx, ny, nz, dt, dx, grav, rho_g, rho_l, cd, evap_k, rmin, lo,  \
                    hi, max_sub);                                                                                 \
  }                                                                                                               \
  void pfo_spray_rasterize_##SFX(int64_t n, const R* px, const int32_t* pstate, const R* pdrop_r, R* density,     \
                                 int sx, int sy, int sz, R dxs) {                                                 \
    spray_rasterize(n, px, pstate, pdrop_r, density, sx, sy, sz, dxs);                                            \
  }                                                                                                               \
  R pfo_particle_max_speed_##SFX(int64_t n, const R* pv, const int32_t* pstate) {                                 \
    return particle_max_speed(n, pv, pstate);                                                                     \
  }                                                                                                               \
  void pfo_apply_A_##SFX(const R* p, const R* bx, const R* by, const R* bz, const R* diag, R* out, int nx,        \
                         int ny, int nz) {                                                                        \
    apply_A(p, bx, by, bz, diag, out, nx, ny, nz);                                                                \
  }                                                                                                               \
  void* pfo_mg_create_##SFX(int nx, int ny, int nz, R omega, int pre, int post, int coarsest, int min_dim) {      \
    MGPCG<R>* m = new MGPCG<R>();                                                                                 \
    m->init(nx, ny, nz, omega, pre, post, coarsest, min_dim);                                                     \
    return m;                                                                                                     \
  }                                                                                                               \
  void pfo_mg_destroy_##SFX(void* h) { delete (MGPCG<R>*)h; }                                                     \
  int pfo_mg_nlev_##SFX(void* h) { return (int)((MGPCG<R>*)h)->levels.size(); }                                   \
  void pfo_mg_level_dims_##SFX(void* h, int lv, int* out) {                                                       \
    Level<R>& L = ((MGPCG<R>*)h)->levels[lv];                                                                     \
    out[0] = L.nx; out[1] = L.ny; out[2] = L.nz;                                                                  \
  }                                                                                                               \
  /* which: 0 bx, 1 by, 2 bz, 3 diag, 4 p, 5 b, 6 r; dir 0 = read out, 1 = write in */                           \
  void pfo_mg_level_io_##SFX(void* h, int lv, int which, R* buf, int dir) {                                       \
    Level<R>& L = ((MGPCG<R>*)h)->levels[lv];                                                                     \
    std::vector<R>* v[7] = {&L.bx, &L.by, &L.bz, &L.diag, &L.p, &L.b, &L.r};                                      \
    if (dir == 0) std::copy(v[which]->begin(), v[which]->end(), buf);                                             \
    else std::copy(buf, buf + v[which]->size(), v[which]->begin());                                               \
  }                                                                                                               \
  void pfo_mg_build_##SFX(void* h, const R* bx, const R* by, const R* bz) {                                       \
    ((MGPCG<R>*)h)->build_hierarchy(bx, by, bz);                                                                  \
  }                                                                                                               \
  void pfo_mg_precondition_##SFX(void* h, const R* r, R* z) { ((MGPCG<R>*)h)->precondition(r, z); }               \
  void pfo_mg_smooth_##SFX(void* h, int lv, int nsweeps, int reverse) {                                           \
    MGPCG<R>* m = (MGPCG<R>*)h;                                                                                   \
    m->smooth(m->levels[lv], nsweeps, reverse != 0);                                                              \
  }                                                                                                               \
  int pfo_mg_solve_##SFX(void* h, const R* b, R* x, double tol, int max_iter, double* rel, double* hist,          \
                         int hist_cap) {                                                                          \
    std::vector<double> hv;                                                                                       \
    int it = ((MGPCG<R>*)h)->solve(b, x, tol, max_iter, rel, &hv);                                                \
    for (int i = 0; i < (int)hv.size() && i < hist_cap; ++i) hist[i] = hv[i];                                    \
    return it;                                                                                                    \
  }

PFO_DEFINE(float, f32)
PFO_DEFINE(double, f64)

}  // extern "C"
