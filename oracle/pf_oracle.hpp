// CPU restatement of the uniform-grid PF-FLIP step — TEST INFRASTRUCTURE ONLY.
//
// This file is the parity oracle and the timed CPU baseline ("port") for the
// CUDA library.  Nothing in the product links or calls it: only tests/,
// __graft_entry__.smoke() and bench.py's CPU legs load it.
//
// Every function restates one reference kernel, cited as file:line inside the
// reference project (pfflip/kernels.py, pfflip/poisson.py, pfflip/sim.py).
// Arithmetic follows the reference's written operation order in IEEE binary32
// (instantiated with R = float) or binary64 (R = double, the 1e-12 FP64 oracle
// and the finite-difference engine).  Build with -ffp-contract=off so no FMA is
// formed that the reference's source does not write.
//
// Parity pin: the reference's GPU/CPU kernels need NVIDIA Warp, which is not
// installed (no network), so the oracle is pinned against the reference's own
// test vectors instead: the SciPy-assembled operator and direct solve of
// tests/test_poisson.py:23-145, the ρ̃₀ closed form of tests/test_pfflip.py:35-41,
// and bit-exact seeding from pfflip/scenes.py (fixtures in tests/golden/).
//
// Layouts follow the reference: 3D arrays are C-order (nx, ny, nz), index
// (i*ny + j)*nz + k; face arrays of axis a have shape res + e_a; particle
// positions/velocities are AoS (n, 3).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace pfo {

// Stencil form of the operator rows.  0: the reference's written form
// diag*p_i - sum_f beta_f p_nbr (pfflip/poisson.py:69-75).  1: the flux form
// sum_f beta_f (p_i - p_nbr), equal in exact arithmetic, free of the
// cancellation that stalls the reference form near 1e-6..1e-5 in binary32.
inline int g_stencil = 0;

struct Dims {
  int n0, n1, n2;
  int64_t size() const { return (int64_t)n0 * n1 * n2; }
  int64_t at(int i, int j, int k) const { return ((int64_t)i * n1 + j) * n2 + k; }
};

inline Dims face_dims(int nx, int ny, int nz, int axis) {
  return Dims{nx + (axis == 0), ny + (axis == 1), nz + (axis == 2)};
}

inline int nthreads_default() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// pfflip/kernels.py:25-33 face_offset: o_a = (.5,.5,.5) - .5 e_a
template <class R> inline R face_off(int axis, int d) { return axis == d ? R(0) : R(0.5); }

// pfflip/kernels.py:41-49 splat_weight, eq. (6)
template <class R> inline R splat_weight(R d2, R r2) {
  R t = R(1) - d2 / r2;
  t = std::max(t, R(0));
  return t * t * t;
}

// pfflip/kernels.py:52-79 sample_face (clamped trilinear).  o = -1 selects the
// cell-centred offset (0.5 on every axis).
template <class R> inline R sample_face(const R* f, Dims d, const R x[3], R dx, int axis) {
  R g0 = x[0] / dx - face_off<R>(axis, 0);
  R g1 = x[1] / dx - face_off<R>(axis, 1);
  R g2 = x[2] / dx - face_off<R>(axis, 2);
  int i0 = (int)std::floor(g0), j0 = (int)std::floor(g1), k0 = (int)std::floor(g2);
  R tx = g0 - (R)i0, ty = g1 - (R)j0, tz = g2 - (R)k0;
  R acc = R(0);
  for (int di = 0; di < 2; ++di) {
    R wi = di == 0 ? R(1) - tx : tx;
    int ii = std::min(std::max(i0 + di, 0), d.n0 - 1);
    for (int dj = 0; dj < 2; ++dj) {
      R wj = dj == 0 ? R(1) - ty : ty;
      int jj = std::min(std::max(j0 + dj, 0), d.n1 - 1);
      for (int dk = 0; dk < 2; ++dk) {
        R wk = dk == 0 ? R(1) - tz : tz;
        int kk = std::min(std::max(k0 + dk, 0), d.n2 - 1);
        acc += wi * wj * wk * f[d.at(ii, jj, kk)];
      }
    }
  }
  return acc;
}

// ---------------------------------------------------------------------------
// particle sort (no reference counterpart: the reference never reorders).
// key = (i*ny + j)*nz + k of the cell floor(x/dx), computed in binary32 with an
// IEEE division and clamped to the grid; stable counting sort.
// ---------------------------------------------------------------------------
inline int32_t cell_key(float x, float y, float z, float dx, int nx, int ny, int nz) {
  int i = (int)std::floor(x / dx), j = (int)std::floor(y / dx), k = (int)std::floor(z / dx);
  i = std::min(std::max(i, 0), nx - 1);
  j = std::min(std::max(j, 0), ny - 1);
  k = std::min(std::max(k, 0), nz - 1);
  return (int32_t)(((int64_t)i * ny + j) * nz + k);
}

inline void sort_by_cell(int64_t n, const float* pos /*n*3*/, float dx, int nx, int ny, int nz,
                         int32_t* keys, int32_t* perm, int32_t* cell_start /*ncell+1*/) {
  const int64_t nc = (int64_t)nx * ny * nz;
  std::vector<int64_t> cnt(nc + 1, 0);
  for (int64_t p = 0; p < n; ++p) {
    keys[p] = cell_key(pos[3 * p], pos[3 * p + 1], pos[3 * p + 2], dx, nx, ny, nz);
    cnt[keys[p] + 1]++;
  }
  for (int64_t c = 0; c < nc; ++c) cnt[c + 1] += cnt[c];
  for (int64_t c = 0; c <= nc; ++c) cell_start[c] = (int32_t)cnt[c];
  for (int64_t p = 0; p < n; ++p) perm[cnt[keys[p]]++] = (int32_t)p;
}

// ---------------------------------------------------------------------------
// P2G: pfflip/kernels.py:100-158 (p2g_face) and :161-209 (p2g_cell).
// Accumulation is per particle in index order.  With nthr > 1 the particles are
// split into nthr contiguous chunks, each accumulated into a private grid, and
// the private grids are summed in chunk order (deterministic for a given nthr).
// ---------------------------------------------------------------------------
template <class R> struct P2GArgs {
  int64_t n;
  const R *px, *pv, *pmass, *prad;
  const int32_t* pstate;
  int nx, ny, nz;
  R dx;
};

template <class R>
inline void p2g_face_one(const P2GArgs<R>& a, int64_t p, int axis, R* mass, R* mom, Dims d) {
  if (a.pstate[p] != 0) return;
  const R* xp = a.px + 3 * p;
  R mp = a.pmass[p], rp = a.prad[p];
  R up = a.pv[3 * p + axis];
  R r2 = rp * rp;
  R Rr = rp / a.dx;
  R cx = xp[0] / a.dx - face_off<R>(axis, 0);
  R cy = xp[1] / a.dx - face_off<R>(axis, 1);
  R cz = xp[2] / a.dx - face_off<R>(axis, 2);
  int ilo = std::max((int)std::floor(cx - Rr) + 1, 0), ihi = std::min((int)std::floor(cx + Rr), d.n0 - 1);
  int jlo = std::max((int)std::floor(cy - Rr) + 1, 0), jhi = std::min((int)std::floor(cy + Rr), d.n1 - 1);
  int klo = std::max((int)std::floor(cz - Rr) + 1, 0), khi = std::min((int)std::floor(cz + Rr), d.n2 - 1);
  for (int i = ilo; i <= ihi; ++i) {
    R fx = ((R)i + face_off<R>(axis, 0)) * a.dx - xp[0];
    for (int j = jlo; j <= jhi; ++j) {
      R fy = ((R)j + face_off<R>(axis, 1)) * a.dx - xp[1];
      for (int k = klo; k <= khi; ++k) {
        R fz = ((R)k + face_off<R>(axis, 2)) * a.dx - xp[2];
        R d2 = fx * fx + fy * fy + fz * fz;
        R w = splat_weight(d2, r2);
        if (w > R(0)) {
          int64_t id = d.at(i, j, k);
          mass[id] += w * mp;
          mom[id] += w * mp * up;
        }
      }
    }
  }
}

template <class R>
inline void p2g_cell_one(const P2GArgs<R>& a, int64_t p, R* cmass, R* cwsum, Dims d) {
  if (a.pstate[p] != 0) return;
  const R* xp = a.px + 3 * p;
  R mp = a.pmass[p], rp = a.prad[p];
  R r2 = rp * rp;
  R Rr = rp / a.dx;
  R cx = xp[0] / a.dx - R(0.5), cy = xp[1] / a.dx - R(0.5), cz = xp[2] / a.dx - R(0.5);
  int ilo = std::max((int)std::floor(cx - Rr) + 1, 0), ihi = std::min((int)std::floor(cx + Rr), d.n0 - 1);
  int jlo = std::max((int)std::floor(cy - Rr) + 1, 0), jhi = std::min((int)std::floor(cy + Rr), d.n1 - 1);
  int klo = std::max((int)std::floor(cz - Rr) + 1, 0), khi = std::min((int)std::floor(cz + Rr), d.n2 - 1);
  for (int i = ilo; i <= ihi; ++i) {
    R fx = ((R)i + R(0.5)) * a.dx - xp[0];
    for (int j = jlo; j <= jhi; ++j) {
      R fy = ((R)j + R(0.5)) * a.dx - xp[1];
      for (int k = klo; k <= khi; ++k) {
        R fz = ((R)k + R(0.5)) * a.dx - xp[2];
        R d2 = fx * fx + fy * fy + fz * fz;
        R w = splat_weight(d2, r2);
        if (w > R(0)) {
          int64_t id = d.at(i, j, k);
          cmass[id] += w * mp;
          cwsum[id] += w;
        }
      }
    }
  }
}

// grids: mass[3], mom[3], cell_mass, cell_wsum (zeroed here, pfflip/sim.py:205-211)
template <class R>
inline void p2g(const P2GArgs<R>& a, R* mass[3], R* mom[3], R* cmass, R* cwsum, int nthr) {
  Dims fd[3] = {face_dims(a.nx, a.ny, a.nz, 0), face_dims(a.nx, a.ny, a.nz, 1),
                face_dims(a.nx, a.ny, a.nz, 2)};
  Dims cd{a.nx, a.ny, a.nz};
  int64_t sz[8] = {fd[0].size(), fd[1].size(), fd[2].size(), fd[0].size(),
                   fd[1].size(), fd[2].size(), cd.size(), cd.size()};
  R* out[8] = {mass[0], mass[1], mass[2], mom[0], mom[1], mom[2], cmass, cwsum};
  for (int g = 0; g < 8; ++g) std::memset(out[g], 0, sizeof(R) * sz[g]);
  if (nthr <= 1) {
    for (int64_t p = 0; p < a.n; ++p) {
      for (int ax = 0; ax < 3; ++ax) p2g_face_one(a, p, ax, mass[ax], mom[ax], fd[ax]);
      p2g_cell_one(a, p, cmass, cwsum, cd);
    }
    return;
  }
  // deterministic chunked parallel version: private grids per chunk
  std::vector<std::vector<R>> priv((size_t)nthr);
  int64_t tot = 0;
  for (int g = 0; g < 8; ++g) tot += sz[g];
#pragma omp parallel for num_threads(nthr) schedule(static, 1)
  for (int t = 0; t < nthr; ++t) {
    priv[t].assign((size_t)tot, R(0));
    R* base = priv[t].data();
    R* g8[8];
    int64_t off = 0;
    for (int g = 0; g < 8; ++g) { g8[g] = base + off; off += sz[g]; }
    int64_t p0 = a.n * t / nthr, p1 = a.n * (t + 1) / nthr;
    for (int64_t p = p0; p < p1; ++p) {
      for (int ax = 0; ax < 3; ++ax) p2g_face_one(a, p, ax, g8[ax], g8[3 + ax], fd[ax]);
      p2g_cell_one(a, p, g8[6], g8[7], cd);
    }
  }
  int64_t off = 0;
  for (int g = 0; g < 8; ++g) {
    R* dst = out[g];
#pragma omp parallel for num_threads(nthr) schedule(static)
    for (int64_t e = 0; e < sz[g]; ++e) {
      R s = R(0);
      for (int t = 0; t < nthr; ++t) s += priv[t][off + e];
      dst[e] = s;
    }
    off += sz[g];
  }
}

// pfflip/kernels.py:212-228
template <class R>
inline void face_velocity_from_momentum(const R* mass, const R* mom, R* vel, int32_t* valid, int64_t n,
                                        R mass_eps) {
#pragma omp parallel for
  for (int64_t e = 0; e < n; ++e) {
    R m = mass[e];
    if (m > mass_eps) { vel[e] = mom[e] / m; valid[e] = 1; }
    else { vel[e] = R(0); valid[e] = 0; }
  }
}

// pfflip/kernels.py:234-241 phase_field, eq. (7)
template <class R> inline R phase_field(R rho_raw, R rho_min, R alpha_phi, R rho_0l) {
  if (rho_raw < rho_min) return R(0);
  return std::min(std::sqrt(std::max(rho_raw - rho_min, R(0)) / (alpha_phi * rho_0l)), R(1));
}

// pfflip/kernels.py:244-255
template <class R>
inline void cell_phase(const R* cmass, R* phi, int32_t* is_liq, int64_t n, R rho_min, R alpha_phi, R rho_0l) {
#pragma omp parallel for
  for (int64_t e = 0; e < n; ++e) {
    R f = phase_field(cmass[e], rho_min, alpha_phi, rho_0l);
    phi[e] = f;
    is_liq[e] = f >= R(0.5) ? 1 : 0;
  }
}

// pfflip/kernels.py:258-311
template <class R>
inline void face_beta(const R* mass, const int32_t* is_liq, R* phi_face, R* beta, int nx, int ny, int nz, int axis,
                      R rho_min, R alpha_phi, R rho_0l, R rho_l, R rho_g) {
  Dims fd = face_dims(nx, ny, nz, axis), cd{nx, ny, nz};
#pragma omp parallel for collapse(2)
  for (int i = 0; i < fd.n0; ++i)
    for (int j = 0; j < fd.n1; ++j)
      for (int k = 0; k < fd.n2; ++k) {
        int im = i - (axis == 0), jm = j - (axis == 1), km = k - (axis == 2);
        bool lo_out = im < 0 || jm < 0 || km < 0;
        bool hi_out = i >= nx || j >= ny || k >= nz;
        int a = 0, b = 0;
        if (!lo_out) a = is_liq[cd.at(im, jm, km)];
        if (!hi_out) b = is_liq[cd.at(i, j, k)];
        if (lo_out) a = b;
        if (hi_out) b = a;
        int64_t e = fd.at(i, j, k);
        R f;
        if (a == 1 && b == 1) f = R(1);
        else if (a == 0 && b == 0) f = R(0);
        else f = phase_field(mass[e], rho_min, alpha_phi, rho_0l);
        phi_face[e] = f;
        R rho = (R(1) - f) * rho_g + f * rho_l;
        beta[e] = R(1) / rho;
      }
}

// pfflip/kernels.py:314-326
template <class R> inline void zero_solid_faces(R* beta, R* vel, int nx, int ny, int nz, int axis) {
  Dims fd = face_dims(nx, ny, nz, axis);
  int last = (axis == 0 ? fd.n0 : axis == 1 ? fd.n1 : fd.n2) - 1;
  for (int i = 0; i < fd.n0; ++i)
    for (int j = 0; j < fd.n1; ++j)
      for (int k = 0; k < fd.n2; ++k) {
        int n = axis == 0 ? i : axis == 1 ? j : k;
        if (n == 0 || n == last) { beta[fd.at(i, j, k)] = R(0); vel[fd.at(i, j, k)] = R(0); }
      }
}

// pfflip/kernels.py:601-627
template <class R>
inline void zero_solid_obstacle_faces(const int32_t* solid, R* beta, R* vel, int nx, int ny, int nz, int axis) {
  Dims fd = face_dims(nx, ny, nz, axis), cd{nx, ny, nz};
  for (int i = 0; i < fd.n0; ++i)
    for (int j = 0; j < fd.n1; ++j)
      for (int k = 0; k < fd.n2; ++k) {
        int im = i - (axis == 0), jm = j - (axis == 1), km = k - (axis == 2);
        int blocked = 0;
        if (i < nx && j < ny && k < nz) blocked = std::max(blocked, (int)solid[cd.at(i, j, k)]);
        if (im >= 0 && jm >= 0 && km >= 0) blocked = std::max(blocked, (int)solid[cd.at(im, jm, km)]);
        if (blocked == 1) { beta[fd.at(i, j, k)] = R(0); vel[fd.at(i, j, k)] = R(0); }
      }
}

// pfflip/kernels.py:332-335
template <class R> inline void add_gravity(R* vel, int64_t n, R g, R dt) {
  R gdt = g * dt;
  for (int64_t e = 0; e < n; ++e) vel[e] += gdt;
}

// pfflip/kernels.py:338-363
template <class R>
inline void build_rhs(const R* u, const R* v, const R* w, const R* cwsum, R* b, int nx, int ny, int nz, R dx, R dt,
                      R rho_0, R k_div) {
  Dims cd{nx, ny, nz}, fu = face_dims(nx, ny, nz, 0), fv = face_dims(nx, ny, nz, 1), fw = face_dims(nx, ny, nz, 2);
#pragma omp parallel for collapse(2)
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        R du = (u[fu.at(i + 1, j, k)] - u[fu.at(i, j, k)]) + (v[fv.at(i, j + 1, k)] - v[fv.at(i, j, k)]) +
               (w[fw.at(i, j, k + 1)] - w[fw.at(i, j, k)]);
        R rhs = -(dx / dt) * du;
        if (k_div > R(0)) {
          R excess = (cwsum[cd.at(i, j, k)] - rho_0) / rho_0;
          rhs -= dx * dx * k_div * std::max(excess, R(0)) / dt;
        }
        b[cd.at(i, j, k)] = rhs;
      }
}

// pfflip/kernels.py:366-387
template <class R>
inline void apply_pressure_gradient(const R* p, const R* beta, R* vel, int nx, int ny, int nz, int axis, R dx, R dt) {
  Dims fd = face_dims(nx, ny, nz, axis), cd{nx, ny, nz};
#pragma omp parallel for collapse(2)
  for (int i = 0; i < fd.n0; ++i)
    for (int j = 0; j < fd.n1; ++j)
      for (int k = 0; k < fd.n2; ++k) {
        int64_t e = fd.at(i, j, k);
        R bc = beta[e];
        if (bc == R(0)) continue;
        int im = i - (axis == 0), jm = j - (axis == 1), km = k - (axis == 2);
        if (im < 0 || jm < 0 || km < 0) continue;
        if (i >= nx || j >= ny || k >= nz) continue;
        vel[e] -= dt * bc * (p[cd.at(i, j, k)] - p[cd.at(im, jm, km)]) / dx;
      }
}

// pfflip/kernels.py:390-400 (returns max |div u| / dx)
template <class R> inline R divergence_norm(const R* u, const R* v, const R* w, int nx, int ny, int nz, R dx) {
  Dims fu = face_dims(nx, ny, nz, 0), fv = face_dims(nx, ny, nz, 1), fw = face_dims(nx, ny, nz, 2);
  R m = R(0);
#pragma omp parallel for collapse(2) reduction(max : m)
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        R d = (u[fu.at(i + 1, j, k)] - u[fu.at(i, j, k)]) + (v[fv.at(i, j + 1, k)] - v[fv.at(i, j, k)]) +
              (w[fw.at(i, j, k + 1)] - w[fw.at(i, j, k)]);
        m = std::max(m, std::fabs(d / dx));
      }
  return m;
}

// pfflip/kernels.py:406-425
template <class R>
inline void seed_liquid_velocity(const R* vel, const int32_t* is_liq, R* vel_l, int32_t* known, int nx, int ny,
                                 int nz, int axis) {
  Dims fd = face_dims(nx, ny, nz, axis), cd{nx, ny, nz};
#pragma omp parallel for collapse(2)
  for (int i = 0; i < fd.n0; ++i)
    for (int j = 0; j < fd.n1; ++j)
      for (int k = 0; k < fd.n2; ++k) {
        int im = i - (axis == 0), jm = j - (axis == 1), km = k - (axis == 2);
        int liq = 0;
        if (i < nx && j < ny && k < nz) liq = std::max(liq, (int)is_liq[cd.at(i, j, k)]);
        if (im >= 0 && jm >= 0 && km >= 0) liq = std::max(liq, (int)is_liq[cd.at(im, jm, km)]);
        int64_t e = fd.at(i, j, k);
        known[e] = liq;
        vel_l[e] = liq == 1 ? vel[e] : R(0);
      }
}

// pfflip/kernels.py:428-462
template <class R>
inline void extrapolate_sweep(const R* vel_l, const int32_t* known, R* vel_out, int32_t* known_out, Dims d) {
#pragma omp parallel for collapse(2)
  for (int i = 0; i < d.n0; ++i)
    for (int j = 0; j < d.n1; ++j)
      for (int k = 0; k < d.n2; ++k) {
        int64_t e = d.at(i, j, k);
        if (known[e] == 1) { vel_out[e] = vel_l[e]; known_out[e] = 1; continue; }
        R acc = R(0);
        int cnt = 0;
        for (int dd = 0; dd < 6; ++dd) {
          int ax = dd / 2, s = (dd % 2 == 0) ? -1 : 1;
          int ii = i + (ax == 0 ? s : 0), jj = j + (ax == 1 ? s : 0), kk = k + (ax == 2 ? s : 0);
          if (ii < 0 || jj < 0 || kk < 0 || ii >= d.n0 || jj >= d.n1 || kk >= d.n2) continue;
          int64_t q = d.at(ii, jj, kk);
          if (known[q] == 1) { acc += vel_l[q]; cnt += 1; }
        }
        if (cnt > 0) { vel_out[e] = acc / (R)cnt; known_out[e] = 1; }
        else { vel_out[e] = vel_l[e]; known_out[e] = 0; }
      }
}

// pfflip/kernels.py:468-496 (g2p) with :499-502 (field_difference) — du fields given.
template <class R>
inline void g2p(int64_t n, const R* px, R* pv, const int32_t* ptype, const int32_t* pstate, const R* u[3],
                const R* du[3], int nx, int ny, int nz, R dx, R a_liq, R a_air) {
  Dims fd[3] = {face_dims(nx, ny, nz, 0), face_dims(nx, ny, nz, 1), face_dims(nx, ny, nz, 2)};
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < n; ++p) {
    if (pstate[p] != 0) continue;
    const R* xp = px + 3 * p;
    R alpha = ptype[p] == 1 ? a_liq : a_air;
    for (int c = 0; c < 3; ++c) {
      R delta = sample_face(du[c], fd[c], xp, dx, c);
      R pic = sample_face(u[c], fd[c], xp, dx, c);
      pv[3 * p + c] = alpha * (pv[3 * p + c] + delta) + (R(1) - alpha) * pic;
    }
  }
}

// pfflip/kernels.py:508-549 advect_rk3 followed by :567-595 reflect_at_walls
template <class R>
inline void advect_reflect(int64_t n, R* px, R* pv, const int32_t* ptype, const int32_t* pstate, const R* u[3],
                           const R* ul[3], int nx, int ny, int nz, R dt, R dx, const R lo[3], const R hi[3]) {
  Dims fd[3] = {face_dims(nx, ny, nz, 0), face_dims(nx, ny, nz, 1), face_dims(nx, ny, nz, 2)};
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < n; ++p) {
    if (pstate[p] == 0) {
      R x[3] = {px[3 * p], px[3 * p + 1], px[3 * p + 2]};
      const R** f = ptype[p] == 1 ? ul : u;
      R k1[3], k2[3], k3[3], y[3];
      for (int c = 0; c < 3; ++c) k1[c] = sample_face(f[c], fd[c], x, dx, c);
      R h1 = R(0.5) * dt;
      for (int c = 0; c < 3; ++c) y[c] = x[c] + h1 * k1[c];
      for (int c = 0; c < 3; ++c) k2[c] = sample_face(f[c], fd[c], y, dx, c);
      R h2 = R(0.75) * dt;
      for (int c = 0; c < 3; ++c) y[c] = x[c] + h2 * k2[c];
      for (int c = 0; c < 3; ++c) k3[c] = sample_face(f[c], fd[c], y, dx, c);
      const R c1 = R(2.0) / R(9.0), c2 = R(3.0) / R(9.0), c3 = R(4.0) / R(9.0);
      for (int c = 0; c < 3; ++c) {
        R xn = x[c] + dt * (c1 * k1[c] + c2 * k2[c] + c3 * k3[c]);
        px[3 * p + c] = std::min(std::max(xn, lo[c]), hi[c]);
      }
    }
    if (pstate[p] == 2) continue;
    for (int c = 0; c < 3; ++c) {
      R xa = px[3 * p + c], va = pv[3 * p + c];
      if (xa <= lo[c]) { xa = lo[c]; va = std::max(va, R(0)); }
      else if (xa >= hi[c]) { xa = hi[c]; va = std::min(va, R(0)); }
      px[3 * p + c] = xa;
      pv[3 * p + c] = va;
    }
  }
}

// pfflip/kernels.py:630-679
template <class R>
inline void push_out_of_solids(int64_t n, R* px, R* pv, const int32_t* pstate, const int32_t* solid, int nx, int ny,
                               int nz, R dx) {
  Dims cd{nx, ny, nz};
  for (int64_t p = 0; p < n; ++p) {
    if (pstate[p] == 2) continue;
    R x[3] = {px[3 * p], px[3 * p + 1], px[3 * p + 2]};
    int i = std::min(std::max((int)(x[0] / dx), 0), nx - 1);
    int j = std::min(std::max((int)(x[1] / dx), 0), ny - 1);
    int k = std::min(std::max((int)(x[2] / dx), 0), nz - 1);
    if (solid[cd.at(i, j, k)] == 0) continue;
    R best = R(1.0e9);
    int bax = 0, bsg = 1;
    for (int d = 0; d < 6; ++d) {
      int ax = d / 2, sg = d % 2 == 0 ? -1 : 1;
      for (int t = 1; t < 8; ++t) {
        int ii = i + (ax == 0 ? sg * t : 0), jj = j + (ax == 1 ? sg * t : 0), kk = k + (ax == 2 ? sg * t : 0);
        if (ii < 0 || jj < 0 || kk < 0 || ii >= nx || jj >= ny || kk >= nz) break;
        if (solid[cd.at(ii, jj, kk)] == 0) {
          R dist = (R)t;
          if (dist < best) { best = dist; bax = ax; bsg = sg; }
          break;
        }
      }
    }
    if (best > R(1.0e8)) continue;
    R off = (best + R(0.5)) * dx * (R)bsg;
    px[3 * p + bax] = x[bax] + off;
    if ((R)bsg * pv[3 * p + bax] < R(0)) pv[3 * p + bax] = R(0);
  }
}

// pfflip/kernels.py:552-564 (CFL speed over FLIP particles)
template <class R> inline R particle_max_speed(int64_t n, const R* pv, const int32_t* pstate) {
  R m = R(0);
  for (int64_t p = 0; p < n; ++p) {
    if (pstate[p] != 0) continue;
    R s = std::sqrt(pv[3 * p] * pv[3 * p] + pv[3 * p + 1] * pv[3 * p + 1] + pv[3 * p + 2] * pv[3 * p + 2]);
    m = std::max(m, s);
  }
  return m;
}

// ===========================================================================
// Droplets: pfflip/droplets.py (escaped particles, droplet dynamics, spray)
// ===========================================================================
// The reference draws radii and spray emission from Warp's rand stream, which
// is not available here.  The library and this oracle share a documented
// stream instead: the PCG-RXS-M-XS 32-bit hash, seeded per particle id with
// hash(hash(seed) + id), uniforms ((s >> 8) + 0.5) * 2^-24, normals by
// Box-Muller, all in binary32.
inline uint32_t pcg_hash(uint32_t v) {
  const uint32_t s = v * 747796405u + 2891336453u;
  const uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}
struct DropRng {
  uint32_t s;
  DropRng(uint32_t seed, uint32_t id) : s(pcg_hash(pcg_hash(seed) + id)) {}
  float uniform() {
    s = pcg_hash(s);
    return ((float)(s >> 8) + 0.5f) * (1.0f / 16777216.0f);
  }
  float normal() {
    const float u1 = uniform(), u2 = uniform();
    return std::sqrt(-2.0f * std::log(u1)) * std::cos(6.28318530717958647692f * u2);
  }
};

// pfflip/droplets.py:41-64 sample_cell
template <class R> inline R sample_cell(const R* f, Dims d, const R x[3], R dx) {
  R g0 = x[0] / dx - R(0.5), g1 = x[1] / dx - R(0.5), g2 = x[2] / dx - R(0.5);
  int i0 = (int)std::floor(g0), j0 = (int)std::floor(g1), k0 = (int)std::floor(g2);
  R tx = g0 - (R)i0, ty = g1 - (R)j0, tz = g2 - (R)k0;
  R acc = R(0);
  for (int a = 0; a < 2; ++a) {
    R wa = a == 0 ? R(1) - tx : tx;
    int ii = std::min(std::max(i0 + a, 0), d.n0 - 1);
    for (int b = 0; b < 2; ++b) {
      R wb = b == 0 ? R(1) - ty : ty;
      int jj = std::min(std::max(j0 + b, 0), d.n1 - 1);
      for (int c = 0; c < 2; ++c) {
        R wc = c == 0 ? R(1) - tz : tz;
        int kk = std::min(std::max(k0 + c, 0), d.n2 - 1);
        acc += wa * wb * wc * f[d.at(ii, jj, kk)];
      }
    }
  }
  return acc;
}

// pfflip/droplets.py:67-106 classify_escaped (counters: emitted, bubbles, merged, spray)
template <class R>
inline void droplet_classify(int64_t n, const R* px, const int32_t* ptype, int32_t* pstate, R* pdrop_r,
                             const R* phi, int nx, int ny, int nz, R dx, R delta_phi, R mu, R sigma, R rmin,
                             R rmax, uint32_t seed, int32_t* counters) {
  Dims cd{nx, ny, nz};
  for (int64_t p = 0; p < n; ++p) {
    const int st = pstate[p];
    if (st == 2) continue;
    const R f = sample_cell(phi, cd, px + 3 * p, dx);
    if (st == 0) {
      if (ptype[p] == 1 && f < R(0.5) - delta_phi) {
        pstate[p] = 1;
        DropRng rng(seed, (uint32_t)p);
        const R r = std::exp(mu + sigma * (R)rng.normal());
        pdrop_r[p] = std::min(std::max(r, rmin), rmax);
        counters[0] += 1;
      } else if (ptype[p] == 0 && f > R(0.5) + delta_phi) {
        pstate[p] = 2;
        counters[1] += 1;
      }
    } else if (st == 1 && f > R(0.5) + delta_phi) {
      pstate[p] = 0;
      counters[2] += 1;
    }
  }
}

// pfflip/droplets.py:153-194 velocity_gradient_magnitude
template <class R>
inline void velocity_gradient(const R* u, const R* v, const R* w, R* out, int nx, int ny, int nz, R dx) {
  Dims fu = face_dims(nx, ny, nz, 0), fv = face_dims(nx, ny, nz, 1), fw = face_dims(nx, ny, nz, 2), cd{nx, ny, nz};
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        R dudx = (u[fu.at(i + 1, j, k)] - u[fu.at(i, j, k)]) / dx;
        R dvdy = (v[fv.at(i, j + 1, k)] - v[fv.at(i, j, k)]) / dx;
        R dwdz = (w[fw.at(i, j, k + 1)] - w[fw.at(i, j, k)]) / dx;
        R acc = dudx * dudx + dvdy * dvdy + dwdz * dwdz;
        int jm = std::max(j - 1, 0), jp = std::min(j + 1, ny - 1), km = std::max(k - 1, 0),
            kp = std::min(k + 1, nz - 1), im = std::max(i - 1, 0), ip = std::min(i + 1, nx - 1);
        R dudy = (R(0.5) * (u[fu.at(i, jp, k)] + u[fu.at(i + 1, jp, k)]) -
                  R(0.5) * (u[fu.at(i, jm, k)] + u[fu.at(i + 1, jm, k)])) / (R(2) * dx);
        R dudz = (R(0.5) * (u[fu.at(i, j, kp)] + u[fu.at(i + 1, j, kp)]) -
                  R(0.5) * (u[fu.at(i, j, km)] + u[fu.at(i + 1, j, km)])) / (R(2) * dx);
        R dvdx = (R(0.5) * (v[fv.at(ip, j, k)] + v[fv.at(ip, j + 1, k)]) -
                  R(0.5) * (v[fv.at(im, j, k)] + v[fv.at(im, j + 1, k)])) / (R(2) * dx);
        R dwdx = (R(0.5) * (w[fw.at(ip, j, k)] + w[fw.at(ip, j, k + 1)]) -
                  R(0.5) * (w[fw.at(im, j, k)] + w[fw.at(im, j, k + 1)])) / (R(2) * dx);
        acc += dudy * dudy + dudz * dudz + dvdx * dvdx + dwdx * dwdx;
        out[cd.at(i, j, k)] = std::sqrt(acc);
      }
}

// pfflip/droplets.py:112-150 emit_spray_in_shear
template <class R>
inline void spray_emit(int64_t n, const R* px, const int32_t* ptype, int32_t* pstate, R* pdrop_r, const R* phi,
                       const R* shear, int nx, int ny, int nz, R dx, R threshold, R rate, R mu, R sigma, R rmin,
                       R rmax, uint32_t seed, int32_t* counters) {
  Dims cd{nx, ny, nz};
  for (int64_t p = 0; p < n; ++p) {
    if (pstate[p] != 0 || ptype[p] != 1) continue;
    const R f = sample_cell(phi, cd, px + 3 * p, dx);
    if (f > R(0.9) || f < R(0.1)) continue;
    if (sample_cell(shear, cd, px + 3 * p, dx) < threshold) continue;
    DropRng rng(seed + 104729u, (uint32_t)p);
    if ((R)rng.uniform() > rate) continue;
    pstate[p] = 1;
    pdrop_r[p] = std::min(std::max((R)std::exp(mu + sigma * (R)rng.normal()), rmin), rmax);
    counters[3] += 1;
  }
}

// pfflip/droplets.py:197-279 drag_acceleration + advance_droplets
template <class R>
inline void droplet_advance(int64_t n, R* px, R* pv, int32_t* pstate, R* pdrop_r, const R* u[3], int nx, int ny,
                            int nz, R dt, R dx, const R grav[3], R rho_g, R rho_l, R cd, R evap_k, R rmin,
                            const R lo[3], const R hi[3], int max_sub) {
  Dims fd[3] = {face_dims(nx, ny, nz, 0), face_dims(nx, ny, nz, 1), face_dims(nx, ny, nz, 2)};
  for (int64_t p = 0; p < n; ++p) {
    if (pstate[p] != 1) continue;
    R x[3] = {px[3 * p], px[3 * p + 1], px[3 * p + 2]}, v[3] = {pv[3 * p], pv[3 * p + 1], pv[3 * p + 2]};
    R r = pdrop_r[p];
    const R speed = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + R(1e-8);
    const int nsub = std::min(std::max((int)(speed * dt / (R(0.5) * dx)) + 1, 1), max_sub);
    const R h = dt / (R)nsub;
    bool dead = false;
    for (int s = 0; s < nsub && !dead; ++s) {
      R ua[3];
      for (int c = 0; c < 3; ++c) ua[c] = sample_face(u[c], fd[c], x, dx, c);
      R vr[3] = {ua[0] - v[0], ua[1] - v[1], ua[2] - v[2]};
      R sr = std::sqrt(vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]);
      bool drag = sr > R(0) && r > R(0);
      R coef = drag ? (R(3) * rho_g * cd * sr / (R(8) * rho_l * r)) : R(0);
      for (int c = 0; c < 3; ++c) {
        R acc = grav[c] + (drag ? coef * vr[c] : R(0));
        v[c] = v[c] + h * acc;
        x[c] = x[c] + h * v[c];
      }
      if (evap_k > R(0) && r > R(0)) {
        R k1 = -evap_k / r;
        R rm = std::max(r + R(0.5) * h * k1, R(1e-9));
        r = r + h * (-evap_k / rm);
        if (r <= rmin) dead = true;
      }
    }
    if (!dead)
      for (int c = 0; c < 3; ++c)
        if (x[c] <= lo[c] || x[c] >= hi[c]) dead = true;
    if (dead) {
      pstate[p] = 2;
      continue;
    }
    pdrop_r[p] = r;
    for (int c = 0; c < 3; ++c) {
      pv[3 * p + c] = v[c];
      px[3 * p + c] = x[c];
    }
  }
}

// pfflip/droplets.py:309-353 rasterize_spray (accumulated in R here; the
// reference and the library add float16 values)
template <class R>
inline void spray_rasterize(int64_t n, const R* px, const int32_t* pstate, const R* pdrop_r, R* density, int sx,
                            int sy, int sz, R dxs) {
  Dims d{sx, sy, sz};
  std::fill(density, density + d.size(), R(0));
  for (int64_t p = 0; p < n; ++p) {
    if (pstate[p] != 1) continue;
    const R r = pdrop_r[p];
    const R vol = R(4.0 / 3.0) * R(3.14159265) * r * r * r;
    R g0 = px[3 * p] / dxs - R(0.5), g1 = px[3 * p + 1] / dxs - R(0.5), g2 = px[3 * p + 2] / dxs - R(0.5);
    int i0 = (int)std::floor(g0), j0 = (int)std::floor(g1), k0 = (int)std::floor(g2);
    R tx = g0 - (R)i0, ty = g1 - (R)j0, tz = g2 - (R)k0;
    const R cv = dxs * dxs * dxs;
    for (int a = 0; a < 2; ++a) {
      R wa = a == 0 ? R(1) - tx : tx;
      int ii = i0 + a;
      if (ii < 0 || ii >= sx) continue;
      for (int b = 0; b < 2; ++b) {
        R wb = b == 0 ? R(1) - ty : ty;
        int jj = j0 + b;
        if (jj < 0 || jj >= sy) continue;
        for (int c = 0; c < 2; ++c) {
          R wc = c == 0 ? R(1) - tz : tz;
          int kk = k0 + c;
          if (kk < 0 || kk >= sz) continue;
          density[d.at(ii, jj, kk)] += wa * wb * wc * vol / cv;
        }
      }
    }
  }
}

// ===========================================================================
// Poisson: pfflip/poisson.py
// ===========================================================================
template <class R> struct Level {
  int nx, ny, nz;
  std::vector<R> bx, by, bz, diag, p, b, r;
  void init(int x, int y, int z) {
    nx = x; ny = y; nz = z;
    int64_t n = (int64_t)x * y * z;
    bx.assign((size_t)(x + 1) * y * z, R(0));
    by.assign((size_t)x * (y + 1) * z, R(0));
    bz.assign((size_t)x * y * (z + 1), R(0));
    diag.assign(n, R(0)); p.assign(n, R(0)); b.assign(n, R(0)); r.assign(n, R(0));
  }
  int64_t size() const { return (int64_t)nx * ny * nz; }
};

// pfflip/poisson.py:41-51
template <class R> inline void compute_diag(Level<R>& L) {
  Dims c{L.nx, L.ny, L.nz}, fx = face_dims(L.nx, L.ny, L.nz, 0), fy = face_dims(L.nx, L.ny, L.nz, 1),
       fz = face_dims(L.nx, L.ny, L.nz, 2);
#pragma omp parallel for collapse(2)
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k)
        L.diag[c.at(i, j, k)] = L.bx[fx.at(i, j, k)] + L.bx[fx.at(i + 1, j, k)] + L.by[fy.at(i, j, k)] +
                                L.by[fy.at(i, j + 1, k)] + L.bz[fz.at(i, j, k)] + L.bz[fz.at(i, j, k + 1)];
}

// pfflip/poisson.py:54-75 _apply_row (g_stencil selects the form)
template <class R>
inline R apply_row(const R* p, const R* bx, const R* by, const R* bz, const R* diag, int nx, int ny, int nz, int i,
                   int j, int k) {
  Dims c{nx, ny, nz}, fx = face_dims(nx, ny, nz, 0), fy = face_dims(nx, ny, nz, 1), fz = face_dims(nx, ny, nz, 2);
  if (g_stencil == 1) {
    const R pc = p[c.at(i, j, k)];
    R s = bx[fx.at(i, j, k)] * (pc - p[c.at(std::max(i - 1, 0), j, k)]);
    s += bx[fx.at(i + 1, j, k)] * (pc - p[c.at(std::min(i + 1, nx - 1), j, k)]);
    s += by[fy.at(i, j, k)] * (pc - p[c.at(i, std::max(j - 1, 0), k)]);
    s += by[fy.at(i, j + 1, k)] * (pc - p[c.at(i, std::min(j + 1, ny - 1), k)]);
    s += bz[fz.at(i, j, k)] * (pc - p[c.at(i, j, std::max(k - 1, 0))]);
    s += bz[fz.at(i, j, k + 1)] * (pc - p[c.at(i, j, std::min(k + 1, nz - 1))]);
    return s;
  }
  R s = bx[fx.at(i, j, k)] * p[c.at(std::max(i - 1, 0), j, k)];
  s += bx[fx.at(i + 1, j, k)] * p[c.at(std::min(i + 1, nx - 1), j, k)];
  s += by[fy.at(i, j, k)] * p[c.at(i, std::max(j - 1, 0), k)];
  s += by[fy.at(i, j + 1, k)] * p[c.at(i, std::min(j + 1, ny - 1), k)];
  s += bz[fz.at(i, j, k)] * p[c.at(i, j, std::max(k - 1, 0))];
  s += bz[fz.at(i, j, k + 1)] * p[c.at(i, j, std::min(k + 1, nz - 1))];
  return diag[c.at(i, j, k)] * p[c.at(i, j, k)] - s;
}

// pfflip/poisson.py:78-88
template <class R>
inline void apply_A(const R* p, const R* bx, const R* by, const R* bz, const R* diag, R* out, int nx, int ny, int nz) {
  Dims c{nx, ny, nz};
#pragma omp parallel for collapse(2)
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) out[c.at(i, j, k)] = apply_row(p, bx, by, bz, diag, nx, ny, nz, i, j, k);
}

// pfflip/poisson.py:91-102
template <class R> inline void residual(Level<R>& L) {
  Dims c{L.nx, L.ny, L.nz};
#pragma omp parallel for collapse(2)
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k)
        L.r[c.at(i, j, k)] = L.b[c.at(i, j, k)] - apply_row(L.p.data(), L.bx.data(), L.by.data(), L.bz.data(),
                                                           L.diag.data(), L.nx, L.ny, L.nz, i, j, k);
}

// pfflip/poisson.py:105-126 (one colour; in place)
template <class R> inline void rbgs_sweep(Level<R>& L, int color, R omega) {
  Dims c{L.nx, L.ny, L.nz};
#pragma omp parallel for collapse(2)
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k) {
        if (((i + j + k) & 1) != color) continue;
        R d = L.diag[c.at(i, j, k)];
        if (d <= R(0)) continue;
        R res = L.b[c.at(i, j, k)] - apply_row(L.p.data(), L.bx.data(), L.by.data(), L.bz.data(), L.diag.data(),
                                               L.nx, L.ny, L.nz, i, j, k);
        L.p[c.at(i, j, k)] += omega * res / d;
      }
}

// pfflip/poisson.py:130-163
template <class R> inline void galerkin_coarsen_faces(const std::vector<R>& fine, Dims fd, std::vector<R>& coarse,
                                                       Dims cd, int axis) {
  for (int I = 0; I < cd.n0; ++I)
    for (int J = 0; J < cd.n1; ++J)
      for (int K = 0; K < cd.n2; ++K) {
        int i0 = 2 * I, j0 = 2 * J, k0 = 2 * K;
        R acc = R(0);
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) {
            int ii, jj, kk;
            if (axis == 0) { ii = i0; jj = j0 + a; kk = k0 + b; }
            else if (axis == 1) { ii = i0 + a; jj = j0; kk = k0 + b; }
            else { ii = i0 + a; jj = j0 + b; kk = k0; }
            if (ii < fd.n0 && jj < fd.n1 && kk < fd.n2) acc += fine[fd.at(ii, jj, kk)];
          }
        coarse[cd.at(I, J, K)] = acc;
      }
}

// pfflip/poisson.py:166-175
template <class R> inline void restrict_sum(const Level<R>& F, Level<R>& C) {
  Dims f{F.nx, F.ny, F.nz}, c{C.nx, C.ny, C.nz};
  for (int I = 0; I < C.nx; ++I)
    for (int J = 0; J < C.ny; ++J)
      for (int K = 0; K < C.nz; ++K) {
        R acc = R(0);
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b)
            for (int cc = 0; cc < 2; ++cc) acc += F.r[f.at(2 * I + a, 2 * J + b, 2 * K + cc)];
        C.b[c.at(I, J, K)] = acc;
      }
}

// pfflip/poisson.py:178-182
template <class R> inline void prolong_inject_add(const Level<R>& C, Level<R>& F) {
  Dims f{F.nx, F.ny, F.nz}, c{C.nx, C.ny, C.nz};
#pragma omp parallel for collapse(2)
  for (int i = 0; i < F.nx; ++i)
    for (int j = 0; j < F.ny; ++j)
      for (int k = 0; k < F.nz; ++k) F.p[f.at(i, j, k)] += C.p[c.at(i / 2, j / 2, k / 2)];
}

// Reductions accumulate in binary64 (the reference uses binary32 atomics whose
// order is unspecified; a binary64 sum is the order-independent ideal).
template <class R> inline double dot(const R* a, const R* b, int64_t n) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t e = 0; e < n; ++e) s += (double)a[e] * (double)b[e];
  return s;
}
template <class R> inline double sum(const R* a, int64_t n) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t e = 0; e < n; ++e) s += (double)a[e];
  return s;
}
template <class R> inline double max_abs(const R* a, int64_t n) {
  double m = 0.0;
#pragma omp parallel for reduction(max : m) schedule(static)
  for (int64_t e = 0; e < n; ++e) m = std::max(m, (double)std::fabs(a[e]));
  return m;
}
// pfflip/poisson.py:291-292 _remove_mean: shift by -(sum/ncells) in R
template <class R> inline void remove_mean(R* a, int64_t n) {
  R c = (R)(-(sum(a, n) / (double)n));
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < n; ++e) a[e] += c;
}

// pfflip/poisson.py:240-409 MGPCG
template <class R> struct MGPCG {
  std::vector<Level<R>> levels;
  R omega;
  int pre, post, coarsest;
  int64_t ncells;
  std::vector<R> rhs, res_v, z, q, Ap, r_prev;

  // pfflip/poisson.py:249-274
  void init(int nx, int ny, int nz, R om, int pre_, int post_, int coarsest_, int min_dim) {
    omega = om; pre = pre_; post = post_; coarsest = coarsest_;
    levels.clear();
    int r[3] = {nx, ny, nz};
    while (true) {
      levels.emplace_back();
      levels.back().init(r[0], r[1], r[2]);
      int mn = std::min(r[0], std::min(r[1], r[2]));
      if (mn / 2 < min_dim || (r[0] % 2) || (r[1] % 2) || (r[2] % 2)) break;
      r[0] /= 2; r[1] /= 2; r[2] /= 2;
    }
    ncells = (int64_t)nx * ny * nz;
    rhs.assign(ncells, R(0)); res_v.assign(ncells, R(0)); z.assign(ncells, R(0));
    q.assign(ncells, R(0)); Ap.assign(ncells, R(0)); r_prev.assign(ncells, R(0));
  }

  // pfflip/poisson.py:295-309
  void build_hierarchy(const R* bx, const R* by, const R* bz) {
    Level<R>& L0 = levels[0];
    std::copy(bx, bx + L0.bx.size(), L0.bx.begin());
    std::copy(by, by + L0.by.size(), L0.by.begin());
    std::copy(bz, bz + L0.bz.size(), L0.bz.begin());
    for (size_t lv = 0; lv < levels.size(); ++lv) {
      Level<R>& L = levels[lv];
      compute_diag(L);
      if (lv + 1 < levels.size()) {
        Level<R>& C = levels[lv + 1];
        galerkin_coarsen_faces(L.bx, face_dims(L.nx, L.ny, L.nz, 0), C.bx, face_dims(C.nx, C.ny, C.nz, 0), 0);
        galerkin_coarsen_faces(L.by, face_dims(L.nx, L.ny, L.nz, 1), C.by, face_dims(C.nx, C.ny, C.nz, 1), 1);
        galerkin_coarsen_faces(L.bz, face_dims(L.nx, L.ny, L.nz, 2), C.bz, face_dims(C.nx, C.ny, C.nz, 2), 2);
      }
    }
  }

  // pfflip/poisson.py:312-321
  void smooth(Level<R>& L, int nsweeps, bool reverse) {
    for (int s = 0; s < nsweeps; ++s) {
      rbgs_sweep(L, reverse ? 1 : 0, omega);
      rbgs_sweep(L, reverse ? 0 : 1, omega);
    }
  }

  // pfflip/poisson.py:323-343
  void vcycle(size_t lv) {
    Level<R>& L = levels[lv];
    if (lv == levels.size() - 1) {
      smooth(L, coarsest, false);
      remove_mean(L.p.data(), L.size());
      return;
    }
    smooth(L, pre, false);
    residual(L);
    Level<R>& C = levels[lv + 1];
    restrict_sum(L, C);
    std::fill(C.p.begin(), C.p.end(), R(0));
    vcycle(lv + 1);
    prolong_inject_add(C, L);
    smooth(L, post, true);
  }

  // pfflip/poisson.py:345-352
  void precondition(const R* r_in, R* z_out) {
    Level<R>& L0 = levels[0];
    std::copy(r_in, r_in + ncells, L0.b.begin());
    std::fill(L0.p.begin(), L0.p.end(), R(0));
    vcycle(0);
    std::copy(L0.p.begin(), L0.p.end(), z_out);
    remove_mean(z_out, ncells);
  }

  // pfflip/poisson.py:355-409; returns iterations, writes rel.
  int solve(const R* b, R* x, double tol, int max_iter, double* rel_out, std::vector<double>* history = nullptr) {
    Level<R>& L0 = levels[0];
    std::copy(b, b + ncells, rhs.begin());
    remove_mean(rhs.data(), ncells);
    double b_norm = max_abs(rhs.data(), ncells);
    if (b_norm == 0.0) {
      std::fill(x, x + ncells, R(0));
      *rel_out = 0.0;
      return 0;
    }
    std::fill(x, x + ncells, R(0));
    res_v = rhs;
    precondition(res_v.data(), z.data());
    q = z;
    double rz = dot(res_v.data(), z.data(), ncells);
    int it = 0;
    double rel = 1.0;
    for (it = 1; it <= max_iter; ++it) {
      apply_A(q.data(), L0.bx.data(), L0.by.data(), L0.bz.data(), L0.diag.data(), Ap.data(), L0.nx, L0.ny, L0.nz);
      double qAq = dot(q.data(), Ap.data(), ncells);
      if (qAq <= 0.0) break;
      double alpha = rz / qAq;
      R af = (R)alpha, naf = (R)(-alpha);
#pragma omp parallel for schedule(static)
      for (int64_t e = 0; e < ncells; ++e) {
        x[e] += af * q[e];
        r_prev[e] = res_v[e];
        res_v[e] += naf * Ap[e];
      }
      rel = max_abs(res_v.data(), ncells) / b_norm;
      if (history) history->push_back(rel);
      if (rel < tol) break;
      precondition(res_v.data(), z.data());
      double rz_new = dot(res_v.data(), z.data(), ncells);
      double num = rz_new - dot(r_prev.data(), z.data(), ncells);
      double beta = rz != 0.0 ? std::max(num / rz, 0.0) : 0.0;
      R bf = (R)beta;
#pragma omp parallel for schedule(static)
      for (int64_t e = 0; e < ncells; ++e) q[e] = z[e] + bf * q[e];
      rz = rz_new;
    }
    if (it > max_iter) it = max_iter;
    remove_mean(x, ncells);
    *rel_out = rel;
    return it;
  }
};

}  // namespace pfo
