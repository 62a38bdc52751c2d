// Grid-side streaming stages of the PF-FLIP step on sm_100a: face velocities,
// eq. (7) phase field and eq. (9) coefficients with the wall/solid zeroing
// fused into one pass; forces; divergence right-hand side; projection; the
// divergence norm; liquid velocity extrapolation (all sweeps of one face array
// in one shared-memory pass); CFL speed.
#include "pf_faces.cuh"

namespace pf {

struct PhaseArgs {
  FaceSpace s;
  const float* mass[3];
  const float* mom[3];
  const float* cmass;
  const int* solid;
  float eps, rho_min, alpha_phi, rho_0l, rho_l, rho_g;
  float* vel[3];
  int* valid[3];
  float* phi_cell;
  int* is_liq;
  float* phi_face[3];
  float* beta[3];
};

__global__ void __launch_bounds__(C3_NT) k_phase_beta(PhaseArgs a) {
  const FaceSpace& S = a.s;
  const int nx = S.nx, ny = S.ny, nz = S.nz;
  {
    long long f;
    int i, j, k;
    const int ax = locate(S, &f, &i, &j, &k);
    if (ax < 0) return;
    if (ax == 3) {  // cell: pfflip/kernels.py:244-255
      const float phi = phase_field(a.cmass[f], a.rho_min, a.alpha_phi, a.rho_0l);
      a.phi_cell[f] = phi;
      a.is_liq[f] = phi >= 0.5f ? 1 : 0;
      return;
    }
    // face velocity, pfflip/kernels.py:212-228
    const float m = a.mass[ax][f];
    const bool ok = m > a.eps;
    float u = ok ? a.mom[ax][f] / m : 0.f;
    if (a.valid[ax]) a.valid[ax][f] = ok ? 1 : 0;
    // face phase field and beta, pfflip/kernels.py:258-311
    const int im = i - (ax == 0), jm = j - (ax == 1), km = k - (ax == 2);
    const bool lo_out = im < 0 || jm < 0 || km < 0;
    const bool hi_out = i >= nx || j >= ny || k >= nz;
    int A = 0, B = 0;
    if (!lo_out)
      A = phase_field(a.cmass[((long long)im * ny + jm) * nz + km], a.rho_min, a.alpha_phi, a.rho_0l) >= 0.5f;
    if (!hi_out) B = phase_field(a.cmass[((long long)i * ny + j) * nz + k], a.rho_min, a.alpha_phi, a.rho_0l) >= 0.5f;
    if (lo_out) A = B;
    if (hi_out) B = A;
    float phi;
    if (A == 1 && B == 1) phi = 1.f;
    else if (A == 0 && B == 0) phi = 0.f;
    else phi = phase_field(m, a.rho_min, a.alpha_phi, a.rho_0l);
    if (a.phi_face[ax]) a.phi_face[ax][f] = phi;
    float beta = 1.f / ((1.f - phi) * a.rho_g + phi * a.rho_l);
    // walls and obstacles, pfflip/kernels.py:314-326 and :601-627
    if (boundary_face(ax, i, j, k, nx, ny, nz) || solid_face(a.solid, ax, i, j, k, nx, ny, nz)) {
      beta = 0.f;
      u = 0.f;
    }
    a.beta[ax][f] = beta;
    a.vel[ax][f] = u;
  }
}

struct ForceArgs {
  FaceSpace s;
  float* vel[3];
  float* vstar[3];
  const int* solid;
  float g[3];
  float dt;
};

// vel_star = vel; vel += g*dt; walls/obstacles zeroed (pfflip/sim.py:176-177, :270-285).
// FP_PZ planes per thread, their loads issued before any store.
constexpr int FP_PZ = 4;

__global__ void __launch_bounds__(C3_NT) k_save_force(const __grid_constant__ ForceArgs a) {
  const FaceSpace& S = a.s;
  const int planes = 3 * S.nx + 1;
  long long f[FP_PZ];
  int ax[FP_PZ], ii[FP_PZ], jj[FP_PZ], kk[FP_PZ];
  float v[FP_PZ];
#pragma unroll
  for (int p = 0; p < FP_PZ; ++p) {
    ax[p] = locate_plane(S, (int)blockIdx.z * FP_PZ + p, planes, &f[p], &ii[p], &jj[p], &kk[p]);
    v[p] = ax[p] >= 0 ? a.vel[ax[p]][f[p]] : 0.f;
  }
#pragma unroll
  for (int p = 0; p < FP_PZ; ++p) {
    const int x = ax[p];
    if (x < 0) continue;
    float u = v[p];
    if (a.vstar[x]) a.vstar[x][f[p]] = u;
    if (a.g[x] != 0.f) u += a.g[x] * a.dt;
    if (boundary_face(x, ii[p], jj[p], kk[p], S.nx, S.ny, S.nz) ||
        solid_face(a.solid, x, ii[p], jj[p], kk[p], S.nx, S.ny, S.nz))
      u = 0.f;
    a.vel[x][f[p]] = u;
  }
}

__device__ __forceinline__ float divergence(const float* u, const float* v, const float* w, int i, int j, int k,
                                            int nx, int ny, int nz) {
  const long long fu = ((long long)i * ny + j) * nz + k;
  const long long fv = ((long long)i * (ny + 1) + j) * nz + k;
  const long long fw = ((long long)i * ny + j) * (nz + 1) + k;
  return (u[fu + (long long)ny * nz] - u[fu]) + (v[fv + nz] - v[fv]) + (w[fw + 1] - w[fw]);
}

// pfflip/kernels.py:338-363
__global__ void __launch_bounds__(C3_NT) k_build_rhs(int nx, int ny, int nz, const float* __restrict__ u,
                                                    const float* __restrict__ v, const float* __restrict__ w,
                                                    const float* __restrict__ wsum, float* __restrict__ b, float dx,
                                                    float dt, float rho_0, float k_div) {
  const Cell3 cc = cell_here();
  if (cc.j >= ny || cc.k >= nz) return;
  {
    const int i = cc.i, j = cc.j, k = cc.k;
    const long long c = ((long long)i * ny + j) * nz + k;
    const float du = divergence(u, v, w, i, j, k, nx, ny, nz);
    float rhs = -(dx / dt) * du;
    if (k_div > 0.f) {
      const float excess = (wsum[c] - rho_0) / rho_0;
      rhs -= dx * dx * k_div * fmaxf(excess, 0.f) / dt;
    }
    b[c] = rhs;
  }
}

struct ProjArgs {
  FaceSpace s;
  const float* p;
  const float* beta[3];
  float* vel[3];
  float dx, dt;
};

// pfflip/kernels.py:366-387, FP_PZ planes per thread with their loads first
__global__ void __launch_bounds__(C3_NT) k_project(const __grid_constant__ ProjArgs a) {
  const FaceSpace& S = a.s;
  const int planes = 3 * S.nx + 1;
  long long f[FP_PZ];
  int ax[FP_PZ];
  float bc[FP_PZ], pi[FP_PZ], pm[FP_PZ], u[FP_PZ];
#pragma unroll
  for (int p = 0; p < FP_PZ; ++p) {
    int i, j, k;
    ax[p] = locate_plane(S, (int)blockIdx.z * FP_PZ + p, planes, &f[p], &i, &j, &k);
    bc[p] = 0.f;
    if (ax[p] < 0) continue;
    const int im = i - (ax[p] == 0), jm = j - (ax[p] == 1), km = k - (ax[p] == 2);
    if (im < 0 || jm < 0 || km < 0 || i >= S.nx || j >= S.ny || k >= S.nz) {  // wall faces: beta is 0
      ax[p] = -1;
      continue;
    }
    bc[p] = a.beta[ax[p]][f[p]];
    pi[p] = a.p[((long long)i * S.ny + j) * S.nz + k];
    pm[p] = a.p[((long long)im * S.ny + jm) * S.nz + km];
    u[p] = a.vel[ax[p]][f[p]];
  }
#pragma unroll
  for (int p = 0; p < FP_PZ; ++p) {
    if (ax[p] < 0 || bc[p] == 0.f) continue;
    a.vel[ax[p]][f[p]] = u[p] - a.dt * bc[p] * (pi[p] - pm[p]) / a.dx;
  }
}

// max |div u|/dx (pfflip/kernels.py:390-400)
__global__ void __launch_bounds__(256) k_max_div(int nx, int ny, int nz, const float* __restrict__ u,
                                                 const float* __restrict__ v, const float* __restrict__ w, float dx,
                                                 float* out) {
  __shared__ float sh[40];
  const Cell3 cc = cell_here();
  float m = 0.f;
  if (cc.j < ny && cc.k < nz) {
    const float d = divergence(u, v, w, cc.i, cc.j, cc.k, nx, ny, nz);
    const float q = fabsf(d / dx);
    m = isnan(q) ? INFINITY : q;
  }
  m = block_max<256>(m, sh);
  if (threadIdx.x == 0) atomic_max_nonneg(out, m);
}

// ---------------------------------------------------------------- extrapolation
// One face array (axis ax) per launch.  A CTA owns EX_TI x EX_TJ x EX_TK faces,
// loads them with an H-face halo (H = sweeps), seeds (pfflip/kernels.py:406-425)
// and runs H Jacobi sweeps (pfflip/kernels.py:428-462) in shared memory, then
// writes its tile.  Entries outside the face array are marked absent: they are
// never updated and never counted, as the reference skips out-of-range
// neighbours.  Errors from the missing outer halo travel one entry per sweep
// and never reach the tile.
constexpr int EX_TI = 4, EX_TJ = 8, EX_TK = 32, EX_NT = 256;
enum : unsigned char { EX_UNKNOWN = 0, EX_KNOWN = 1, EX_ABSENT = 2 };

template <int H>
__global__ void __launch_bounds__(EX_NT) k_extrapolate(int nx, int ny, int nz, int ax,
                                                       const float* __restrict__ vel, const int* __restrict__ is_liq,
                                                       float* __restrict__ vel_liq, int* __restrict__ known_out) {
  extern __shared__ __align__(16) unsigned char exsm[];
  const int n0 = nx + (ax == 0), n1 = ny + (ax == 1), n2 = nz + (ax == 2);
  constexpr int R0 = EX_TI + 2 * H, R1 = EX_TJ + 2 * H, R2 = EX_TK + 2 * H;
  constexpr int RN = R0 * R1 * R2;
  float* V0 = reinterpret_cast<float*>(exsm);
  float* V1 = V0 + RN;
  unsigned char* K0 = reinterpret_cast<unsigned char*>(V1 + RN);
  unsigned char* K1 = K0 + RN;
  const int i0 = blockIdx.z * EX_TI - H, j0 = blockIdx.y * EX_TJ - H, k0 = blockIdx.x * EX_TK - H;
  for (int e = threadIdx.x; e < RN; e += EX_NT) {
    const int r2 = e % R2, t = e / R2, r1 = t % R1, r0 = t / R1;
    const int i = i0 + r0, j = j0 + r1, k = k0 + r2;
    if (i < 0 || j < 0 || k < 0 || i >= n0 || j >= n1 || k >= n2) {
      V0[e] = 0.f;
      K0[e] = EX_ABSENT;
      continue;
    }
    const int im = i - (ax == 0), jm = j - (ax == 1), km = k - (ax == 2);
    int liq = 0;
    if (i < nx && j < ny && k < nz) liq = max(liq, is_liq[((long long)i * ny + j) * nz + k]);
    if (im >= 0 && jm >= 0 && km >= 0) liq = max(liq, is_liq[((long long)im * ny + jm) * nz + km]);
    V0[e] = (liq == 1) ? vel[((long long)i * n1 + j) * n2 + k] : 0.f;
    K0[e] = (liq == 1) ? EX_KNOWN : EX_UNKNOWN;
  }
  __syncthreads();
  float *Vi = V0, *Vo = V1;
  unsigned char *Ki = K0, *Ko = K1;
  const int st[3] = {R1 * R2, R2, 1};
  for (int s = 0; s < H; ++s) {
    for (int e = threadIdx.x; e < RN; e += EX_NT) {
      const unsigned char kn = Ki[e];
      if (kn != EX_UNKNOWN) {
        Vo[e] = Vi[e];
        Ko[e] = kn;
        continue;
      }
      const int r2 = e % R2, t = e / R2, r1 = t % R1, r0 = t / R1;
      const int rr[3] = {r0, r1, r2}, RR[3] = {R0, R1, R2};
      float acc = 0.f;
      int cnt = 0;
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        const int a = d >> 1, sg = (d & 1) ? 1 : -1;
        const int q = rr[a] + sg;
        if (q < 0 || q >= RR[a]) continue;
        const int nb = e + sg * st[a];
        if (Ki[nb] == EX_KNOWN) {
          acc += Vi[nb];
          cnt += 1;
        }
      }
      if (cnt > 0) {
        Vo[e] = acc / (float)cnt;
        Ko[e] = EX_KNOWN;
      } else {
        Vo[e] = Vi[e];
        Ko[e] = EX_UNKNOWN;
      }
    }
    __syncthreads();
    float* tv = Vi; Vi = Vo; Vo = tv;
    unsigned char* tk = Ki; Ki = Ko; Ko = tk;
  }
  for (int e = threadIdx.x; e < EX_TI * EX_TJ * EX_TK; e += EX_NT) {
    const int c2 = e % EX_TK, t = e / EX_TK, c1 = t % EX_TJ, c0 = t / EX_TJ;
    const int i = i0 + H + c0, j = j0 + H + c1, k = k0 + H + c2;
    if (i >= n0 || j >= n1 || k >= n2) continue;
    const int r = ((c0 + H) * R1 + (c1 + H)) * R2 + (c2 + H);
    const long long g = ((long long)i * n1 + j) * n2 + k;
    vel_liq[g] = Vi[r];
    if (known_out) known_out[g] = (Ki[r] == EX_KNOWN) ? 1 : 0;
  }
}

// ---------------------------------------------------------------- extrapolation by levels
// The same extrapolation, computed level by level in place.  A face becomes
// known at sweep s exactly when it was unknown and has a neighbour known
// after sweep s-1; from then on every sweep copies it.  So its final value is
// the mean, over its neighbours of level <= s-1, of their final values, and
// the faces set in pass s read only faces set in earlier passes.  The known
// arrays hold the level during the passes (kExNever = not reached) and 0/1
// at the end.  Sums run over the neighbours in the reference's order (-i, +i,
// -j, +j, -k, +k), so every value is the reference's.
constexpr int kExNever = 0x7fffffff;

struct ExLevelArgs {
  FaceSpace s;
  const float* vel[3];
  const int* is_liq;
  float* out[3];
  int* lv[3];
  int pass;  // 0: seed; 1..S: sweep; -1: levels -> 0/1 (S in `last`)
  int last;
};

__global__ void __launch_bounds__(C3_NT) k_ex_levels(ExLevelArgs a) {
  long long f;
  int i, j, k;
  const int ax = locate(a.s, &f, &i, &j, &k);
  if (ax < 0 || ax > 2) return;
  int* lv = a.lv[ax];
  if (a.pass == 0) {  // seed_liquid_velocity, pfflip/kernels.py:406-425
    const int nx = a.s.nx, ny = a.s.ny, nz = a.s.nz;
    const int im = i - (ax == 0), jm = j - (ax == 1), km = k - (ax == 2);
    int liq = 0;
    if (i < nx && j < ny && k < nz) liq = max(liq, a.is_liq[((long long)i * ny + j) * nz + k]);
    if (im >= 0 && jm >= 0 && km >= 0) liq = max(liq, a.is_liq[((long long)im * ny + jm) * nz + km]);
    lv[f] = liq == 1 ? 0 : kExNever;
    a.out[ax][f] = liq == 1 ? a.vel[ax][f] : 0.f;
    return;
  }
  if (a.pass < 0) {
    lv[f] = lv[f] <= a.last ? 1 : 0;
    return;
  }
  if (lv[f] != kExNever) return;
  const int n0 = a.s.nx + (ax == 0), n1 = a.s.ny + (ax == 1), n2 = a.s.nz + (ax == 2);
  const long long st[3] = {(long long)n1 * n2, n2, 1};
  const int id[3] = {i, j, k}, nn[3] = {n0, n1, n2};
  const float* out = a.out[ax];
  float acc = 0.f;
  int cnt = 0;
#pragma unroll
  for (int d = 0; d < 6; ++d) {  // extrapolate_sweep, pfflip/kernels.py:428-462
    const int ad = d >> 1, sg = (d & 1) ? 1 : -1;
    const int q = id[ad] + sg;
    if (q < 0 || q >= nn[ad]) continue;
    const long long g = f + sg * st[ad];
    if (lv[g] <= a.pass - 1) {
      acc += out[g];
      cnt += 1;
    }
  }
  if (cnt > 0) {
    a.out[ax][f] = acc / (float)cnt;
    lv[f] = a.pass;
  }
}

// CFL speed over particles with pstate == 0 (pfflip/kernels.py:552-564)
__global__ void __launch_bounds__(256) k_max_speed(long long n, const float4* __restrict__ pos,
                                                   const float4* __restrict__ vel, float* out) {
  __shared__ float sh[40];
  float m = 0.f;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int flags = __float_as_int(__ldg(&pos[p].w));
    if ((flags >> PF_PSTATE_SHIFT) & 3) continue;
    const float4 v = __ldg(vel + p);
    m = fmaxf(m, sqrtf(v.x * v.x + v.y * v.y + v.z * v.z));
  }
  m = block_max<256>(m, sh);
  if (threadIdx.x == 0) atomic_max_nonneg(out, m);
}

int ew_blocks(long long n) { return grid_for(n, 256, kNumSMs * 16); }

}  // namespace pf

using namespace pf;

extern "C" {

int pf_phase_beta(const pf_grid* g, const float* mass_x, const float* mass_y, const float* mass_z,
                  const float* mom_x, const float* mom_y, const float* mom_z, const float* cell_mass,
                  const int32_t* solid, float mass_eps, float rho_min, float alpha_phi, float rho_0l, float rho_l,
                  float rho_g, float* vel_x, float* vel_y, float* vel_z, int32_t* valid_x, int32_t* valid_y,
                  int32_t* valid_z, float* phi_cell, int32_t* is_liquid, float* phi_face_x, float* phi_face_y,
                  float* phi_face_z, float* beta_x, float* beta_y, float* beta_z, void* stream) {
  PF_REQUIRE(g && mass_x && mass_y && mass_z && mom_x && mom_y && mom_z && cell_mass && vel_x && vel_y && vel_z &&
                 phi_cell && is_liquid && beta_x && beta_y && beta_z,
             "null argument");
  PhaseArgs a;
  a.s = make_space(g->nx, g->ny, g->nz);
  a.mass[0] = mass_x; a.mass[1] = mass_y; a.mass[2] = mass_z;
  a.mom[0] = mom_x; a.mom[1] = mom_y; a.mom[2] = mom_z;
  a.cmass = cell_mass;
  a.solid = solid;
  a.eps = mass_eps; a.rho_min = rho_min; a.alpha_phi = alpha_phi; a.rho_0l = rho_0l;
  a.rho_l = rho_l; a.rho_g = rho_g;
  a.vel[0] = vel_x; a.vel[1] = vel_y; a.vel[2] = vel_z;
  a.valid[0] = valid_x; a.valid[1] = valid_y; a.valid[2] = valid_z;
  a.phi_cell = phi_cell; a.is_liq = is_liquid;
  a.phi_face[0] = phi_face_x; a.phi_face[1] = phi_face_y; a.phi_face[2] = phi_face_z;
  a.beta[0] = beta_x; a.beta[1] = beta_y; a.beta[2] = beta_z;
  k_phase_beta<<<grid_faces(g->nx, g->ny, g->nz, true), C3_NT, 0, S(stream)>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_save_and_force(const pf_grid* g, float* vel_x, float* vel_y, float* vel_z, float* vel_star_x,
                      float* vel_star_y, float* vel_star_z, const int32_t* solid, float gx, float gy, float gz,
                      float dt, void* stream) {
  PF_REQUIRE(g && vel_x && vel_y && vel_z, "null argument");
  ForceArgs a;
  a.s = make_space(g->nx, g->ny, g->nz);
  a.vel[0] = vel_x; a.vel[1] = vel_y; a.vel[2] = vel_z;
  a.vstar[0] = vel_star_x; a.vstar[1] = vel_star_y; a.vstar[2] = vel_star_z;
  a.solid = solid;
  a.g[0] = gx; a.g[1] = gy; a.g[2] = gz;
  a.dt = dt;
  k_save_force<<<grid_faces_multi(g->nx, g->ny, g->nz, false, FP_PZ), C3_NT, 0, S(stream)>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_build_rhs(const pf_grid* g, const float* vel_x, const float* vel_y, const float* vel_z,
                 const float* cell_wsum, float* b, float dt, float rho_0, float k_div, void* stream) {
  PF_REQUIRE(g && vel_x && vel_y && vel_z && b, "null argument");
  PF_REQUIRE(k_div <= 0.f || cell_wsum, "cell_wsum required when k_div > 0");
  const long long n = (long long)g->nx * g->ny * g->nz;
  (void)n;
  k_build_rhs<<<grid_cells(g->nx, g->ny, g->nz), C3_NT, 0, S(stream)>>>(g->nx, g->ny, g->nz, vel_x, vel_y, vel_z,
                                                                        cell_wsum, b, g->dx, dt, rho_0, k_div);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_project(const pf_grid* g, const float* p, const float* beta_x, const float* beta_y, const float* beta_z,
               float* vel_x, float* vel_y, float* vel_z, float dt, void* stream) {
  PF_REQUIRE(g && p && beta_x && beta_y && beta_z && vel_x && vel_y && vel_z, "null argument");
  ProjArgs a;
  a.s = make_space(g->nx, g->ny, g->nz);
  a.p = p;
  a.beta[0] = beta_x; a.beta[1] = beta_y; a.beta[2] = beta_z;
  a.vel[0] = vel_x; a.vel[1] = vel_y; a.vel[2] = vel_z;
  a.dx = g->dx;
  a.dt = dt;
  k_project<<<grid_faces_multi(g->nx, g->ny, g->nz, false, FP_PZ), C3_NT, 0, S(stream)>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_max_divergence(const pf_grid* g, const float* vel_x, const float* vel_y, const float* vel_z, float* out,
                      void* stream) {
  PF_REQUIRE(g && vel_x && vel_y && vel_z && out, "null argument");
  cudaStream_t s = S(stream);
  PF_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float), s));
  const long long n = (long long)g->nx * g->ny * g->nz;
  (void)n;
  k_max_div<<<grid_cells(g->nx, g->ny, g->nz), C3_NT, 0, s>>>(g->nx, g->ny, g->nz, vel_x, vel_y, vel_z, g->dx, out);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_extrapolate(const pf_grid* g, const float* vel_x, const float* vel_y, const float* vel_z,
                   const int32_t* is_liquid, int32_t sweeps, float* vel_liq_x, float* vel_liq_y, float* vel_liq_z,
                   int32_t* known_x, int32_t* known_y, int32_t* known_z, void* stream) {
  PF_REQUIRE(g && vel_x && vel_y && vel_z && is_liquid && vel_liq_x && vel_liq_y && vel_liq_z, "null argument");
  PF_REQUIRE(sweeps >= 0 && sweeps <= 4, "sweeps must be in [0, 4]");
  const float* vin[3] = {vel_x, vel_y, vel_z};
  float* vout[3] = {vel_liq_x, vel_liq_y, vel_liq_z};
  int* kout[3] = {known_x, known_y, known_z};
  if (known_x && known_y && known_z) {  // level passes, in place in vel_liq and known
    ExLevelArgs a;
    a.s = make_space(g->nx, g->ny, g->nz);
    for (int c = 0; c < 3; ++c) {
      a.vel[c] = vin[c];
      a.out[c] = vout[c];
      a.lv[c] = kout[c];
    }
    a.is_liq = is_liquid;
    a.last = sweeps;
    const dim3 grid = grid_faces(g->nx, g->ny, g->nz, false);
    for (int pass = 0; pass <= sweeps + 1; ++pass) {
      a.pass = pass <= sweeps ? pass : -1;
      k_ex_levels<<<grid, C3_NT, 0, S(stream)>>>(a);
      PF_LAUNCHED();
    }
    return PF_OK;
  }
  const int H = sweeps;
  const size_t rn = (size_t)(EX_TI + 2 * H) * (EX_TJ + 2 * H) * (EX_TK + 2 * H);
  const size_t smem = rn * (2 * sizeof(float) + 2);
  static int attr_done = 0;
  if (!attr_done) {
    PF_CUDA_TRY(cudaFuncSetAttribute(k_extrapolate<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    PF_CUDA_TRY(cudaFuncSetAttribute(k_extrapolate<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    PF_CUDA_TRY(cudaFuncSetAttribute(k_extrapolate<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    PF_CUDA_TRY(cudaFuncSetAttribute(k_extrapolate<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    PF_CUDA_TRY(cudaFuncSetAttribute(k_extrapolate<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    attr_done = 1;
  }
  for (int ax = 0; ax < 3; ++ax) {
    const int n0 = g->nx + (ax == 0), n1 = g->ny + (ax == 1), n2 = g->nz + (ax == 2);
    dim3 grid((n2 + EX_TK - 1) / EX_TK, (n1 + EX_TJ - 1) / EX_TJ, (n0 + EX_TI - 1) / EX_TI);
    cudaStream_t st = S(stream);
    switch (H) {
      case 0: k_extrapolate<0><<<grid, EX_NT, smem, st>>>(g->nx, g->ny, g->nz, ax, vin[ax], is_liquid, vout[ax], kout[ax]); break;
      case 1: k_extrapolate<1><<<grid, EX_NT, smem, st>>>(g->nx, g->ny, g->nz, ax, vin[ax], is_liquid, vout[ax], kout[ax]); break;
      case 2: k_extrapolate<2><<<grid, EX_NT, smem, st>>>(g->nx, g->ny, g->nz, ax, vin[ax], is_liquid, vout[ax], kout[ax]); break;
      case 3: k_extrapolate<3><<<grid, EX_NT, smem, st>>>(g->nx, g->ny, g->nz, ax, vin[ax], is_liquid, vout[ax], kout[ax]); break;
      default: k_extrapolate<4><<<grid, EX_NT, smem, st>>>(g->nx, g->ny, g->nz, ax, vin[ax], is_liquid, vout[ax], kout[ax]); break;
    }
    PF_LAUNCHED();
  }
  return PF_OK;
}

int pf_particle_max_speed(int64_t n, const float* pos4, const float* vel4, float* out, void* stream) {
  PF_REQUIRE(n >= 0 && pos4 && vel4 && out, "null argument");
  PF_REQUIRE(aligned16(pos4) && aligned16(vel4), "particle streams must be 16-byte aligned");
  cudaStream_t s = S(stream);
  PF_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float), s));
  if (n == 0) return PF_OK;
  k_max_speed<<<ew_blocks(n), 256, 0, s>>>(n, reinterpret_cast<const float4*>(pos4),
                                           reinterpret_cast<const float4*>(vel4), out);
  PF_LAUNCHED();
  return PF_OK;
}

}  // extern "C"
