// Reverse-mode (adjoint) kernels of one uniform PF-FLIP step on sm_100a.
//
// The reference step (pfflip/sim.py:168-202) is not differentiable; these
// kernels give the vector-Jacobian product of the step this library runs,
// stage by stage in reverse order:
//
//   k_adj_g2p_advect   wall reflection + clamp, Ralston RK3 (pfflip/kernels.py:
//                      508-549, :567-595) and the FLIP/PIC update (:468-502):
//                      per particle, the forward taps are recomputed and the
//                      adjoint is scattered onto the face grids (a P2G-shaped
//                      scatter), the particle adjoints are written
//   k_adj_ex_*         transpose of the seed + Jacobi extrapolation
//                      (pfflip/kernels.py:406-462)
//   k_adj_project      adjoint of u -= dt*beta*(p_i - p_{i-1})/dx
//                      (pfflip/kernels.py:366-387): pressure and beta adjoints
//   (solve)            lambda = A^+ (p_bar - mean): a second MG-PCG solve with
//                      the same operator, run by the caller through pf_mg_solve
//   k_adj_face_sources adjoint of the divergence right-hand side (:338-363),
//                      gravity and wall zeroing (:332-335, :314-326), the u*
//                      copy, beta = 1/rho(phi) with eq. (7) at mixed faces
//                      (:258-311) and u = P/m (:212-228), including the
//                      operator's beta sensitivity -(lam_i - lam_j)(p_i - p_j)
//   k_adj_p2g          adjoint of the eq. (6) splat (pfflip/kernels.py:100-
//                      209): a per-particle gather of the face-mass and
//                      momentum adjoints through the kernel weight and its
//                      gradient 6 t^2 (x_node - x_p) / r^2, t = 1 - d^2/r^2
//   k_adj_phase_cell   eq. (7) on cells, for losses on phi
//
// Discrete decisions (sort order, liquid tags, extrapolation masks, clamps,
// the valid-face test) are held fixed: the result is the derivative of the
// step almost everywhere, i.e. away from the clamp/max kinks.
#include "pf_faces.cuh"

namespace pf {

// ---------------------------------------------------------------- sampling
// Frame of face grid c at position x: the clamped lower/upper tap indices and
// upper weights, exactly as the forward G2P/RK3 kernel forms them.
struct TapFrame {
  int I[2], J[2], K[2];
  float t[3];
};

__device__ __forceinline__ void tap_frame(const float x[3], float inv_dx, int nx, int ny, int nz, int c,
                                          TapFrame& fr) {
  const int n[3] = {nx, ny, nz};
  int lo[3], hi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float q = x[d] * inv_dx;
    const float g = d == c ? q : q - 0.5f;
    const int i0 = (int)floorf(g);
    const int last = d == c ? n[d] : n[d] - 1;
    fr.t[d] = g - (float)i0;
    lo[d] = min(max(i0, 0), last);
    hi[d] = min(max(i0 + 1, 0), last);
  }
  fr.I[0] = lo[0]; fr.I[1] = hi[0];
  fr.J[0] = lo[1]; fr.J[1] = hi[1];
  fr.K[0] = lo[2]; fr.K[1] = hi[2];
}

// value of the trilinear sample (forward tap order) and its gradient in x
__device__ __forceinline__ float sample_grad(const float* __restrict__ f, int c, const TapFrame& fr, int ny, int nz,
                                            float inv_dx, float grad[3]) {
  const int n1 = ny + (c == 1), n2 = nz + (c == 2);
  const float wi[2] = {1.f - fr.t[0], fr.t[0]}, wj[2] = {1.f - fr.t[1], fr.t[1]}, wk[2] = {1.f - fr.t[2], fr.t[2]};
  const float s[2] = {-1.f, 1.f};
  float acc = 0.f, g0 = 0.f, g1 = 0.f, g2 = 0.f;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj) {
      const int row = (fr.I[di] * n1 + fr.J[dj]) * n2;
      const float wij = wi[di] * wj[dj];
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) {
        const float v = __ldg(f + row + fr.K[dk]);
        acc += wij * wk[dk] * v;
        g0 += s[di] * wj[dj] * wk[dk] * v;
        g1 += wi[di] * s[dj] * wk[dk] * v;
        g2 += wij * s[dk] * v;
      }
    }
  grad[0] = g0 * inv_dx;
  grad[1] = g1 * inv_dx;
  grad[2] = g2 * inv_dx;
  return acc;
}

// forward value of (f - fs) sampled tap by tap (the reference's interpolation of
// the difference field)
__device__ __forceinline__ float sample_diff(const float* __restrict__ f, const float* __restrict__ fs, int c,
                                            const TapFrame& fr, int ny, int nz) {
  const int n1 = ny + (c == 1), n2 = nz + (c == 2);
  const float wi[2] = {1.f - fr.t[0], fr.t[0]}, wj[2] = {1.f - fr.t[1], fr.t[1]}, wk[2] = {1.f - fr.t[2], fr.t[2]};
  float acc = 0.f;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj) {
      const int row = (fr.I[di] * n1 + fr.J[dj]) * n2;
      const float wij = wi[di] * wj[dj];
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) acc += wij * wk[dk] * (__ldg(f + row + fr.K[dk]) - __ldg(fs + row + fr.K[dk]));
    }
  return acc;
}

// adjoint of the sample: fb[tap] += w_tap * g
__device__ __forceinline__ void scatter_taps(float* __restrict__ fb, int c, const TapFrame& fr, int ny, int nz,
                                             float g) {
  if (g == 0.f) return;
  const int n1 = ny + (c == 1), n2 = nz + (c == 2);
  const float wi[2] = {1.f - fr.t[0], fr.t[0]}, wj[2] = {1.f - fr.t[1], fr.t[1]}, wk[2] = {1.f - fr.t[2], fr.t[2]};
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj) {
      const int row = (fr.I[di] * n1 + fr.J[dj]) * n2;
      const float wij = wi[di] * wj[dj] * g;
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) atomicAdd(fb + row + fr.K[dk], wij * wk[dk]);
    }
}

__device__ __forceinline__ void sample_vec(const float* const f[3], const float x[3], float inv_dx, int nx, int ny,
                                           int nz, float out[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    TapFrame fr;
    tap_frame(x, inv_dx, nx, ny, nz, c, fr);
    float gdummy[3];
    out[c] = sample_grad(f[c], c, fr, ny, nz, inv_dx, gdummy);
  }
}

// gx += sum_c g[c] * grad_x sample(f_c, y);  fb_c[taps of y] += w * g[c]
__device__ __forceinline__ void sample_vec_adjoint(const float* const f[3], float* const fb[3], const float y[3],
                                                   float inv_dx, int nx, int ny, int nz, const float g[3],
                                                   float gy[3]) {
  gy[0] = gy[1] = gy[2] = 0.f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    TapFrame fr;
    tap_frame(y, inv_dx, nx, ny, nz, c, fr);
    float gr[3];
    sample_grad(f[c], c, fr, ny, nz, inv_dx, gr);
    gy[0] += g[c] * gr[0];
    gy[1] += g[c] * gr[1];
    gy[2] += g[c] * gr[2];
    scatter_taps(fb[c], c, fr, ny, nz, g[c]);
  }
}

// ---------------------------------------------------------------- G2P + RK3 + reflection
struct AdjG2PArgs {
  long long n;
  int nx, ny, nz;
  float inv_dx, dt, a_liq, a_air;
  float lo[3], hi[3];
  const float4* pos;
  const float4* vel;
  const float4* gpos_in;
  const float4* gvel_in;
  float4* gpos_out;
  float4* gvel_out;
  const float* u[3];
  const float* us[3];
  const float* ul[3];
  float* gu[3];
  float* gus[3];
  float* gul[3];
  int do_g2p, do_advect;
};

__global__ void __launch_bounds__(128) k_adj_g2p_advect(AdjG2PArgs a) {
  long long c0, c1;  // a contiguous chunk of the sorted streams per warp: gathers and scatters stay local
  warp_chunk(a.n, c0, c1);
  for (long long p = c0 + (threadIdx.x & 31); p < c1; p += 32) {
    const float4 P = a.pos[p], V = a.vel[p];
    const float4 GP = a.gpos_in[p], GV = a.gvel_in[p];
    const int flags = __float_as_int(P.w);
    const int pstate = (flags >> PF_PSTATE_SHIFT) & 3;
    const bool liquid = (flags & PF_FLAG_LIQUID) != 0;
    const float alpha = liquid ? a.a_liq : a.a_air;
    const float x[3] = {P.x, P.y, P.z};
    float vp[3] = {V.x, V.y, V.z};
    // ---- forward recompute: G2P
    if (a.do_g2p && pstate == 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        TapFrame fr;
        tap_frame(x, a.inv_dx, a.nx, a.ny, a.nz, c, fr);
        const float delta = sample_diff(a.u[c], a.us[c], c, fr, a.ny, a.nz);
        float gdummy[3];
        const float pic = sample_grad(a.u[c], c, fr, a.ny, a.nz, a.inv_dx, gdummy);
        vp[c] = alpha * (vp[c] + delta) + (1.f - alpha) * pic;
      }
    }
    // ---- forward recompute: RK3 and clamp
    const bool rk = a.do_advect && pstate == 0;
    const float* F[3] = {liquid ? a.ul[0] : a.u[0], liquid ? a.ul[1] : a.u[1], liquid ? a.ul[2] : a.u[2]};
    float* FB[3] = {liquid ? a.gul[0] : a.gu[0], liquid ? a.gul[1] : a.gu[1], liquid ? a.gul[2] : a.gu[2]};
    const float h1 = 0.5f * a.dt, h2 = 0.75f * a.dt;
    const float c1 = 2.0f / 9.0f, c2 = 3.0f / 9.0f, c3 = 4.0f / 9.0f;
    float y2[3], y3[3], xe[3] = {x[0], x[1], x[2]};
    if (rk) {
      float k1[3], k2[3], k3[3];
      sample_vec(F, x, a.inv_dx, a.nx, a.ny, a.nz, k1);
#pragma unroll
      for (int c = 0; c < 3; ++c) y2[c] = x[c] + h1 * k1[c];
      sample_vec(F, y2, a.inv_dx, a.nx, a.ny, a.nz, k2);
#pragma unroll
      for (int c = 0; c < 3; ++c) y3[c] = x[c] + h2 * k2[c];
      sample_vec(F, y3, a.inv_dx, a.nx, a.ny, a.nz, k3);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float xn = x[c] + a.dt * (c1 * k1[c] + c2 * k2[c] + c3 * k3[c]);
        xe[c] = fminf(fmaxf(xn, a.lo[c]), a.hi[c]);
      }
    }
    // ---- reverse: wall reflection (a clamped component carries no position
    // adjoint; v = max(v,0) / min(v,0) passes the adjoint where it is active)
    float gx[3] = {GP.x, GP.y, GP.z}, gv[3] = {GV.x, GV.y, GV.z};
    if (a.do_advect && pstate != 2) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (xe[c] <= a.lo[c]) {
          gx[c] = 0.f;
          if (!(vp[c] > 0.f)) gv[c] = 0.f;
        } else if (xe[c] >= a.hi[c]) {
          gx[c] = 0.f;
          if (!(vp[c] < 0.f)) gv[c] = 0.f;
        }
      }
    }
    // ---- reverse: RK3 (gx is now the adjoint of the unclamped update).  An
    // air particle's first stage samples u at x, exactly as its G2P does: its
    // adjoint joins the G2P adjoint's u taps below (one scatter, one gradient)
    const bool merge_k1 = rk && a.do_g2p && !liquid;
    float gk1[3] = {0.f, 0.f, 0.f};
    if (rk) {
      float gk2[3], gk3[3], gy[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        gk1[c] = a.dt * c1 * gx[c];
        gk2[c] = a.dt * c2 * gx[c];
        gk3[c] = a.dt * c3 * gx[c];
      }
      sample_vec_adjoint(F, FB, y3, a.inv_dx, a.nx, a.ny, a.nz, gk3, gy);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        gx[c] += gy[c];
        gk2[c] += h2 * gy[c];
      }
      sample_vec_adjoint(F, FB, y2, a.inv_dx, a.nx, a.ny, a.nz, gk2, gy);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        gx[c] += gy[c];
        gk1[c] += h1 * gy[c];
      }
      if (!merge_k1) {
        sample_vec_adjoint(F, FB, x, a.inv_dx, a.nx, a.ny, a.nz, gk1, gy);
#pragma unroll
        for (int c = 0; c < 3; ++c) gx[c] += gy[c];
      }
    }
    // ---- reverse: G2P, v' = alpha v + I(u) - alpha I(u*)
    if (a.do_g2p && pstate == 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float g = gv[c];
        const float gu = merge_k1 ? g + gk1[c] : g;  // adjoint of I(u)(x)
        TapFrame fr;
        tap_frame(x, a.inv_dx, a.nx, a.ny, a.nz, c, fr);
        float gr_u[3], gr_s[3];
        sample_grad(a.u[c], c, fr, a.ny, a.nz, a.inv_dx, gr_u);
        sample_grad(a.us[c], c, fr, a.ny, a.nz, a.inv_dx, gr_s);
#pragma unroll
        for (int d = 0; d < 3; ++d) gx[d] += gu * gr_u[d] - alpha * g * gr_s[d];
        scatter_taps(a.gu[c], c, fr, a.ny, a.nz, gu);
        scatter_taps(a.gus[c], c, fr, a.ny, a.nz, -alpha * g);
        gv[c] = alpha * g;
      }
    }
    a.gpos_out[p] = make_float4(gx[0], gx[1], gx[2], 0.f);
    a.gvel_out[p] = make_float4(gv[0], gv[1], gv[2], 0.f);
  }
}

// ---------------------------------------------------------------- extrapolation transpose
// level[f] = the sweep at which face f becomes known: 0 for seeded faces
// (a liquid cell on either side), s for faces first reached by sweep s (the
// L1 distance to the nearest seeded face in the face array's index space),
// kLevelNever beyond the last sweep.
constexpr unsigned char kLevelNever = 255;

__device__ __forceinline__ void face_dims(const FaceSpace& S, int ax, int& n0, int& n1, int& n2) {
  n0 = S.nx + (ax == 0);
  n1 = S.ny + (ax == 1);
  n2 = S.nz + (ax == 2);
}

__global__ void __launch_bounds__(C3_NT) k_adj_ex_seed(FaceSpace S, const int* __restrict__ is_liq,
                                                       unsigned char* lvx, unsigned char* lvy, unsigned char* lvz) {
  long long f;
  int i, j, k;
  const int ax = locate(S, &f, &i, &j, &k);
  if (ax < 0 || ax > 2) return;
  const int nx = S.nx, ny = S.ny, nz = S.nz;
  const int im = i - (ax == 0), jm = j - (ax == 1), km = k - (ax == 2);
  int liq = 0;
  if (i < nx && j < ny && k < nz) liq = max(liq, is_liq[((long long)i * ny + j) * nz + k]);
  if (im >= 0 && jm >= 0 && km >= 0) liq = max(liq, is_liq[((long long)im * ny + jm) * nz + km]);
  unsigned char* lv = ax == 0 ? lvx : ax == 1 ? lvy : lvz;
  lv[f] = liq == 1 ? 0 : kLevelNever;
}

// one growth step: faces not yet known with a neighbour of level <= s-1 get s
__global__ void __launch_bounds__(C3_NT) k_adj_ex_grow(FaceSpace S, int s, const unsigned char* ix,
                                                       const unsigned char* iy, const unsigned char* iz,
                                                       unsigned char* ox, unsigned char* oy, unsigned char* oz) {
  long long f;
  int i, j, k;
  const int ax = locate(S, &f, &i, &j, &k);
  if (ax < 0 || ax > 2) return;
  const unsigned char* in = ax == 0 ? ix : ax == 1 ? iy : iz;
  unsigned char* out = ax == 0 ? ox : ax == 1 ? oy : oz;
  unsigned char l = in[f];
  if (l == kLevelNever) {
    int n0, n1, n2;
    face_dims(S, ax, n0, n1, n2);
    const long long st[3] = {(long long)n1 * n2, n2, 1};
    const int id[3] = {i, j, k}, nn[3] = {n0, n1, n2};
#pragma unroll
    for (int d = 0; d < 6; ++d) {
      const int a = d >> 1, sg = (d & 1) ? 1 : -1;
      const int q = id[a] + sg;
      if (q < 0 || q >= nn[a]) continue;
      if (in[f + sg * st[a]] <= s - 1) l = (unsigned char)s;
    }
  }
  out[f] = l;
}

// number of in-bounds neighbours of face (i,j,k) with level <= s-1
__device__ __forceinline__ int known_nbrs(const unsigned char* lv, long long f, int i, int j, int k, int n0, int n1,
                                          int n2, int s) {
  const long long st[3] = {(long long)n1 * n2, n2, 1};
  const int id[3] = {i, j, k}, nn[3] = {n0, n1, n2};
  int cnt = 0;
#pragma unroll
  for (int d = 0; d < 6; ++d) {
    const int a = d >> 1, sg = (d & 1) ? 1 : -1;
    const int q = id[a] + sg;
    if (q < 0 || q >= nn[a]) continue;
    cnt += lv[f + sg * st[a]] <= s - 1;
  }
  return cnt;
}

// reverse of sweep s: B[f] = (level f != s ? A[f] : 0)
//                           + (level f <= s-1 ? sum over neighbours g of level s of A[g]/cnt(g) : 0)
struct ExSweepArgs {
  FaceSpace S;
  int s;
  const unsigned char* lv[3];
  const float* A[3];
  float* B[3];
};

__global__ void __launch_bounds__(C3_NT) k_adj_ex_sweep(const __grid_constant__ ExSweepArgs a) {
  long long f;
  int i, j, k;
  const int ax = locate(a.S, &f, &i, &j, &k);
  if (ax < 0 || ax > 2) return;
  int n0, n1, n2;
  face_dims(a.S, ax, n0, n1, n2);
  const unsigned char* lv = a.lv[ax];
  const float* A = a.A[ax];
  const int s = a.s;
  const int l = lv[f];
  float acc = (l != s) ? A[f] : 0.f;
  if (l <= s - 1) {
    const long long st[3] = {(long long)n1 * n2, n2, 1};
    const int id[3] = {i, j, k}, nn[3] = {n0, n1, n2};
#pragma unroll
    for (int d = 0; d < 6; ++d) {
      const int ad = d >> 1, sg = (d & 1) ? 1 : -1;
      const int q = id[ad] + sg;
      if (q < 0 || q >= nn[ad]) continue;
      const long long g = f + sg * st[ad];
      if (lv[g] != s) continue;
      const int gi = ad == 0 ? q : i, gj = ad == 1 ? q : j, gk = ad == 2 ? q : k;
      const int cnt = known_nbrs(lv, g, gi, gj, gk, n0, n1, n2, s);
      acc += A[g] / (float)cnt;
    }
  }
  a.B[ax][f] = acc;
}

// seed: gvel[f] += (level f == 0) ? A[f] : 0
__global__ void __launch_bounds__(C3_NT) k_adj_ex_seed_add(FaceSpace S, const unsigned char* lvx,
                                                           const unsigned char* lvy, const unsigned char* lvz,
                                                           const float* ax_, const float* ay_, const float* az_,
                                                           float* gx, float* gy, float* gz) {
  long long f;
  int i, j, k;
  const int ax = locate(S, &f, &i, &j, &k);
  if (ax < 0 || ax > 2) return;
  const unsigned char* lv = ax == 0 ? lvx : ax == 1 ? lvy : lvz;
  const float* A = ax == 0 ? ax_ : ax == 1 ? ay_ : az_;
  float* G = ax == 0 ? gx : ax == 1 ? gy : gz;
  if (lv[f] == 0) G[f] += A[f];
}

// ---------------------------------------------------------------- projection adjoint
struct AdjProjArgs {
  FaceSpace s;
  const float* p;
  const float* beta[3];
  const float* gu[3];
  float* gp;
  float* gbeta[3];
  float dx, dt;
};

__global__ void __launch_bounds__(C3_NT) k_adj_project(AdjProjArgs a) {
  const FaceSpace& S = a.s;
  long long f;
  int i, j, k;
  const int ax = locate(S, &f, &i, &j, &k);
  if (ax < 0) return;
  const int nx = S.nx, ny = S.ny, nz = S.nz;
  if (ax < 3) {  // beta adjoint of u -= dt*beta*(p_i - p_{i-1})/dx
    float gb = 0.f;
    const float bc = a.beta[ax][f];
    const int im = i - (ax == 0), jm = j - (ax == 1), km = k - (ax == 2);
    if (bc != 0.f && im >= 0 && jm >= 0 && km >= 0 && i < nx && j < ny && k < nz) {
      const float pi = a.p[((long long)i * ny + j) * nz + k];
      const float pm = a.p[((long long)im * ny + jm) * nz + km];
      gb = -a.dt * (pi - pm) / a.dx * a.gu[ax][f];
    }
    a.gbeta[ax][f] = gb;
    return;
  }
  // pressure adjoint of cell (i,j,k): its lower face on each axis has it as
  // the upper cell (-), its upper face as the lower cell (+)
  const int n[3] = {nx, ny, nz}, id[3] = {i, j, k};
  float gp = 0.f;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int n1 = ny + (d == 1), n2 = nz + (d == 2);
    const long long lo = ((long long)i * n1 + j) * n2 + k;
    const long long up = lo + (d == 0 ? (long long)n1 * n2 : d == 1 ? (long long)n2 : 1LL);
    if (id[d] > 0) {  // lower face is interior
      const float bc = a.beta[d][lo];
      if (bc != 0.f) gp -= a.dt * bc / a.dx * a.gu[d][lo];
    }
    if (id[d] < n[d] - 1) {  // upper face is interior
      const float bc = a.beta[d][up];
      if (bc != 0.f) gp += a.dt * bc / a.dx * a.gu[d][up];
    }
  }
  a.gp[f] = gp;
}

// ---------------------------------------------------------------- face sources
struct AdjFaceArgs {
  FaceSpace s;
  const float* p;
  const float* lam;
  const float* beta[3];
  const float* mass[3];
  const float* mom[3];
  const int* is_liq;
  const float* gu[3];
  const float* gus[3];
  const float* gbeta[3];
  float* gmass[3];
  float* gmom[3];
  float eps, rho_min, alpha_phi, rho_0l, rho_l, rho_g, dx, dt;
};

// d/d rho of eq. (7) where it is smooth; 0 on the clamped pieces and at the
// square root's origin
__device__ __forceinline__ float phase_field_deriv(float rho, float rho_min, float alpha_phi, float rho_0l) {
  if (rho < rho_min) return 0.f;
  const float s = fmaxf(rho - rho_min, 0.f) / (alpha_phi * rho_0l);
  const float r = sqrtf(s);
  if (!(r > 0.f) || r >= 1.f) return 0.f;
  return 0.5f / (r * alpha_phi * rho_0l);
}

__global__ void __launch_bounds__(C3_NT) k_adj_face_sources(AdjFaceArgs a) {
  const FaceSpace& S = a.s;
  long long f;
  int i, j, k;
  const int ax = locate(S, &f, &i, &j, &k);
  if (ax < 0 || ax > 2) return;
  const int nx = S.nx, ny = S.ny, nz = S.nz;
  if (boundary_face(ax, i, j, k, nx, ny, nz)) {  // u and beta are zeroed there: no dependence
    a.gmass[ax][f] = 0.f;
    a.gmom[ax][f] = 0.f;
    return;
  }
  const long long up = ((long long)i * ny + j) * nz + k;
  const long long lo = up - (ax == 0 ? (long long)ny * nz : ax == 1 ? (long long)nz : 1LL);
  const float dlam = a.lam[up] - a.lam[lo];
  // beta: projection term + operator sensitivity -(lam_i - lam_j)(p_i - p_j)
  const float gb = a.gbeta[ax][f] - dlam * (a.p[up] - a.p[lo]);
  // u after gravity: its own adjoint + the RHS b = -(dx/dt) div u (b_bar = lam)
  const float gu1 = a.gu[ax][f] + (a.dx / a.dt) * dlam;
  // u before gravity = the saved u*
  const float gu0 = gu1 + a.gus[ax][f];
  const float m = a.mass[ax][f];
  float gm = 0.f, gq = 0.f;
  if (m > a.eps) {  // u = P/m
    const float u0 = a.mom[ax][f] / m;
    gq = gu0 / m;
    gm = -gu0 * u0 / m;
  }
  if (a.is_liq[up] != a.is_liq[lo]) {  // mixed face: phi = eq. (7) of the face mass
    const float bc = a.beta[ax][f];
    const float gphi = gb * (-(a.rho_l - a.rho_g) * bc * bc);
    gm += phase_field_deriv(m, a.rho_min, a.alpha_phi, a.rho_0l) * gphi;
  }
  a.gmass[ax][f] = gm;
  a.gmom[ax][f] = gq;
}

// ---------------------------------------------------------------- P2G adjoint (gather)
struct AdjP2GArgs {
  long long n;
  int nx, ny, nz;
  float dx, inv_dx, rho_l, rho_g, r;
  const float4* pos;
  const float4* vel;
  const float* gmass[3];
  const float* gmom[3];
  const float* gcell;
  float4* gpos;
  float4* gvel;
};

// one grid (face axis c, or cells for c = 3): window floor(x/dx - o - R) + 1 ..
// floor(x/dx - o + R), clamped (pfflip/kernels.py:100-209)
__device__ __forceinline__ void p2g_adjoint_grid(const AdjP2GArgs& a, int c, const float x[3], float mp, float vc,
                                                 float gx[3], float& gvc) {
  const int n[3] = {a.nx + (c == 0), a.ny + (c == 1), a.nz + (c == 2)};
  const float Rr = a.r * a.inv_dx, r2 = a.r * a.r, inv_r2 = 1.f / r2;
  int lo[3], hi[3];
  float off[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    off[d] = (c == d) ? 0.f : 0.5f;
    const float cc = x[d] * a.inv_dx - off[d];
    lo[d] = max((int)floorf(cc - Rr) + 1, 0);
    hi[d] = min((int)floorf(cc + Rr), n[d] - 1);
  }
  const float* GM = c < 3 ? a.gmass[c] : a.gcell;
  const float* GQ = c < 3 ? a.gmom[c] : nullptr;
  for (int i = lo[0]; i <= hi[0]; ++i) {
    const float fx = ((float)i + off[0]) * a.dx - x[0];
    for (int j = lo[1]; j <= hi[1]; ++j) {
      const float fy = ((float)j + off[1]) * a.dx - x[1];
      const long long row = ((long long)i * n[1] + j) * n[2];
      for (int k = lo[2]; k <= hi[2]; ++k) {
        const float fz = ((float)k + off[2]) * a.dx - x[2];
        const float d2 = fx * fx + fy * fy + fz * fz;
        const float t = 1.f - d2 * inv_r2;
        if (!(t > 0.f)) continue;
        const float gmn = __ldg(GM + row + k);
        float coef = gmn;
        if (GQ) {
          const float gq = __ldg(GQ + row + k);
          gvc += mp * t * t * t * gq;
          coef += vc * gq;
        }
        const float s = 6.f * mp * t * t * inv_r2 * coef;  // dW/dx_p = 6 t^2 (x_node - x_p) / r^2
        gx[0] += s * fx;
        gx[1] += s * fy;
        gx[2] += s * fz;
      }
    }
  }
}

__global__ void __launch_bounds__(128) k_adj_p2g(const __grid_constant__ AdjP2GArgs a) {
  long long c0, c1;  // a contiguous chunk of the sorted streams per warp: gathers stay local
  warp_chunk(a.n, c0, c1);
  for (long long p = c0 + (threadIdx.x & 31); p < c1; p += 32) {
    const float4 P = a.pos[p], V = a.vel[p];
    const int flags = __float_as_int(P.w);
    if (((flags >> PF_PSTATE_SHIFT) & 3) != 0) continue;
    const float mp = (flags & PF_FLAG_LIQUID) ? a.rho_l : a.rho_g;
    const float x[3] = {P.x, P.y, P.z}, v[3] = {V.x, V.y, V.z};
    float gx[3] = {0.f, 0.f, 0.f}, gv[3] = {0.f, 0.f, 0.f};
    if (a.gmass[0]) {
#pragma unroll 1
      for (int c = 0; c < 3; ++c) p2g_adjoint_grid(a, c, x, mp, v[c], gx, gv[c]);
    }
    if (a.gcell) {
      float unused = 0.f;
      p2g_adjoint_grid(a, 3, x, mp, 0.f, gx, unused);
    }
    float4 G = a.gpos[p], H = a.gvel[p];
    G.x += gx[0]; G.y += gx[1]; G.z += gx[2];
    H.x += gv[0]; H.y += gv[1]; H.z += gv[2];
    a.gpos[p] = G;
    a.gvel[p] = H;
  }
}

__global__ void k_adj_phase_cell(long long n, const float* __restrict__ cmass, const float* __restrict__ gphi,
                                 float rho_min, float alpha_phi, float rho_0l, float* __restrict__ gcell) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    gcell[e] = phase_field_deriv(cmass[e], rho_min, alpha_phi, rho_0l) * gphi[e];
}

__global__ void k_adj_unsort(long long n, const int* __restrict__ perm, const float4* __restrict__ gp_in,
                             const float4* __restrict__ gv_in, float4* __restrict__ gp_out,
                             float4* __restrict__ gv_out) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int q = perm[t];
    gp_out[q] = gp_in[t];
    gv_out[q] = gv_in[t];
  }
}

}  // namespace pf

using namespace pf;

extern "C" {

int pf_adj_g2p_advect(const pf_grid* g, int64_t n, const float* pos4, const float* vel4, const float* vel_x,
                      const float* vel_y, const float* vel_z, const float* vstar_x, const float* vstar_y,
                      const float* vstar_z, const float* vliq_x, const float* vliq_y, const float* vliq_z,
                      float alpha_liquid, float alpha_air, float dt, const float lo[3], const float hi[3],
                      int32_t do_g2p, int32_t do_advect, const float* gpos4_in, const float* gvel4_in,
                      float* gpos4_out, float* gvel4_out, float* gvel_x, float* gvel_y, float* gvel_z,
                      float* gvstar_x, float* gvstar_y, float* gvstar_z, float* gvliq_x, float* gvliq_y,
                      float* gvliq_z, void* stream) {
  PF_REQUIRE(g && pos4 && vel4 && vel_x && vel_y && vel_z && gpos4_in && gvel4_in && gpos4_out && gvel4_out,
             "null argument");
  PF_REQUIRE(gvel_x && gvel_y && gvel_z, "adjoint of the face velocity required");
  PF_REQUIRE(!do_g2p || (vstar_x && vstar_y && vstar_z && gvstar_x && gvstar_y && gvstar_z),
             "u* and its adjoint required for G2P");
  PF_REQUIRE(!do_advect || (vliq_x && vliq_y && vliq_z && gvliq_x && gvliq_y && gvliq_z && lo && hi),
             "extrapolated field, its adjoint and the bounds required for advection");
  PF_REQUIRE(aligned16(pos4) && aligned16(vel4) && aligned16(gpos4_in) && aligned16(gvel4_in) &&
                 aligned16(gpos4_out) && aligned16(gvel4_out),
             "particle streams must be 16-byte aligned");
  if (n <= 0) return PF_OK;
  AdjG2PArgs a;
  a.n = n;
  a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
  a.inv_dx = (float)(1.0 / (double)g->dx);
  a.dt = dt;
  a.a_liq = alpha_liquid; a.a_air = alpha_air;
  for (int c = 0; c < 3; ++c) {
    a.lo[c] = lo ? lo[c] : 0.f;
    a.hi[c] = hi ? hi[c] : 0.f;
  }
  a.pos = reinterpret_cast<const float4*>(pos4);
  a.vel = reinterpret_cast<const float4*>(vel4);
  a.gpos_in = reinterpret_cast<const float4*>(gpos4_in);
  a.gvel_in = reinterpret_cast<const float4*>(gvel4_in);
  a.gpos_out = reinterpret_cast<float4*>(gpos4_out);
  a.gvel_out = reinterpret_cast<float4*>(gvel4_out);
  a.u[0] = vel_x; a.u[1] = vel_y; a.u[2] = vel_z;
  a.us[0] = vstar_x; a.us[1] = vstar_y; a.us[2] = vstar_z;
  a.ul[0] = vliq_x; a.ul[1] = vliq_y; a.ul[2] = vliq_z;
  a.gu[0] = gvel_x; a.gu[1] = gvel_y; a.gu[2] = gvel_z;
  a.gus[0] = gvstar_x; a.gus[1] = gvstar_y; a.gus[2] = gvstar_z;
  a.gul[0] = gvliq_x; a.gul[1] = gvliq_y; a.gul[2] = gvliq_z;
  a.do_g2p = do_g2p;
  a.do_advect = do_advect;
  k_adj_g2p_advect<<<grid_for(n, 128, kNumSMs * 16), 128, 0, S(stream)>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_adj_extrapolate(const pf_grid* g, const int32_t* is_liquid, int32_t sweeps, float* gliq_x, float* gliq_y,
                       float* gliq_z, float* tmp_x, float* tmp_y, float* tmp_z, uint8_t* level_x, uint8_t* level_y,
                       uint8_t* level_z, uint8_t* level_tmp_x, uint8_t* level_tmp_y, uint8_t* level_tmp_z,
                       float* gvel_x, float* gvel_y, float* gvel_z, void* stream) {
  PF_REQUIRE(g && is_liquid && gliq_x && gliq_y && gliq_z && tmp_x && tmp_y && tmp_z && gvel_x && gvel_y && gvel_z,
             "null argument");
  PF_REQUIRE(level_x && level_y && level_z && level_tmp_x && level_tmp_y && level_tmp_z, "null level scratch");
  PF_REQUIRE(sweeps >= 0 && sweeps < 200, "sweeps must be in [0, 200)");
  cudaStream_t s = S(stream);
  const FaceSpace sp = make_space(g->nx, g->ny, g->nz);
  const dim3 grid = grid_faces(g->nx, g->ny, g->nz, false);
  // levels: seed, then one growth step per sweep (ping-pong)
  unsigned char* L[2][3] = {{level_x, level_y, level_z}, {level_tmp_x, level_tmp_y, level_tmp_z}};
  k_adj_ex_seed<<<grid, C3_NT, 0, s>>>(sp, is_liquid, L[0][0], L[0][1], L[0][2]);
  PF_LAUNCHED();
  int cur = 0;
  for (int sw = 1; sw <= sweeps; ++sw) {
    k_adj_ex_grow<<<grid, C3_NT, 0, s>>>(sp, sw, L[cur][0], L[cur][1], L[cur][2], L[1 - cur][0], L[1 - cur][1],
                                         L[1 - cur][2]);
    PF_LAUNCHED();
    cur = 1 - cur;
  }
  // reverse sweeps on the adjoint field (ping-pong with tmp)
  float* A[3] = {gliq_x, gliq_y, gliq_z};
  float* B[3] = {tmp_x, tmp_y, tmp_z};
  for (int sw = sweeps; sw >= 1; --sw) {
    ExSweepArgs ea;
    ea.S = sp;
    ea.s = sw;
    for (int c = 0; c < 3; ++c) {
      ea.lv[c] = L[cur][c];
      ea.A[c] = A[c];
      ea.B[c] = B[c];
    }
    k_adj_ex_sweep<<<grid, C3_NT, 0, s>>>(ea);
    PF_LAUNCHED();
    for (int c = 0; c < 3; ++c) {
      float* t = A[c];
      A[c] = B[c];
      B[c] = t;
    }
  }
  k_adj_ex_seed_add<<<grid, C3_NT, 0, s>>>(sp, L[cur][0], L[cur][1], L[cur][2], A[0], A[1], A[2], gvel_x, gvel_y,
                                           gvel_z);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_adj_project(const pf_grid* g, const float* p, const float* beta_x, const float* beta_y, const float* beta_z,
                   const float* gvel_x, const float* gvel_y, const float* gvel_z, float dt, float* gp,
                   float* gbeta_x, float* gbeta_y, float* gbeta_z, void* stream) {
  PF_REQUIRE(g && p && beta_x && beta_y && beta_z && gvel_x && gvel_y && gvel_z && gp && gbeta_x && gbeta_y &&
                 gbeta_z,
             "null argument");
  AdjProjArgs a;
  a.s = make_space(g->nx, g->ny, g->nz);
  a.p = p;
  a.beta[0] = beta_x; a.beta[1] = beta_y; a.beta[2] = beta_z;
  a.gu[0] = gvel_x; a.gu[1] = gvel_y; a.gu[2] = gvel_z;
  a.gp = gp;
  a.gbeta[0] = gbeta_x; a.gbeta[1] = gbeta_y; a.gbeta[2] = gbeta_z;
  a.dx = g->dx;
  a.dt = dt;
  k_adj_project<<<grid_faces(g->nx, g->ny, g->nz, true), C3_NT, 0, S(stream)>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_adj_face_sources(const pf_grid* g, const float* p, const float* lam, const float* beta_x, const float* beta_y,
                        const float* beta_z, const float* mass_x, const float* mass_y, const float* mass_z,
                        const float* mom_x, const float* mom_y, const float* mom_z, const int32_t* is_liquid,
                        float mass_eps, float rho_min, float alpha_phi, float rho_0l, float rho_l, float rho_g,
                        float dt, const float* gvel_x, const float* gvel_y, const float* gvel_z,
                        const float* gvstar_x, const float* gvstar_y, const float* gvstar_z, const float* gbeta_x,
                        const float* gbeta_y, const float* gbeta_z, float* gmass_x, float* gmass_y, float* gmass_z,
                        float* gmom_x, float* gmom_y, float* gmom_z, void* stream) {
  PF_REQUIRE(g && p && lam && beta_x && beta_y && beta_z && mass_x && mass_y && mass_z && mom_x && mom_y && mom_z &&
                 is_liquid,
             "null argument");
  PF_REQUIRE(gvel_x && gvel_y && gvel_z && gvstar_x && gvstar_y && gvstar_z && gbeta_x && gbeta_y && gbeta_z &&
                 gmass_x && gmass_y && gmass_z && gmom_x && gmom_y && gmom_z,
             "null adjoint argument");
  PF_REQUIRE(dt > 0.f, "dt must be positive");
  AdjFaceArgs a;
  a.s = make_space(g->nx, g->ny, g->nz);
  a.p = p;
  a.lam = lam;
  a.beta[0] = beta_x; a.beta[1] = beta_y; a.beta[2] = beta_z;
  a.mass[0] = mass_x; a.mass[1] = mass_y; a.mass[2] = mass_z;
  a.mom[0] = mom_x; a.mom[1] = mom_y; a.mom[2] = mom_z;
  a.is_liq = is_liquid;
  a.gu[0] = gvel_x; a.gu[1] = gvel_y; a.gu[2] = gvel_z;
  a.gus[0] = gvstar_x; a.gus[1] = gvstar_y; a.gus[2] = gvstar_z;
  a.gbeta[0] = gbeta_x; a.gbeta[1] = gbeta_y; a.gbeta[2] = gbeta_z;
  a.gmass[0] = gmass_x; a.gmass[1] = gmass_y; a.gmass[2] = gmass_z;
  a.gmom[0] = gmom_x; a.gmom[1] = gmom_y; a.gmom[2] = gmom_z;
  a.eps = mass_eps;
  a.rho_min = rho_min;
  a.alpha_phi = alpha_phi;
  a.rho_0l = rho_0l;
  a.rho_l = rho_l;
  a.rho_g = rho_g;
  a.dx = g->dx;
  a.dt = dt;
  k_adj_face_sources<<<grid_faces(g->nx, g->ny, g->nz, false), C3_NT, 0, S(stream)>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_adj_p2g(const pf_grid* g, int64_t n, const float* pos4, const float* vel4, float rho_l, float rho_g, float r_p,
               const float* gmass_x, const float* gmass_y, const float* gmass_z, const float* gmom_x,
               const float* gmom_y, const float* gmom_z, const float* gcell_mass, float* gpos4, float* gvel4,
               void* stream) {
  PF_REQUIRE(g && pos4 && vel4 && gpos4 && gvel4, "null argument");
  const bool faces = gmass_x || gmass_y || gmass_z || gmom_x || gmom_y || gmom_z;
  PF_REQUIRE(!faces || (gmass_x && gmass_y && gmass_z && gmom_x && gmom_y && gmom_z),
             "face adjoints must be given for all three axes, or none");
  PF_REQUIRE(r_p > 0.f && r_p <= g->dx, "support radius must be in (0, dx]");
  PF_REQUIRE(aligned16(pos4) && aligned16(vel4) && aligned16(gpos4) && aligned16(gvel4),
             "particle streams must be 16-byte aligned");
  if (n <= 0 || (!faces && !gcell_mass)) return PF_OK;
  AdjP2GArgs a;
  a.n = n;
  a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
  a.dx = g->dx;
  a.inv_dx = (float)(1.0 / (double)g->dx);
  a.rho_l = rho_l;
  a.rho_g = rho_g;
  a.r = r_p;
  a.pos = reinterpret_cast<const float4*>(pos4);
  a.vel = reinterpret_cast<const float4*>(vel4);
  a.gmass[0] = gmass_x; a.gmass[1] = gmass_y; a.gmass[2] = gmass_z;
  a.gmom[0] = gmom_x; a.gmom[1] = gmom_y; a.gmom[2] = gmom_z;
  a.gcell = gcell_mass;
  a.gpos = reinterpret_cast<float4*>(gpos4);
  a.gvel = reinterpret_cast<float4*>(gvel4);
  k_adj_p2g<<<grid_for(n, 128, kNumSMs * 16), 128, 0, S(stream)>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_adj_phase_cell(const pf_grid* g, const float* cell_mass, const float* gphi, float rho_min, float alpha_phi,
                      float rho_0l, float* gcell_mass, void* stream) {
  PF_REQUIRE(g && cell_mass && gphi && gcell_mass, "null argument");
  const long long n = (long long)g->nx * g->ny * g->nz;
  k_adj_phase_cell<<<grid_for(n, 256, kNumSMs * 8), 256, 0, S(stream)>>>(n, cell_mass, gphi, rho_min, alpha_phi,
                                                                          rho_0l, gcell_mass);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_adj_unsort(int64_t n, const int32_t* perm, const float* gpos4_sorted, const float* gvel4_sorted,
                  float* gpos4_out, float* gvel4_out, void* stream) {
  PF_REQUIRE(n >= 0 && perm && gpos4_sorted && gvel4_sorted && gpos4_out && gvel4_out, "null argument");
  PF_REQUIRE(gpos4_sorted != gpos4_out && gvel4_sorted != gvel4_out, "output must not alias the input");
  PF_REQUIRE(aligned16(gpos4_sorted) && aligned16(gvel4_sorted) && aligned16(gpos4_out) && aligned16(gvel4_out),
             "particle streams must be 16-byte aligned");
  if (n == 0) return PF_OK;
  k_adj_unsort<<<grid_for(n, 256, kNumSMs * 16), 256, 0, S(stream)>>>(
      n, perm, reinterpret_cast<const float4*>(gpos4_sorted), reinterpret_cast<const float4*>(gvel4_sorted),
      reinterpret_cast<float4*>(gpos4_out), reinterpret_cast<float4*>(gvel4_out));
  PF_LAUNCHED();
  return PF_OK;
}

}  // extern "C"
