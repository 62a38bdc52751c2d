// Variable-coefficient Poisson solver for sm_100a: aggregation Galerkin
// multigrid (red-black weighted Gauss-Seidel smoother) preconditioning a
// Polak-Ribiere flexible CG.  Follows the algorithm of pfflip/poisson.py
// (apply_A :54-88, rbgs_sweep :105-126, galerkin_coarsen_faces :130-163,
// restrict_sum :166-175, prolong_inject_add :178-182, MGPCG :240-409) with a
// B200-first kernel structure:
//
// * one kernel per red+black sweep.  A CTA owns a (j,k) tile of 8x32 cells and
//   an i-range, marches along i with a 4-plane ring of p (2-cell halo) in
//   shared memory, updates colour 1 on plane m (tile + 1-cell ring), then
//   colour 2 on plane m-1 (tile), and writes plane m-1 — colour 2 lags colour
//   1 by one plane.  Input and output p are different buffers (ping-pong), so
//   halos never mix old and new values across CTAs.  The result equals the
//   reference's two half-sweep launches.
// * the residual is fused with restriction, the prolongation with the first
//   post-smoothing sweep, a zero initial guess skips the p read, and the mean
//   of the level-0 V-cycle output is reduced inside the last sweep.
// * CG scalars never leave the device: every reduction is a deterministic
//   two-level FP64 sum (block partials, then the last CTA sums them in block
//   order), and the last CTA also forms alpha/beta and the stop test.  Every
//   kernel reads a device "done" flag, so the host can enqueue (or replay as a
//   CUDA graph) one CG iteration ahead and poll convergence one iteration late
//   without changing the result.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <utility>
#include <vector>

#include <cooperative_groups.h>
#include <cuda.h>

#include "pf_common.cuh"

namespace pf {

// --------------------------------------------------------------- device state
struct MGState {
  double rz, qAq, alpha, beta, bnorm, rel, rz_new, rpz;
  double sum_last;
  float c_shift;   // float(-mean) of the last mean reduction
  float alpha_f, neg_alpha_f, beta_f;
  float tol;
  float scale_r;   // 16-bit storage: level-0 b = r * scale_r
  float zscale;    // 16-bit storage: z = p_lp * zscale
  float maxabs_last;
  int32_t it, done, status, max_iter;
};
static_assert(sizeof(MGState) <= PF_MG_STATE_BYTES, "state size");

enum { ST_RUNNING = 0, ST_CONVERGED = 1, ST_BREAKDOWN = 2, ST_NONFINITE = 3, ST_ZERO_RHS = 4, ST_TMA_TIMEOUT = 5 };

// counters used by the last-CTA reductions (one per call site so that two
// reductions in flight never share a ticket)
enum {
  CNT_SUM_B = 0, CNT_INIT_R, CNT_INIT_Q, CNT_APPLY_DOT, CNT_UPDATE_XR, CNT_DOTS, CNT_SWEEP_MEAN, CNT_FINAL_SUM,
  CNT_COARSE, CNT_PRECOND, CNT_SCALE, CNT_MAX
};
static_assert(CNT_MAX <= PF_MG_COUNTERS, "counters");

constexpr int RED_NT = 256;
constexpr int64_t kPartials = 1 << 16;  // >= CTAs of any one reduction (sweep tiles up to 512^3)

__device__ __forceinline__ bool is_done(const MGState* st) { return st != nullptr && st->done != 0; }

// --------------------------------------------------------------- apply_A
// pfflip/poisson.py:54-75 with clamped neighbour indices and diag formed on
// the fly in compute_diag's order (pfflip/poisson.py:49-51) when diag is null.
__device__ __forceinline__ float apply_row(const float* __restrict__ p, const float* __restrict__ bx,
                                           const float* __restrict__ by, const float* __restrict__ bz,
                                           const float* __restrict__ diag, int nx, int ny, int nz, int i, int j,
                                           int k, int flux) {
  const long long c = ((long long)i * ny + j) * nz + k;
  const long long fxi = c;                                  // bx(i,j,k) = (i*ny + j)*nz + k
  const long long fxu = c + (long long)ny * nz;             // bx(i+1,j,k)
  const long long fyi = ((long long)i * (ny + 1) + j) * nz + k;
  const long long fyu = fyi + nz;
  const long long fzi = ((long long)i * ny + j) * (nz + 1) + k;
  const long long fzu = fzi + 1;
  const float bxl = bx[fxi], bxu = bx[fxu], byl = by[fyi], byu = by[fyu], bzl = bz[fzi], bzu = bz[fzu];
  const long long sI = (long long)ny * nz;
  const float pc = p[c];
  const float p0 = p[i > 0 ? c - sI : c], p1 = p[i < nx - 1 ? c + sI : c];
  const float p2 = p[j > 0 ? c - nz : c], p3 = p[j < ny - 1 ? c + nz : c];
  const float p4 = p[k > 0 ? c - 1 : c], p5 = p[k < nz - 1 ? c + 1 : c];
  if (flux) {
    float s = bxl * (pc - p0);
    s += bxu * (pc - p1);
    s += byl * (pc - p2);
    s += byu * (pc - p3);
    s += bzl * (pc - p4);
    s += bzu * (pc - p5);
    return s;
  }
  const float d = diag ? diag[c] : (bxl + bxu + byl + byu + bzl + bzu);
  float s = bxl * p0;
  s += bxu * p1;
  s += byl * p2;
  s += byu * p3;
  s += bzl * p4;
  s += bzu * p5;
  return d * pc - s;
}

__global__ void __launch_bounds__(C3_NT) k_apply_A(int nx, int ny, int nz, const float* __restrict__ p,
                                                  const float* __restrict__ bx, const float* __restrict__ by,
                                                  const float* __restrict__ bz, const float* __restrict__ diag,
                                                  float* __restrict__ out, int flux) {
  const Cell3 c = cell_here();
  if (c.j >= ny || c.k >= nz) return;
  out[((long long)c.i * ny + c.j) * nz + c.k] = apply_row(p, bx, by, bz, diag, nx, ny, nz, c.i, c.j, c.k, flux);
}

// --------------------------------------------------------------- hierarchy build
template <class T>
__global__ void k_level_coefs(int nx, int ny, int nz, const float* __restrict__ bx, const float* __restrict__ by,
                              const float* __restrict__ bz, float* __restrict__ diag, T* bx_lp, T* by_lp, T* bz_lp,
                              float lp_scale, float* __restrict__ bz_pad, int bz_pitch) {
  // diag (pfflip/poisson.py:41-51), the row-padded z-faces for TMA and, in
  // 16-bit mode, the scaled copies
  const long long nc = (long long)nx * ny * nz;
  const long long nfx = (long long)(nx + 1) * ny * nz, nfy = (long long)nx * (ny + 1) * nz,
                  nfz = (long long)nx * ny * (nz + 1);
  if (bz_pad) {  // fp32 hierarchy: fp32 rows; 16-bit hierarchy: the scaled 16-bit z-faces in the same buffer
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nfz; f += (long long)gridDim.x * blockDim.x) {
      const long long row = f / (nz + 1);
      const long long o = row * bz_pitch + (f - row * (nz + 1));
      if (bz_lp) stT(reinterpret_cast<T*>(bz_pad) + o, bz[f] * lp_scale);
      else bz_pad[o] = bz[f];
    }
  }
  const long long tot = nc + (bx_lp ? nfx + nfy + nfz : 0);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    if (e < nc) {
      const int k = (int)(e % nz);
      const long long t = e / nz;
      const int j = (int)(t % ny), i = (int)(t / ny);
      const long long fyi = ((long long)i * (ny + 1) + j) * nz + k;
      const long long fzi = ((long long)i * ny + j) * (nz + 1) + k;
      diag[e] = bx[e] + bx[e + (long long)ny * nz] + by[fyi] + by[fyi + nz] + bz[fzi] + bz[fzi + 1];
    } else {
      long long f = e - nc;
      if (f < nfx) stT(bx_lp + f, bx[f] * lp_scale);
      else if ((f -= nfx) < nfy) stT(by_lp + f, by[f] * lp_scale);
      else { f -= nfy; stT(bz_lp + f, bz[f] * lp_scale); }
    }
  }
}

// pfflip/poisson.py:130-163 for all three axes in one launch
__global__ void k_coarsen_faces(int fx, int fy, int fz, int cx, int cy, int cz, const float* __restrict__ fbx,
                                const float* __restrict__ fby, const float* __restrict__ fbz, float* __restrict__ cbx,
                                float* __restrict__ cby, float* __restrict__ cbz) {
  const long long ncx = (long long)(cx + 1) * cy * cz, ncy = (long long)cx * (cy + 1) * cz,
                  ncz = (long long)cx * cy * (cz + 1);
  const long long tot = ncx + ncy + ncz;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    int axis;
    long long f = e;
    Dim3i cd, fd;
    const float* fine;
    float* coarse;
    if (f < ncx) { axis = 0; cd = face_dims(cx, cy, cz, 0); fd = face_dims(fx, fy, fz, 0); fine = fbx; coarse = cbx; }
    else if ((f -= ncx) < ncy) { axis = 1; cd = face_dims(cx, cy, cz, 1); fd = face_dims(fx, fy, fz, 1); fine = fby; coarse = cby; }
    else { f -= ncy; axis = 2; cd = face_dims(cx, cy, cz, 2); fd = face_dims(fx, fy, fz, 2); fine = fbz; coarse = cbz; }
    const int K = (int)(f % cd.n2);
    const long long t = f / cd.n2;
    const int J = (int)(t % cd.n1), I = (int)(t / cd.n1);
    const int i0 = 2 * I, j0 = 2 * J, k0 = 2 * K;
    float acc = 0.f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        int ii, jj, kk;
        if (axis == 0) { ii = i0; jj = j0 + a; kk = k0 + b; }
        else if (axis == 1) { ii = i0 + a; jj = j0; kk = k0 + b; }
        else { ii = i0 + a; jj = j0 + b; kk = k0; }
        if (ii < fd.n0 && jj < fd.n1 && kk < fd.n2) acc += fine[fd.at(ii, jj, kk)];
      }
    coarse[f] = acc;
  }
}

// --------------------------------------------------------------- fused red-black sweep
// One CTA owns a TI x TJ x TK tile of cells.  It loads, with every load in
// flight at once, p with a 2-cell halo and b and the three face arrays with a
// 1-cell halo into shared memory (zero outside the level: boundary faces are
// zero, so the stencil never sees the fill), updates colour 1 on the tile and
// its 1-cell ring, then colour 2 on the tile, and writes the tile to p_out.
// p_in and p_out are different buffers, so the halo a CTA reads is never
// updated under it.  Within a row, thread q handles the q-th cell of the
// colour being updated, so no lane idles on the other colour.
constexpr int SW_TJ = 8, SW_TK = 32, SW_NT = 256;

template <int TI> struct TileDims {
  static constexpr int PI = TI + 4, PJ = SW_TJ + 4, PK = SW_TK + 4;  // p with 2-ring
  static constexpr int CI = TI + 2, CJ = SW_TJ + 2, CK = SW_TK + 2;  // cells with 1-ring
  static constexpr int PN = PI * PJ * PK;
  static constexpr int CN = CI * CJ * CK;
  static constexpr int XN = (CI + 1) * CJ * CK;
  static constexpr int YN = CI * (CJ + 1) * CK;
  static constexpr int ZN = CI * CJ * (CK + 1);
  static constexpr size_t SMEM = sizeof(float) * (PN + CN + XN + YN + ZN);
};

template <class T, class TB> struct SweepArgs {
  int n0, n1, n2;
  const T* p_in;           // ignored when zero_in
  T* p_out;
  const TB* b;
  const float* b_scale;    // device scalar (may be null = 1)
  const T* bx;
  const T* by;
  const T* bz;
  const T* pc;             // prolongation source (coarse p) or null
  float pc_scale;
  float omega;
  int first_color;
  int zero_in;
  double* partials;        // mean accumulation of p_out (null = off)
  unsigned* counter;
  MGState* st;             // done flag + mean output (may be null)
  int n_total;             // cells of the level (mean divisor)
  int mixed;               // mean is of p*zscale (16-bit hierarchy)
  int flux;                // PF_STENCIL_FLUX rows
};

// Gauss-Seidel update of one cell from shared-memory neighbourhoods.
// P: centre value pointer; sP[...] strides; faces and b passed in.
__device__ __forceinline__ float gs_update(float pv, float pxl, float pxu, float pyl, float pyu, float pzl, float pzu,
                                           float bxl, float bxu, float byl, float byu, float bzl, float bzu, float bb,
                                           float omega, int flux, bool* ok) {
  const float d = bxl + bxu + byl + byu + bzl + bzu;
  *ok = d > 0.f;
  float res;
  if (flux) {
    float sum = bxl * (pv - pxl);
    sum += bxu * (pv - pxu);
    sum += byl * (pv - pyl);
    sum += byu * (pv - pyu);
    sum += bzl * (pv - pzl);
    sum += bzu * (pv - pzu);
    res = bb - sum;
  } else {
    float sum = bxl * pxl;
    sum += bxu * pxu;
    sum += byl * pyl;
    sum += byu * pyu;
    sum += bzl * pzl;
    sum += bzu * pzu;
    res = bb - (d * pv - sum);
  }
  // (omega res) / d by the fast reciprocal (2 ulp; d is a sum of face
  // coefficients, far inside the range where that bound holds): the IEEE
  // division's refinement steps are a tenth of a relaxation's instructions
  return pv + __fdividef(omega * res, d);
}

template <class T, class TB, int TI>
__global__ void __launch_bounds__(SW_NT) k_rb_tile(SweepArgs<T, TB> a) {
  if (is_done(a.st)) return;
  using D = TileDims<TI>;
  extern __shared__ __align__(16) float smem[];
  float* sP = smem;
  float* sB = sP + D::PN;
  float* sX = sB + D::CN;
  float* sY = sX + D::XN;
  float* sZ = sY + D::YN;
  __shared__ double sred[40];

  const int n0 = a.n0, n1 = a.n1, n2 = a.n2;
  const int k0 = blockIdx.x * SW_TK, j0 = blockIdx.y * SW_TJ, i0 = blockIdx.z * TI;
  const int tid = threadIdx.x;
  const long long sI = (long long)n1 * n2;
  const float bsc = a.b_scale ? *a.b_scale : 1.f;
  const int hn1 = n1 >> 1, hn2 = n2 >> 1;

  // ---- loads (zero outside the level): every load of the CTA is issued into
  // registers before any is stored, so they are all in flight together
  constexpr int IP = (D::PN + SW_NT - 1) / SW_NT, IB = (D::CN + SW_NT - 1) / SW_NT;
  constexpr int IX = (D::XN + SW_NT - 1) / SW_NT, IY = (D::YN + SW_NT - 1) / SW_NT;
  constexpr int IZ = (D::ZN + SW_NT - 1) / SW_NT;
  float vp[IP], vb[IB], vx[IX], vy[IY], vz[IZ];
#pragma unroll
  for (int u = 0; u < IP; ++u) {
    const int e = tid + u * SW_NT;
    const int c = e % D::PK, t = e / D::PK, r = t % D::PJ, q = t / D::PJ;
    const int i = i0 - 2 + q, j = j0 - 2 + r, k = k0 - 2 + c;
    float v = 0.f;
    if (e < D::PN && i >= 0 && i < n0 && j >= 0 && j < n1 && k >= 0 && k < n2) {
      const long long g = i * sI + (long long)j * n2 + k;
      if (!a.zero_in) v = ldT(a.p_in + g);
      if (a.pc) v += ldT(a.pc + ((long long)(i >> 1) * hn1 + (j >> 1)) * hn2 + (k >> 1)) * a.pc_scale;
    }
    vp[u] = v;
  }
#pragma unroll
  for (int u = 0; u < IB; ++u) {
    const int e = tid + u * SW_NT;
    const int c = e % D::CK, t = e / D::CK, r = t % D::CJ, q = t / D::CJ;
    const int i = i0 - 1 + q, j = j0 - 1 + r, k = k0 - 1 + c;
    const bool in = e < D::CN && i >= 0 && i < n0 && j >= 0 && j < n1 && k >= 0 && k < n2;
    vb[u] = in ? ldT(a.b + i * sI + (long long)j * n2 + k) * bsc : 0.f;
  }
#pragma unroll
  for (int u = 0; u < IX; ++u) {  // x-faces i0-1 .. i0+TI+1
    const int e = tid + u * SW_NT;
    const int c = e % D::CK, t = e / D::CK, r = t % D::CJ, q = t / D::CJ;
    const int f = i0 - 1 + q, j = j0 - 1 + r, k = k0 - 1 + c;
    const bool in = e < D::XN && f >= 0 && f <= n0 && j >= 0 && j < n1 && k >= 0 && k < n2;
    vx[u] = in ? ldT(a.bx + (long long)f * sI + (long long)j * n2 + k) : 0.f;
  }
#pragma unroll
  for (int u = 0; u < IY; ++u) {  // y-faces j0-1 .. j0+TJ+1
    const int e = tid + u * SW_NT;
    const int c = e % D::CK, t = e / D::CK, r = t % (D::CJ + 1), q = t / (D::CJ + 1);
    const int i = i0 - 1 + q, f = j0 - 1 + r, k = k0 - 1 + c;
    const bool in = e < D::YN && i >= 0 && i < n0 && f >= 0 && f <= n1 && k >= 0 && k < n2;
    vy[u] = in ? ldT(a.by + ((long long)i * (n1 + 1) + f) * n2 + k) : 0.f;
  }
#pragma unroll
  for (int u = 0; u < IZ; ++u) {  // z-faces k0-1 .. k0+TK+1
    const int e = tid + u * SW_NT;
    const int c = e % (D::CK + 1), t = e / (D::CK + 1), r = t % D::CJ, q = t / D::CJ;
    const int i = i0 - 1 + q, j = j0 - 1 + r, f = k0 - 1 + c;
    const bool in = e < D::ZN && i >= 0 && i < n0 && j >= 0 && j < n1 && f >= 0 && f <= n2;
    vz[u] = in ? ldT(a.bz + ((long long)i * n1 + j) * (n2 + 1) + f) : 0.f;
  }
#pragma unroll
  for (int u = 0; u < IP; ++u)
    if (tid + u * SW_NT < D::PN) sP[tid + u * SW_NT] = vp[u];
#pragma unroll
  for (int u = 0; u < IB; ++u)
    if (tid + u * SW_NT < D::CN) sB[tid + u * SW_NT] = vb[u];
#pragma unroll
  for (int u = 0; u < IX; ++u)
    if (tid + u * SW_NT < D::XN) sX[tid + u * SW_NT] = vx[u];
#pragma unroll
  for (int u = 0; u < IY; ++u)
    if (tid + u * SW_NT < D::YN) sY[tid + u * SW_NT] = vy[u];
#pragma unroll
  for (int u = 0; u < IZ; ++u)
    if (tid + u * SW_NT < D::ZN) sZ[tid + u * SW_NT] = vz[u];
  __syncthreads();

  // relax the cell at coefficient-frame coordinates (q, r, c)
  auto relax = [&](int q, int r, int c) {
    float* pp = sP + ((q + 1) * D::PJ + (r + 1)) * D::PK + (c + 1);
    const int ce = (q * D::CJ + r) * D::CK + c;
    const float bxl = sX[ce], bxu = sX[ce + D::CJ * D::CK];
    const int ye = (q * (D::CJ + 1) + r) * D::CK + c;
    const float byl = sY[ye], byu = sY[ye + D::CK];
    const int ze = (q * D::CJ + r) * (D::CK + 1) + c;
    const float bzl = sZ[ze], bzu = sZ[ze + 1];
    bool ok;
    const float v = gs_update(*pp, pp[-D::PJ * D::PK], pp[D::PJ * D::PK], pp[-D::PK], pp[D::PK], pp[-1], pp[1], bxl,
                              bxu, byl, byu, bzl, bzu, sB[ce], a.omega, a.flux, &ok);
    if (ok) *pp = v;
  };

  // ---- colour 1 on the tile and its ring: per row of CK cells, CK/2 cells of the colour
  const int c1 = a.first_color, c2 = c1 ^ 1;
  {
    constexpr int HALF = D::CK / 2;  // 17
    for (int e = tid; e < D::CI * D::CJ * HALF; e += SW_NT) {
      const int h = e % HALF, row = e / HALF, r = row % D::CJ, q = row / D::CJ;
      const int i = i0 - 1 + q, j = j0 - 1 + r;
      const int par = (c1 - i - j - (k0 - 1)) & 1;
      const int c = 2 * h + par, k = k0 - 1 + c;
      if (i < 0 || i >= n0 || j < 0 || j >= n1 || k < 0 || k >= n2) continue;
      relax(q, r, c);
    }
  }
  __syncthreads();
  // ---- colour 2 on the tile
  {
    constexpr int HALF = SW_TK / 2;  // 16
    for (int e = tid; e < TI * SW_TJ * HALF; e += SW_NT) {
      const int h = e % HALF, row = e / HALF, r = row % SW_TJ, q = row / SW_TJ;
      const int i = i0 + q, j = j0 + r;
      const int par = (c2 - i - j - k0) & 1;
      const int c = 2 * h + par, k = k0 + c;
      if (i >= n0 || j >= n1 || k >= n2) continue;
      relax(q + 1, r + 1, c + 1);
    }
  }
  __syncthreads();
  // ---- write the tile
  double msum = 0.0;
  for (int e = tid; e < TI * SW_TJ * SW_TK; e += SW_NT) {
    const int c = e % SW_TK, t = e / SW_TK, r = t % SW_TJ, q = t / SW_TJ;
    const int i = i0 + q, j = j0 + r, k = k0 + c;
    if (i >= n0 || j >= n1 || k >= n2) continue;
    const float v = sP[((q + 2) * D::PJ + (r + 2)) * D::PK + (c + 2)];
    stT(a.p_out + i * sI + (long long)j * n2 + k, v);
    if (a.partials) msum += (double)roundT<T>(v);
  }
  if (a.partials) {
    const double bs = block_sum<SW_NT>(msum, sred);
    const int nb = gridDim.x * gridDim.y * gridDim.z;
    const int bid = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    __shared__ bool s_last;
    if (tid == 0) {
      a.partials[bid] = bs;
      __threadfence();
      s_last = (atomicAdd(a.counter, 1u) == (unsigned)nb - 1);
    }
    __syncthreads();
    if (s_last) {
      __threadfence();
      double v = 0.0;
      for (int q = tid; q < nb; q += SW_NT) v += __ldcg(a.partials + q);
      v = block_sum<SW_NT>(v, sred);
      if (tid == 0) {
        a.st->sum_last = v;
        a.st->c_shift = (float)(-(v / (double)a.n_total) * (a.mixed ? (double)a.st->zscale : 1.0));
        *a.counter = 0u;
      }
    }
  }
}

// --------------------------------------------------------------- TMA-staged sweep (fp32)
// Same sweep as k_rb_tile, but one thread stages the five tiles (p with a
// 2-cell halo; b, x-, y- and z-faces with a 1-cell halo) into shared memory
// with cp.async.bulk.tensor (TMA, no multicast), completing on an mbarrier.
// The boxes are 40 floats wide starting at k0 - 4, so every x coordinate is a
// multiple of 4 floats (16 bytes); cells outside the level read the TMA zero
// fill.  The mbarrier wait is bounded: on expiry the kernel flags
// ST_TMA_TIMEOUT, stops the solve and waits (bounded) before returning.
constexpr int TM_W = 40, TM_X0 = 4;  // box width, k offset of the box start

template <int TI> struct TmaDims {
  static constexpr int PI = TI + 4, PJ = SW_TJ + 4;
  static constexpr int CI = TI + 2, CJ = SW_TJ + 2;
  static constexpr int PN = PI * PJ * TM_W, BN = CI * CJ * TM_W, XN = (CI + 1) * CJ * TM_W, YN = CI * (CJ + 1) * TM_W,
                       ZN = CI * CJ * TM_W;
  static constexpr int r128(int b) { return (b + 127) / 128 * 128; }
  static constexpr int OFF_B = r128(PN * 4), OFF_X = OFF_B + r128(BN * 4), OFF_Y = OFF_X + r128(XN * 4),
                       OFF_Z = OFF_Y + r128(YN * 4), OFF_BAR = OFF_Z + r128(ZN * 4);
  static constexpr size_t SMEM = OFF_BAR + 128 + 128;  // + slack to align the base to 128 bytes
};

struct TileMaps {
  CUtensorMap p, b, x, y, z;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

constexpr unsigned kTmaWaitLimit = 1u << 22;

// One staged tile of the red-black sweep: prolongation folded into the staged
// p (first post-sweep), colour 1 on the tile and its ring, colour 2 on the
// tile, write-back of the tile to p_out (msum += the written values).
//   FS, FW, FX0: element type, row width and k offset (the row starts at
//   k0 - FX0) of the staged faces; BS, BW, BX0 the same for b.  p is staged as
//   float rows of TM_W starting at k0 - TM_X0.
template <int TI, int NT, class T, class TB, class FS = float, int FW = TM_W, int FX0 = TM_X0, class BS = float,
          int BW = TM_W, int BX0 = TM_X0>
__device__ __forceinline__ void tma_tile_sweep(float* sP, const BS* sB, const FS* sX, const FS* sY, const FS* sZ,
                                               const SweepArgs<T, TB>& a, int k0, int j0, int i0, double& msum) {
  using D = TmaDims<TI>;
  const float bsc = a.b_scale ? *a.b_scale : 1.f;
  const int n0 = a.n0, n1 = a.n1, n2 = a.n2;
  const int tid = threadIdx.x;
  const long long sI = (long long)n1 * n2;
  const int hn1 = n1 >> 1, hn2 = n2 >> 1;
  if (a.pc) {  // prolongation folded into the staged p
    for (int e = tid; e < D::PN; e += NT) {
      const int c = e % TM_W, t = e / TM_W, r = t % D::PJ, q = t / D::PJ;
      const int i = i0 - 2 + q, j = j0 - 2 + r, k = k0 - TM_X0 + c;
      if (i >= 0 && i < n0 && j >= 0 && j < n1 && k >= 0 && k < n2)
        sP[e] += ldT(a.pc + ((long long)(i >> 1) * hn1 + (j >> 1)) * hn2 + (k >> 1)) * a.pc_scale;
    }
    __syncthreads();
  }

  // Relax the cells of colour `col` in column (r, c) of the coefficient frame
  // (cell (q, r, c) is (i0 - 1 + q, j0 - 1 + r, k0 - 1 + c)), planes
  // qlo <= q < qhi.  Along a column the colour alternates with q, so the
  // column's cells of one colour are every other plane: the plane steps are
  // compile-time offsets into the staged boxes.
  auto relax_column = [&](int r, int c, int qlo, int qhi, int col) {
    const int j = j0 - 1 + r, k = k0 - 1 + c;
    if (j < 0 || j >= n1 || k < 0 || k >= n2) return;
    const int q0 = qlo + ((col - (i0 - 1 + qlo) - j - k) & 1);
    float* pp = sP + ((q0 + 1) * D::PJ + (r + 1)) * TM_W + (c + TM_X0 - 1);
    const int cf = (q0 * D::CJ + r) * FW + (c + FX0 - 1);
    const FS* px = sX + cf;
    const FS* pz = sZ + cf;
    const FS* py = sY + (q0 * (D::CJ + 1) + r) * FW + (c + FX0 - 1);
    const BS* pb = sB + (q0 * D::CJ + r) * BW + (c + BX0 - 1);
#pragma unroll
    for (int u = 0; u < (D::CI + 1) / 2; ++u) {
      const int q = q0 + 2 * u, i = i0 - 1 + q;
      if (q < qhi && i >= 0 && i < n0) {
        float* P = pp + u * 2 * D::PJ * TM_W;
        const FS* X = px + u * 2 * D::CJ * FW;
        const FS* Y = py + u * 2 * (D::CJ + 1) * FW;
        const FS* Z = pz + u * 2 * D::CJ * FW;
        const float bb = ldT(pb + u * 2 * D::CJ * BW) * bsc;
        bool ok;
        const float v = gs_update(*P, P[-D::PJ * TM_W], P[D::PJ * TM_W], P[-TM_W], P[TM_W], P[-1], P[1], ldT(X),
                                  ldT(X + D::CJ * FW), ldT(Y), ldT(Y + FW), ldT(Z), ldT(Z + 1), bb, a.omega, a.flux,
                                  &ok);
        if (ok) *P = v;
      }
    }
  };
  const int c1 = a.first_color, c2 = c1 ^ 1;
  // colour 1 on the tile and its 1-cell ring: columns (r, c) of the
  // CJ x (SW_TK + 2) frame, planes 0 .. CI-1
  for (int t = tid; t < D::CJ * (SW_TK + 2); t += NT) {
    const int r = t / (SW_TK + 2), c = t - r * (SW_TK + 2);
    relax_column(r, c, 0, D::CI, c1);
  }
  __syncthreads();
  // colour 2 on the tile: columns (1 .. SW_TJ, 1 .. SW_TK), planes 1 .. TI
  for (int t = tid; t < SW_TJ * SW_TK; t += NT) {
    const int r = 1 + (t >> 5), c = 1 + (t & 31);  // SW_TK == 32
    relax_column(r, c, 1, TI + 1, c2);
  }
  __syncthreads();
  for (int e = tid; e < TI * SW_TJ * SW_TK; e += NT) {
    const int c = e & 31, r = (e >> 5) & 7, q = e >> 8;  // SW_TK == 32, SW_TJ == 8
    const int i = i0 + q, j = j0 + r, k = k0 + c;
    if (i >= n0 || j >= n1 || k >= n2) continue;
    const float v = sP[((q + 2) * D::PJ + (r + 2)) * TM_W + (c + TM_X0)];
    stT(a.p_out + i * sI + (long long)j * n2 + k, v);
    if (a.partials) msum += (double)roundT<T>(v);
  }
}

// mean of p_out over the grid: one partial per CTA, the last CTA sums them in
// order and stores the shift in the solver state
template <int NT, class T, class TB>
__device__ __forceinline__ void sweep_mean_finish(const SweepArgs<T, TB>& a, double msum, double* sred) {
  const int tid = threadIdx.x;
  if (a.partials) {
    const double bs = block_sum<NT>(msum, sred);
    const int nb = gridDim.x * gridDim.y * gridDim.z;
    const int bid = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    __shared__ bool s_last;
    if (tid == 0) {
      a.partials[bid] = bs;
      __threadfence();
      s_last = (atomicAdd(a.counter, 1u) == (unsigned)nb - 1);
    }
    __syncthreads();
    if (s_last) {
      __threadfence();
      double v = 0.0;
      for (int q = tid; q < nb; q += NT) v += __ldcg(a.partials + q);
      v = block_sum<NT>(v, sred);
      if (tid == 0) {
        a.st->sum_last = v;
        a.st->c_shift = (float)(-(v / (double)a.n_total) * (a.mixed ? (double)a.st->zscale : 1.0));
        *a.counter = 0u;
      }
    }
  }
}

// Programmatic dependent launch: a sweep is launched so that it may start
// while the kernel before it finishes.  Until griddepcontrol.wait returns (all
// prerequisite grids complete, their writes visible) it touches only its own
// shared memory and the face coefficients, which no kernel of a solve writes.
// Once its tile has landed it lets the next kernel launch (which then starts
// when every CTA of this one has done so or exited).
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <int TI, int NT>
__global__ void __launch_bounds__(NT) k_rb_tile_tma(const __grid_constant__ TileMaps maps, SweepArgs<float, float> a) {
  using D = TmaDims<TI>;
  extern __shared__ __align__(128) unsigned char tsm_raw[];
  unsigned char* tsm = tsm_raw + ((128u - (smem_u32(tsm_raw) & 127u)) & 127u);
  float* sP = reinterpret_cast<float*>(tsm);
  float* sB = reinterpret_cast<float*>(tsm + D::OFF_B);
  float* sX = reinterpret_cast<float*>(tsm + D::OFF_X);
  float* sY = reinterpret_cast<float*>(tsm + D::OFF_Y);
  float* sZ = reinterpret_cast<float*>(tsm + D::OFF_Z);
  uint64_t* bar = reinterpret_cast<uint64_t*>(tsm + D::OFF_BAR);
  __shared__ double sred[40];
  __shared__ int s_fail;

  const int k0 = blockIdx.x * SW_TK, j0 = blockIdx.y * SW_TJ, i0 = blockIdx.z * TI;
  const int tid = threadIdx.x;
  const bool load_p = !a.zero_in;

  const int x = k0 - TM_X0;
  if (tid == 0) {
    s_fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    // the faces first, while the previous kernel may still run
    const unsigned fbytes = 4u * (unsigned)(D::XN + D::YN + D::ZN);
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(fbytes)
                 : "memory");
    tma_load_3d(sX, &maps.x, x, j0 - 1, i0 - 1, bar);
    tma_load_3d(sY, &maps.y, x, j0 - 1, i0 - 1, bar);
    tma_load_3d(sZ, &maps.z, x, j0 - 1, i0 - 1, bar);
  }
  if (!load_p)
    for (int e = tid; e < D::PN; e += NT) sP[e] = 0.f;
  grid_dep_wait();
  const bool done = is_done(a.st);
  if (tid == 0) {
    // p and b come from the previous kernels; a finished solve loads nothing
    // more and only lets the face copies land before the CTA leaves
    const unsigned bytes = done ? 0u : 4u * (unsigned)((load_p ? D::PN : 0) + D::BN);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    if (!done) {
      if (load_p) tma_load_3d(sP, &maps.p, x, j0 - 2, i0 - 2, bar);
      tma_load_3d(sB, &maps.b, x, j0 - 1, i0 - 1, bar);
    }
  }
  __syncthreads();  // barrier initialised before anyone waits on it
  {
    unsigned it = 0;
    while (!mbar_try_wait(bar, 0)) {
      if (++it > kTmaWaitLimit) {
        s_fail = 1;
        break;
      }
    }
  }
  __syncthreads();
  if (s_fail) {
    if (tid == 0 && a.st) {
      a.st->status = ST_TMA_TIMEOUT;
      a.st->done = 1;
    }
    unsigned it = 0;  // give the copies in flight a last bounded chance to land
    while (!mbar_try_wait(bar, 0) && ++it < kTmaWaitLimit) {
    }
    return;
  }
  grid_dep_launch();  // staged: the next kernel may start its own staging now
  if (done) return;
  double msum = 0.0;
  tma_tile_sweep<TI, NT, float, float>(sP, sB, sX, sY, sZ, a, k0, j0, i0, msum);
  sweep_mean_finish<NT>(a, msum, sred);
}

// --------------------------------------------------------------- TMA-staged sweep (16-bit hierarchy)
// The same sweep over FP16/BF16 levels.  16-bit rows are 48 elements (96 bytes)
// from k0 - 8, so every x coordinate stays a multiple of 16 bytes; b comes in
// as fp32 rows of 40 from k0 - 4 on the finest level (the FP32 residual) and
// as 16-bit rows elsewhere.  p is staged raw and widened once into fp32 rows,
// so both colours relax in fp32 exactly as k_rb_tile does; faces and b are
// widened where they are read.  The z-faces come from the padded 16-bit copy
// k_level_coefs writes into the level's bz_pad buffer.
constexpr int TM16_W = 48, TM16_X0 = 8;

template <int TI, bool B32> struct Tma16Dims {
  static constexpr int PI = TI + 4, PJ = SW_TJ + 4, CI = TI + 2, CJ = SW_TJ + 2;
  static constexpr int BW = B32 ? TM_W : TM16_W, BES = B32 ? 4 : 2;
  static constexpr int P16N = PI * PJ * TM16_W, P32N = PI * PJ * TM_W, BN = CI * CJ * BW;
  static constexpr int XN = (CI + 1) * CJ * TM16_W, YN = CI * (CJ + 1) * TM16_W, ZN = CI * CJ * TM16_W;
  static constexpr int r128(int b) { return (b + 127) / 128 * 128; }
  static constexpr int OFF_P32 = r128(P16N * 2), OFF_B = OFF_P32 + r128(P32N * 4), OFF_X = OFF_B + r128(BN * BES),
                       OFF_Y = OFF_X + r128(XN * 2), OFF_Z = OFF_Y + r128(YN * 2), OFF_BAR = OFF_Z + r128(ZN * 2);
  static constexpr size_t SMEM = OFF_BAR + 128 + 128;
};

template <int TI, int NT, class T, class TB>
__global__ void __launch_bounds__(NT) k_rb_tile_tma16(const __grid_constant__ TileMaps maps, SweepArgs<T, TB> a) {
  // launched like k_rb_tile_tma: faces before the wait, p and b after it
  constexpr bool B32 = std::is_same<TB, float>::value;
  using D = TmaDims<TI>;
  using E = Tma16Dims<TI, B32>;
  extern __shared__ __align__(128) unsigned char hsm_raw[];
  unsigned char* hsm = hsm_raw + ((128u - (smem_u32(hsm_raw) & 127u)) & 127u);
  T* sP16 = reinterpret_cast<T*>(hsm);
  float* sP = reinterpret_cast<float*>(hsm + E::OFF_P32);
  TB* sB = reinterpret_cast<TB*>(hsm + E::OFF_B);
  T* sX = reinterpret_cast<T*>(hsm + E::OFF_X);
  T* sY = reinterpret_cast<T*>(hsm + E::OFF_Y);
  T* sZ = reinterpret_cast<T*>(hsm + E::OFF_Z);
  uint64_t* bar = reinterpret_cast<uint64_t*>(hsm + E::OFF_BAR);
  __shared__ double sred[40];
  __shared__ int s_fail;
  const int k0 = blockIdx.x * SW_TK, j0 = blockIdx.y * SW_TJ, i0 = blockIdx.z * TI;
  const int tid = threadIdx.x;
  const bool load_p = !a.zero_in;
  const int x16 = k0 - TM16_X0, xb = B32 ? k0 - TM_X0 : k0 - TM16_X0;
  if (tid == 0) {
    s_fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const unsigned fbytes = (unsigned)((E::XN + E::YN + E::ZN) * 2);
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(fbytes)
                 : "memory");
    tma_load_3d(sX, &maps.x, x16, j0 - 1, i0 - 1, bar);
    tma_load_3d(sY, &maps.y, x16, j0 - 1, i0 - 1, bar);
    tma_load_3d(sZ, &maps.z, x16, j0 - 1, i0 - 1, bar);
  }
  grid_dep_wait();
  const bool done = is_done(a.st);
  if (tid == 0) {
    const unsigned bytes = done ? 0u : (unsigned)((load_p ? E::P16N * 2 : 0) + E::BN * E::BES);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    if (!done) {
      if (load_p) tma_load_3d(sP16, &maps.p, x16, j0 - 2, i0 - 2, bar);
      tma_load_3d(sB, &maps.b, xb, j0 - 1, i0 - 1, bar);
    }
  }
  __syncthreads();  // barrier initialised before anyone waits on it
  {
    unsigned it = 0;
    while (!mbar_try_wait(bar, 0)) {
      if (++it > kTmaWaitLimit) {
        s_fail = 1;
        break;
      }
    }
  }
  __syncthreads();
  if (s_fail) {
    if (tid == 0 && a.st) {
      a.st->status = ST_TMA_TIMEOUT;
      a.st->done = 1;
    }
    unsigned it = 0;  // give the copies in flight a last bounded chance to land
    while (!mbar_try_wait(bar, 0) && ++it < kTmaWaitLimit) {
    }
    return;
  }
  grid_dep_launch();
  if (done) return;
  for (int e = tid; e < D::PN; e += NT) {  // p: 16-bit rows from k0 - 8 -> fp32 rows from k0 - 4
    const int row = e / TM_W, c = e - row * TM_W;
    sP[e] = load_p ? ldT(sP16 + row * TM16_W + c + (TM16_X0 - TM_X0)) : 0.f;
  }
  __syncthreads();
  double msum = 0.0;
  tma_tile_sweep<TI, NT, T, TB, T, TM16_W, TM16_X0, TB, E::BW, (B32 ? TM_X0 : TM16_X0)>(sP, sB, sX, sY, sZ, a, k0,
                                                                                       j0, i0, msum);
  sweep_mean_finish<NT>(a, msum, sred);
}


// --------------------------------------------------------------- residual + restriction
// coarse b = rscale * sum over the 8 fine cells of (b - A p)  (pfflip/poisson.py:91-102, :166-175)
template <class T, class TB>
__global__ void k_residual_restrict(int n0, int n1, int n2, const T* __restrict__ p, const TB* __restrict__ b,
                                    const float* b_scale, const T* __restrict__ bx, const T* __restrict__ by,
                                    const T* __restrict__ bz, T* __restrict__ cb, float rscale, float* fine_r,
                                    const MGState* st, int flux) {
  if (is_done(st)) return;
  const int C1 = n1 >> 1, C2 = n2 >> 1;
  const float bsc = b_scale ? *b_scale : 1.f;
  const long long sI = (long long)n1 * n2;
  {
    const Cell3 cc3 = cell_here();
    const int I = cc3.i, J = cc3.j, K = cc3.k;
    if (J >= C1 || K >= C2) return;
    const long long e = ((long long)I * C1 + J) * C2 + K;
    float acc = 0.f;
#pragma unroll
    for (int aa = 0; aa < 2; ++aa)
#pragma unroll
      for (int bb = 0; bb < 2; ++bb)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          const int i = 2 * I + aa, j = 2 * J + bb, k = 2 * K + cc;
          const long long c = i * sI + (long long)j * n2 + k;
          const long long fyi = ((long long)i * (n1 + 1) + j) * n2 + k;
          const long long fzi = ((long long)i * n1 + j) * (n2 + 1) + k;
          const float bxl = ldT(bx + c), bxu = ldT(bx + c + sI), byl = ldT(by + fyi), byu = ldT(by + fyi + n2),
                      bzl = ldT(bz + fzi), bzu = ldT(bz + fzi + 1);
          const float pv = ldT(p + c);
          const float q0 = ldT(p + (i > 0 ? c - sI : c)), q1 = ldT(p + (i < n0 - 1 ? c + sI : c));
          const float q2 = ldT(p + (j > 0 ? c - n2 : c)), q3 = ldT(p + (j < n1 - 1 ? c + n2 : c));
          const float q4 = ldT(p + (k > 0 ? c - 1 : c)), q5 = ldT(p + (k < n2 - 1 ? c + 1 : c));
          float Ap;
          if (flux) {
            float s = bxl * (pv - q0);
            s += bxu * (pv - q1);
            s += byl * (pv - q2);
            s += byu * (pv - q3);
            s += bzl * (pv - q4);
            s += bzu * (pv - q5);
            Ap = s;
          } else {
            const float d = bxl + bxu + byl + byu + bzl + bzu;
            float s = bxl * q0;
            s += bxu * q1;
            s += byl * q2;
            s += byu * q3;
            s += bzl * q4;
            s += bzu * q5;
            Ap = d * pv - s;
          }
          const float r = ldT(b + c) * bsc - Ap;
          if (fine_r) fine_r[c] = r;
          acc += r;
        }
    stT(cb + e, acc * rscale);
  }
}

// --------------------------------------------------------------- bottom of the V-cycle
// All levels from `lb` down (each <= kBottomMaxCells cells) run inside one CTA
// with the levels in shared memory: pre-smoothing, residual + restriction,
// the coarsest solve (`coarsest` sweeps from zero, then mean removal,
// pfflip/poisson.py:325-328), prolongation and post-smoothing, exactly the
// reference's recursion (pfflip/poisson.py:323-343) with in-place red/black
// half-sweeps separated by barriers.  Replaces ~7 launches per level.  The
// coarsest level runs in AccT (float reproduces the reference; double is the
// FP64 coarsest solve of the 16-bit hierarchy), by one warp when it has at most
// 256 cells.
constexpr int kBottomMaxCells = 4096;
constexpr int BT_NT = 1024;

struct BottomLevel {
  int n0, n1, n2;
  int s1, s2;  // log2(n1), log2(n2) when both are powers of two, else -1
  const void* bx;
  const void* by;
  const void* bz;
};

template <class T, class TB> struct BottomArgs {
  int nl;                           // bottom levels, [0] = top
  BottomLevel L[PF_MG_MAX_LEVELS];
  const TB* b;                      // right-hand side of the top bottom level
  const float* b_scale;
  T* p_out;                         // solution of the top bottom level
  float omega;
  int pre, post, coarsest;
  float rscale, pscale;
  int flux;
  MGState* st;
  int want_mean, mixed;
  int bulk;  // stage faces and b with cp.async.bulk: 1 = fp32 storage straight into the level arrays,
             // 2 = 16-bit storage into a staging area behind Pc, widened there (16-byte sizes)
};

__host__ __device__ inline size_t bottom_level_floats(int n0, int n1, int n2) {
  const size_t n = (size_t)n0 * n1 * n2;
  return 2 * n + (size_t)(n0 + 1) * n1 * n2 + (size_t)n0 * (n1 + 1) * n2 + (size_t)n0 * n1 * (n2 + 1);
}

// cell (i,j,k) of linear index e
__device__ __forceinline__ void bt_ijk(const BottomLevel& L, int e, int& i, int& j, int& k) {
  if (L.s1 >= 0) {
    k = e & (L.n2 - 1);
    const int t = e >> L.s2;
    j = t & (L.n1 - 1);
    i = t >> L.s1;
  } else {
    k = e % L.n2;
    const int t = e / L.n2;
    j = t % L.n1;
    i = t / L.n1;
  }
}

// in-place relax of cell (i,j,k) of a shared-memory level, clamped neighbours
template <class R>
__device__ __forceinline__ void bt_relax(R* P, const float* B, const float* X, const float* Y, const float* Z, int n0,
                                         int n1, int n2, int i, int j, int k, R omega, int flux) {
  const int sI = n1 * n2, e = (i * n1 + j) * n2 + k;
  const int fyi = (i * (n1 + 1) + j) * n2 + k, fzi = (i * n1 + j) * (n2 + 1) + k;
  const R bxl = X[e], bxu = X[e + sI], byl = Y[fyi], byu = Y[fyi + n2], bzl = Z[fzi], bzu = Z[fzi + 1];
  const R d = (R)(X[e] + X[e + sI] + Y[fyi] + Y[fyi + n2] + Z[fzi] + Z[fzi + 1]);
  if (!(d > R(0))) return;
  const R pv = P[e];
  const R q0 = P[i > 0 ? e - sI : e], q1 = P[i < n0 - 1 ? e + sI : e];
  const R q2 = P[j > 0 ? e - n2 : e], q3 = P[j < n1 - 1 ? e + n2 : e];
  const R q4 = P[k > 0 ? e - 1 : e], q5 = P[k < n2 - 1 ? e + 1 : e];
  R res;
  if (flux) {
    R sum = bxl * (pv - q0);
    sum += bxu * (pv - q1);
    sum += byl * (pv - q2);
    sum += byu * (pv - q3);
    sum += bzl * (pv - q4);
    sum += bzu * (pv - q5);
    res = (R)B[e] - sum;
  } else {
    R sum = bxl * q0;
    sum += bxu * q1;
    sum += byl * q2;
    sum += byu * q3;
    sum += bzl * q4;
    sum += bzu * q5;
    res = (R)B[e] - (d * pv - sum);
  }
  if constexpr (std::is_same<R, float>::value) P[e] = pv + __fdividef(omega * res, d);  // as gs_update
  else P[e] = pv + omega * res / d;
}

// `sweeps` red-black sweeps of a coarsest level of at most 64 cells with an
// even k extent, by one warp with everything in registers.  Lane l holds the
// cells 2l and 2l+1 (same row, k = 2h and 2h+1): one of each colour.  For a
// half-sweep of colour c every lane publishes its other-colour cell; that is
// exactly the value each neighbour of a colour-c cell needs (its +-i and +-j
// neighbours sit at the same k in lanes l -+ n1*n2/2 and l -+ n2/2, its +-k
// neighbours are the lane's own other cell or the one published by lane l-+1).
// Neighbours past the walls take the cell's own value, as bt_relax clamps
// them.  Faces, b and the diagonal are read once; the row arithmetic is
// bt_relax's, operation for operation, so the result equals the shared-memory
// sweeps bit for bit.  P (AccT, shared) holds zeros on entry and the solution
// on return.
template <class R>
__device__ __forceinline__ void bt_coarsest_regs(const BottomLevel& L, R* P, const float* B, const float* X,
                                                 const float* Y, const float* Z, R omega, int sweeps, int flux,
                                                 int lane) {
  const int n0 = L.n0, n1 = L.n1, n2 = L.n2, hk = n2 >> 1;
  const int half = (n0 * n1 * n2) >> 1;
  const bool act = lane < half;
  const int l = act ? lane : 0;
  const int h = l % hk, row = l / hk, j = row % n1, i = row / n1;
  const int sI = n1 * n2;
  float cx0[2], cx1[2], cy0[2], cy1[2], cz0[2], cz1[2], cb[2], cd[2];  // as stored; widened at use
  // FP64 (16-bit hierarchy): omega/d once per cell instead of a division per
  // relaxation; FP32 keeps bt_relax's omega*res/d
  constexpr bool kRecip = std::is_same<R, double>::value;
  R cw[2];
  R p[2];
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int k = 2 * h + s, e = (i * n1 + j) * n2 + k;
    const int fyi = (i * (n1 + 1) + j) * n2 + k, fzi = (i * n1 + j) * (n2 + 1) + k;
    cx0[s] = X[e];
    cx1[s] = X[e + sI];
    cy0[s] = Y[fyi];
    cy1[s] = Y[fyi + n2];
    cz0[s] = Z[fzi];
    cz1[s] = Z[fzi + 1];
    cd[s] = X[e] + X[e + sI] + Y[fyi] + Y[fyi + n2] + Z[fzi] + Z[fzi + 1];
    cb[s] = B[e];
    cw[s] = kRecip ? omega / (R)cd[s] : R(0);
    p[s] = act ? P[2 * l + s] : R(0);
  }
  const int di = n1 * hk;
  const int sim = max(lane - di, 0), sip = min(lane + di, 31);
  const int sjm = max(lane - hk, 0), sjp = min(lane + hk, 31);
  const int skm = max(lane - 1, 0), skp = min(lane + 1, 31);
  for (int sw = 0; sw < sweeps; ++sw) {
#pragma unroll
    for (int color = 0; color < 2; ++color) {
      const int sc = (color - i - j) & 1;
      const R pub = sc ? p[0] : p[1];
      const R vim = __shfl_sync(0xffffffffu, pub, sim), vip = __shfl_sync(0xffffffffu, pub, sip);
      const R vjm = __shfl_sync(0xffffffffu, pub, sjm), vjp = __shfl_sync(0xffffffffu, pub, sjp);
      const R vkm = __shfl_sync(0xffffffffu, pub, skm), vkp = __shfl_sync(0xffffffffu, pub, skp);
      const R pv = sc ? p[1] : p[0];
      const R q0 = i > 0 ? vim : pv, q1 = i < n0 - 1 ? vip : pv;
      const R q2 = j > 0 ? vjm : pv, q3 = j < n1 - 1 ? vjp : pv;
      const R q4 = sc ? p[0] : (h > 0 ? vkm : pv);
      const R q5 = sc ? (h < hk - 1 ? vkp : pv) : p[1];
      const R bxl = sc ? cx0[1] : cx0[0], bxu = sc ? cx1[1] : cx1[0];
      const R byl = sc ? cy0[1] : cy0[0], byu = sc ? cy1[1] : cy1[0];
      const R bzl = sc ? cz0[1] : cz0[0], bzu = sc ? cz1[1] : cz1[0];
      const R d = sc ? cd[1] : cd[0], bb = sc ? cb[1] : cb[0];
      R res;
      if (flux) {
        R sum = bxl * (pv - q0);
        sum += bxu * (pv - q1);
        sum += byl * (pv - q2);
        sum += byu * (pv - q3);
        sum += bzl * (pv - q4);
        sum += bzu * (pv - q5);
        res = bb - sum;
      } else {
        R sum = bxl * q0;
        sum += bxu * q1;
        sum += byl * q2;
        sum += byu * q3;
        sum += bzl * q4;
        sum += bzu * q5;
        res = bb - (d * pv - sum);
      }
      R nv = pv;
      if (act && d > R(0)) nv = kRecip ? pv + res * (sc ? cw[1] : cw[0]) : pv + omega * res / d;
      if (sc) p[1] = nv;
      else p[0] = nv;
    }
  }
  if (act) {
    P[2 * l] = p[0];
    P[2 * l + 1] = p[1];
  }
}

// one half-sweep (cells of `color`) over a level with nt threads starting at tid
template <class R>
__device__ __forceinline__ void bt_half_sweep(const BottomLevel& L, R* P, const float* B, const float* X,
                                              const float* Y, const float* Z, int color, R omega, int flux, int tid,
                                              int nt) {
  const int n0 = L.n0, n1 = L.n1, n2 = L.n2;
  if (L.s1 >= 0 && n2 >= 2) {  // powers of two: only the cells of this colour, shift indexing
    const int hn = (n0 * n1 * n2) >> 1, sh = L.s2 - 1, hm = (n2 >> 1) - 1;
    for (int e = tid; e < hn; e += nt) {
      const int h = e & hm, row = e >> sh, j = row & (n1 - 1), i = row >> L.s1;
      const int k = 2 * h + ((color - i - j) & 1);
      bt_relax<R>(P, B, X, Y, Z, n0, n1, n2, i, j, k, omega, flux);
    }
  } else if ((n2 & 1) == 0) {  // only the cells of this colour: two per pair along k
    const int hn = (n0 * n1 * n2) >> 1, hk = n2 >> 1;
    for (int e = tid; e < hn; e += nt) {
      const int h = e % hk, row = e / hk, j = row % n1, i = row / n1;
      const int k = 2 * h + ((color - i - j) & 1);
      bt_relax<R>(P, B, X, Y, Z, n0, n1, n2, i, j, k, omega, flux);
    }
  } else {
    const int n = n0 * n1 * n2;
    for (int e = tid; e < n; e += nt) {
      int i, j, k;
      bt_ijk(L, e, i, j, k);
      if (((i + j + k) & 1) != color) continue;
      bt_relax<R>(P, B, X, Y, Z, n0, n1, n2, i, j, k, omega, flux);
    }
  }
}

// dst[e] = src[e] (converted) for e < n, loads issued 8 at a time
template <class T, int NT = BT_NT>
__device__ __forceinline__ void bt_load(float* dst, const T* src, int n, float scale, int tid) {
  for (int base = tid; base < n; base += 8 * NT) {
    float v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = base + u * NT;
      v[u] = (e < n) ? ldT(src + e) * scale : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = base + u * NT;
      if (e < n) dst[e] = v[u];
    }
  }
}

struct BtPtrs {
  float *P, *B, *X, *Y, *Z;
};

// arrays of level l of a run of levels laid out back to back from base
// (per level P, B, X, Y, Z in that order)
__device__ __forceinline__ BtPtrs bt_ptrs(const BottomLevel* Ls, float* base, int l) {
  size_t off = 0;
  for (int q = 0; q < l; ++q) off += bottom_level_floats(Ls[q].n0, Ls[q].n1, Ls[q].n2);
  const int n0 = Ls[l].n0, n1 = Ls[l].n1, n2 = Ls[l].n2, n = n0 * n1 * n2;
  BtPtrs r;
  r.P = base + off;
  r.B = r.P + n;
  r.X = r.B + n;
  r.Y = r.X + (n0 + 1) * n1 * n2;
  r.Z = r.Y + n0 * (n1 + 1) * n2;
  return r;
}

// The V-cycle over levels l0 .. nl-1 held in one CTA's shared memory from
// base (NT threads, CTA barriers only): level l0's B is set and every P is zero
// on entry; level l0's P holds the result on return.  Pre-smoothing, residual
// and restriction on the way down, `coarsest` sweeps from zero in AccT with the
// mean removed, prolongation and post-smoothing with the colours reversed on
// the way up (pfflip/poisson.py:312-345).
template <class T, class AccT, int NT = BT_NT>
__device__ void bt_local_vcycle(const BottomLevel* Ls, float* base, int l0, int nl, AccT* Pc, float om, int pre,
                                int post, int coarsest, float rscale, float pscale, int flux, double* sred,
                                double* s_mean) {
  const int tid = threadIdx.x;
  // ---- down: pre-smoothing, residual, restriction
  for (int l = l0; l < nl - 1; ++l) {
    const BottomLevel& L = Ls[l];
    const BtPtrs q = bt_ptrs(Ls, base, l);
    for (int sw = 0; sw < pre; ++sw)
      for (int cc = 0; cc < 2; ++cc) {
        bt_half_sweep<float>(L, q.P, q.B, q.X, q.Y, q.Z, cc, om, flux, tid, NT);
        __syncthreads();
      }
    const int n0 = L.n0, n1 = L.n1, n2 = L.n2;
    const int C1 = n1 >> 1, C2 = n2 >> 1, nc = (n0 >> 1) * C1 * C2;
    float* Bc = bt_ptrs(Ls, base, l + 1).B;
    const int sI = n1 * n2;
    const bool p2 = L.s1 >= 1 && L.s2 >= 1;
    for (int ec = tid; ec < nc; ec += NT) {
      int I, J, K;
      if (p2) {
        K = ec & (C2 - 1);
        const int t = ec >> (L.s2 - 1);
        J = t & (C1 - 1);
        I = t >> (L.s1 - 1);
      } else {
        K = ec % C2;
        const int t = ec / C2;
        J = t % C1;
        I = t / C1;
      }
      float acc = 0.f;
#pragma unroll
      for (int aa = 0; aa < 2; ++aa)
#pragma unroll
        for (int bb = 0; bb < 2; ++bb)
#pragma unroll
          for (int cc = 0; cc < 2; ++cc) {
            const int i = 2 * I + aa, j = 2 * J + bb, k = 2 * K + cc;
            const int e = (i * n1 + j) * n2 + k;
            const int fyi = (i * (n1 + 1) + j) * n2 + k, fzi = (i * n1 + j) * (n2 + 1) + k;
            const float bxl = q.X[e], bxu = q.X[e + sI], byl = q.Y[fyi], byu = q.Y[fyi + n2], bzl = q.Z[fzi],
                        bzu = q.Z[fzi + 1];
            const float pv = q.P[e];
            const float q0 = q.P[i > 0 ? e - sI : e], q1 = q.P[i < n0 - 1 ? e + sI : e];
            const float q2 = q.P[j > 0 ? e - n2 : e], q3 = q.P[j < n1 - 1 ? e + n2 : e];
            const float q4 = q.P[k > 0 ? e - 1 : e], q5 = q.P[k < n2 - 1 ? e + 1 : e];
            float Ap;
            if (flux) {
              float sm = bxl * (pv - q0);
              sm += bxu * (pv - q1);
              sm += byl * (pv - q2);
              sm += byu * (pv - q3);
              sm += bzl * (pv - q4);
              sm += bzu * (pv - q5);
              Ap = sm;
            } else {
              const float d = bxl + bxu + byl + byu + bzl + bzu;
              float sm = bxl * q0;
              sm += bxu * q1;
              sm += byl * q2;
              sm += byu * q3;
              sm += bzl * q4;
              sm += bzu * q5;
              Ap = d * pv - sm;
            }
            acc += q.B[e] - Ap;
          }
      Bc[ec] = roundT<T>(acc * rscale);
    }
    __syncthreads();
  }
  // ---- coarsest: sweeps from zero in AccT, then mean removal
  {
    const BottomLevel& L = Ls[nl - 1];
    const BtPtrs q = bt_ptrs(Ls, base, nl - 1);
    const int n = L.n0 * L.n1 * L.n2;
    for (int e = tid; e < n; e += NT) Pc[e] = AccT(0);
    __syncthreads();
    const bool one_warp = n <= 256;
    const AccT omc = (AccT)om;
    if (n <= 64 && (L.n2 & 1) == 0) {
      if (tid < 32) bt_coarsest_regs<AccT>(L, Pc, q.B, q.X, q.Y, q.Z, omc, coarsest, flux, tid);
    } else if (!one_warp || tid < 32) {
      const int nt = one_warp ? 32 : NT;
      for (int sw = 0; sw < coarsest; ++sw) {
        for (int color = 0; color < 2; ++color) {
          bt_half_sweep<AccT>(L, Pc, q.B, q.X, q.Y, q.Z, color, omc, flux, tid, nt);
          if (one_warp) __syncwarp();
          else __syncthreads();
        }
      }
    }
    __syncthreads();
    double ls = 0.0;
    for (int e = tid; e < n; e += NT) ls += (double)Pc[e];
    const double tot = block_sum<NT>(ls, sred);
    if (tid == 0) *s_mean = tot / (double)n;
    __syncthreads();
    const AccT shift = (AccT)(-*s_mean);
    for (int e = tid; e < n; e += NT) q.P[e] = roundT<T>((float)(Pc[e] + shift));
    __syncthreads();
  }
  // ---- up: prolongation, post-smoothing with the colours reversed
  for (int l = nl - 2; l >= l0; --l) {
    const BottomLevel& L = Ls[l];
    const BtPtrs q = bt_ptrs(Ls, base, l);
    const float* Pcoarse = bt_ptrs(Ls, base, l + 1).P;
    const int n = L.n0 * L.n1 * L.n2, h1 = L.n1 >> 1, h2 = L.n2 >> 1;
    for (int e = tid; e < n; e += NT) {
      int i, j, k;
      bt_ijk(L, e, i, j, k);
      q.P[e] += Pcoarse[((i >> 1) * h1 + (j >> 1)) * h2 + (k >> 1)] * pscale;
    }
    __syncthreads();
    for (int sw = 0; sw < post; ++sw)
      for (int cc = 0; cc < 2; ++cc) {
        bt_half_sweep<float>(L, q.P, q.B, q.X, q.Y, q.Z, 1 ^ cc, om, flux, tid, NT);
        __syncthreads();
      }
  }
}

template <class T, class TB, class AccT>
__global__ void __launch_bounds__(BT_NT) k_bottom(const __grid_constant__ BottomArgs<T, TB> a) {
  if (is_done(a.st)) return;
  extern __shared__ __align__(16) unsigned char btsm[];
  __shared__ double sred[40];
  __shared__ double s_mean;
  const int tid = threadIdx.x;
  const int nl = a.nl;
  // level l starts at float offset base(l); arrays P, B, X, Y, Z in that order
  auto base = [&](int l) {
    size_t off = 0;
    for (int q = 0; q < l; ++q) off += bottom_level_floats(a.L[q].n0, a.L[q].n1, a.L[q].n2);
    return reinterpret_cast<float*>(btsm) + off;
  };
  struct LvPtr {
    float *P, *B, *X, *Y, *Z;
  };
  auto ptrs = [&](int l) {
    const int n0 = a.L[l].n0, n1 = a.L[l].n1, n2 = a.L[l].n2, n = n0 * n1 * n2;
    LvPtr r;
    r.P = base(l);
    r.B = r.P + n;
    r.X = r.B + n;
    r.Y = r.X + (n0 + 1) * n1 * n2;
    r.Z = r.Y + n0 * (n1 + 1) * n2;
    return r;
  };
  AccT* Pc;
  unsigned char* stg;  // 16-bit staging (bulk == 2)
  {
    float* end = base(nl);
    Pc = reinterpret_cast<AccT*>((reinterpret_cast<uintptr_t>(end) + 15) & ~uintptr_t(15));
    const BottomLevel& Lc = a.L[nl - 1];
    stg = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(Pc + Lc.n0 * Lc.n1 * Lc.n2) + 15) & ~uintptr_t(15));
  }
  // ---- load faces of every level and b of the top level; zero p
  if (a.bulk) {
    // one thread issues a bulk copy per array (the host checked that every
    // array is 16-byte aligned and a multiple of 16 bytes long); all complete
    // on one mbarrier, waited on with a bound.  fp32 arrays land in place;
    // 16-bit arrays land back to back in the staging area and are widened
    // after the wait
    __shared__ __align__(8) uint64_t bt_bar;
    __shared__ int bt_fail;
    const bool wide = a.bulk == 1;
    constexpr unsigned kES = sizeof(T), kBS = sizeof(TB);
    if (tid == 0) {
      bt_fail = 0;
      unsigned bytes = (wide ? 4u : kBS) * (unsigned)(a.L[0].n0 * a.L[0].n1 * a.L[0].n2);
      for (int l = 0; l < nl; ++l) {
        const BottomLevel& L = a.L[l];
        bytes += (wide ? 4u : kES) *
                 (unsigned)((L.n0 + 1) * L.n1 * L.n2 + L.n0 * (L.n1 + 1) * L.n2 + L.n0 * L.n1 * (L.n2 + 1));
      }
      const unsigned bar = smem_u32(&bt_bar);
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
      auto bulk = [&](void* dst, const void* src, unsigned nbytes) {
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_u32(dst)),
            "l"(reinterpret_cast<uint64_t>(src)), "r"(nbytes), "r"(bar)
            : "memory");
      };
      unsigned char* sp = stg;
      for (int l = 0; l < nl; ++l) {
        const BottomLevel& L = a.L[l];
        const LvPtr q = ptrs(l);
        const unsigned nx = (L.n0 + 1) * L.n1 * L.n2, ny = L.n0 * (L.n1 + 1) * L.n2, nz = L.n0 * L.n1 * (L.n2 + 1);
        if (wide) {
          bulk(q.X, L.bx, 4u * nx);
          bulk(q.Y, L.by, 4u * ny);
          bulk(q.Z, L.bz, 4u * nz);
        } else {
          bulk(sp, L.bx, kES * nx);
          sp += kES * nx;
          bulk(sp, L.by, kES * ny);
          sp += kES * ny;
          bulk(sp, L.bz, kES * nz);
          sp += kES * nz;
        }
      }
      const unsigned n0c = a.L[0].n0 * a.L[0].n1 * a.L[0].n2;
      if (wide) bulk(ptrs(0).B, a.b, 4u * n0c);
      else bulk(sp, a.b, kBS * n0c);
    }
    for (int l = 0; l < nl; ++l) {
      const LvPtr q = ptrs(l);
      const int n = a.L[l].n0 * a.L[l].n1 * a.L[l].n2;
      for (int e = tid; e < n; e += BT_NT) q.P[e] = 0.f;
    }
    __syncthreads();  // barrier initialised before anyone waits on it
    {
      unsigned it = 0;
      while (!mbar_try_wait(&bt_bar, 0)) {
        if (++it > kTmaWaitLimit) {
          bt_fail = 1;
          break;
        }
      }
    }
    __syncthreads();
    if (bt_fail) {
      if (tid == 0 && a.st) {
        a.st->status = ST_TMA_TIMEOUT;
        a.st->done = 1;
      }
      unsigned it = 0;  // give the copies in flight a last bounded chance to land
      while (!mbar_try_wait(&bt_bar, 0) && ++it < kTmaWaitLimit) {
      }
      return;
    }
    if (!wide) {  // widen the staged 16-bit faces and b
      const T* sp = reinterpret_cast<const T*>(stg);
      for (int l = 0; l < nl; ++l) {
        const BottomLevel& L = a.L[l];
        const LvPtr q = ptrs(l);
        const int nf = (L.n0 + 1) * L.n1 * L.n2 + L.n0 * (L.n1 + 1) * L.n2 + L.n0 * L.n1 * (L.n2 + 1);
        for (int e = tid; e < nf; e += BT_NT) q.X[e] = ldT(sp + e);  // X, Y, Z are contiguous
        sp += nf;
      }
      const float bsc = a.b_scale ? *a.b_scale : 1.f;
      const TB* sb = reinterpret_cast<const TB*>(sp);
      const LvPtr q = ptrs(0);
      const int n0c = a.L[0].n0 * a.L[0].n1 * a.L[0].n2;
      for (int e = tid; e < n0c; e += BT_NT) q.B[e] = ldT(sb + e) * bsc;
      __syncthreads();
    }
  } else {
    for (int l = 0; l < nl; ++l) {
      const BottomLevel& L = a.L[l];
      const LvPtr q = ptrs(l);
      const int n = L.n0 * L.n1 * L.n2;
      bt_load(q.X, reinterpret_cast<const T*>(L.bx), (L.n0 + 1) * L.n1 * L.n2, 1.f, tid);
      bt_load(q.Y, reinterpret_cast<const T*>(L.by), L.n0 * (L.n1 + 1) * L.n2, 1.f, tid);
      bt_load(q.Z, reinterpret_cast<const T*>(L.bz), L.n0 * L.n1 * (L.n2 + 1), 1.f, tid);
      for (int e = tid; e < n; e += BT_NT) q.P[e] = 0.f;
    }
    {
      const LvPtr q = ptrs(0);
      bt_load(q.B, a.b, a.L[0].n0 * a.L[0].n1 * a.L[0].n2, a.b_scale ? *a.b_scale : 1.f, tid);
    }
    __syncthreads();
  }
  bt_local_vcycle<T, AccT>(a.L, reinterpret_cast<float*>(btsm), 0, nl, Pc, a.omega, a.pre, a.post, a.coarsest,
                           a.rscale, a.pscale, a.flux, sred, &s_mean);
  // ---- output (and the mean when the top level is level 0)
  const float* P0 = ptrs(0).P;
  const int n = a.L[0].n0 * a.L[0].n1 * a.L[0].n2;
  double ls = 0.0;
  for (int e = tid; e < n; e += BT_NT) {
    stT(a.p_out + e, P0[e]);
    ls += (double)roundT<T>(P0[e]);
  }
  if (a.want_mean) {
    const double tot = block_sum<BT_NT>(ls, sred);
    if (tid == 0) {
      a.st->sum_last = tot;
      a.st->c_shift = (float)(-(tot / (double)n) * (a.mixed ? (double)a.st->zscale : 1.0));
    }
  }
}

// --------------------------------------------------------------- bottom V-cycle on a CTA cluster
// The coarse end of the V-cycle from a level of up to ~32^3 cells down, in one
// launch of one cluster of BC_CTAS CTAs (distributed shared memory, no TMA).
// The finer "distributed" levels are split into slabs of s = n0/BC_CTAS
// planes along i, one slab per CTA, held in that CTA's shared memory with two
// halo planes (the neighbours' boundary planes) in two slots.  After every
// change of a slab (a half-sweep, a prolongation) each CTA writes its first
// and last plane into the other slot of its neighbours' halos (distributed
// shared memory stores), and one cluster barrier makes them visible: the next
// half-sweep reads only local shared memory, and since a half-sweep reads the
// slot the previous step wrote while the writes of its own step go to the
// other slot, one barrier per half-sweep is enough.  Restriction and prolongation between distributed
// levels stay inside a slab (s even); the coarsest distributed level
// restricts into CTA 0, which runs the remaining levels alone with
// bt_local_vcycle while the other CTAs wait at the next cluster barrier.
// Arithmetic per cell is bt_relax's and the restriction's of k_bottom, with
// the same colour orders.
constexpr int BC_CTAS = 8;
constexpr int BC_MAX_DIST = 4;
constexpr int BC_NT = 512;  // threads per CTA (128 registers a thread)
constexpr int kDenseMaxCells = 1024;  // largest level applied as a dense operator
static_assert(kDenseMaxCells / BC_CTAS <= BC_NT, "dense rows of a CTA must fit its partial-sum buffer");

template <class T, class TB> struct ClusterArgs {
  int nd;                           // distributed levels, [0] = top
  BottomLevel D[BC_MAX_DIST];
  int nl;                           // levels on CTA 0, [0] = the one below D[nd-1]
  BottomLevel L[PF_MG_MAX_LEVELS];
  const TB* b;                      // right-hand side of D[0]
  const float* b_scale;
  T* p_out;                         // solution of D[0]
  float omega;
  int pre, post, coarsest;
  float rscale, pscale;
  int flux;
  MGState* st;
  int want_mean, mixed;
  const float* M;                   // dense operator of the levels below (null: CTA 0 runs them)
  int nb;                           // its size: cells of the level below D[nd-1]
};

// floats of one CTA's slab of a distributed level: P, B (s planes), X (s+1
// face planes), Y, Z (s planes), H (2 slots x (lower, upper) halo planes)
__host__ __device__ inline size_t bc_level_floats(int n0, int n1, int n2) {
  const size_t s = (size_t)(n0 / BC_CTAS);
  return 2 * s * n1 * n2 + (s + 1) * n1 * n2 + s * (n1 + 1) * n2 + s * n1 * (n2 + 1) + 4 * (size_t)n1 * n2;
}

// one CTA's slab of a distributed level: planes i0 .. i0+s-1; Plo / Phi point
// at the current halo slot's copies of the last plane of the CTA below and the
// first plane of the CTA above (unused at the domain walls)
struct DLv {
  float *P, *B, *X, *Y, *Z, *H;
  const float* Plo;
  const float* Phi;
  int n0, n1, n2, s, i0;
  int s1, s2;  // log2(n1), log2(n2) when both are powers of two, else -1
  __device__ __forceinline__ void use_slot(int slot) {
    Plo = H + (2 * slot) * n1 * n2;
    Phi = Plo + n1 * n2;
  }
};

__device__ __forceinline__ DLv bc_level(const BottomLevel* D, float* base, int l, int rank,
                                        cooperative_groups::cluster_group& cl) {
  size_t off = 0;
  for (int q = 0; q < l; ++q) off += bc_level_floats(D[q].n0, D[q].n1, D[q].n2);
  DLv v;
  v.n0 = D[l].n0;
  v.n1 = D[l].n1;
  v.n2 = D[l].n2;
  v.s = v.n0 / BC_CTAS;
  v.i0 = rank * v.s;
  v.s1 = D[l].s1;
  v.s2 = D[l].s2;
  const int pl = v.n1 * v.n2;
  v.P = base + off;
  v.B = v.P + v.s * pl;
  v.X = v.B + v.s * pl;
  v.Y = v.X + (v.s + 1) * pl;
  v.Z = v.Y + v.s * (v.n1 + 1) * v.n2;
  v.H = v.Z + v.s * v.n1 * (v.n2 + 1);
  v.use_slot(0);
  return v;
}

// write this slab's first plane into the lower neighbour's upper halo and its
// last plane into the upper neighbour's lower halo, both in `slot`
__device__ __forceinline__ void bc_push(const DLv& L, int slot, int rank, cooperative_groups::cluster_group& cl,
                                        int tid) {
  const int pl = L.n1 * L.n2;
  if (rank > 0) {
    float* dst = cl.map_shared_rank(L.H, rank - 1) + (2 * slot + 1) * pl;
    for (int e = tid; e < pl; e += BC_NT) dst[e] = L.P[e];
  }
  if (rank < BC_CTAS - 1) {
    float* dst = cl.map_shared_rank(L.H, rank + 1) + (2 * slot) * pl;
    const float* src = L.P + (L.s - 1) * pl;
    for (int e = tid; e < pl; e += BC_NT) dst[e] = src[e];
  }
}

// b - A p at slab cell (li, j, k): k_bottom's restriction arithmetic, walls clamped
__device__ __forceinline__ float bc_residual(const DLv& L, int li, int j, int k, int flux) {
  const int n1 = L.n1, n2 = L.n2, sI = n1 * n2, i = L.i0 + li;
  const int e = (li * n1 + j) * n2 + k, e2 = j * n2 + k;
  const int fyi = (li * (n1 + 1) + j) * n2 + k, fzi = (li * n1 + j) * (n2 + 1) + k;
  const float bxl = L.X[e], bxu = L.X[e + sI], byl = L.Y[fyi], byu = L.Y[fyi + n2], bzl = L.Z[fzi],
              bzu = L.Z[fzi + 1];
  const float* P = L.P;
  const float pv = P[e];
  const float q0 = li > 0 ? P[e - sI] : (i > 0 ? L.Plo[e2] : pv);
  const float q1 = li < L.s - 1 ? P[e + sI] : (i < L.n0 - 1 ? L.Phi[e2] : pv);
  const float q2 = P[j > 0 ? e - n2 : e], q3 = P[j < n1 - 1 ? e + n2 : e];
  const float q4 = P[k > 0 ? e - 1 : e], q5 = P[k < n2 - 1 ? e + 1 : e];
  float Ap;
  if (flux) {
    float sm = bxl * (pv - q0);
    sm += bxu * (pv - q1);
    sm += byl * (pv - q2);
    sm += byu * (pv - q3);
    sm += bzl * (pv - q4);
    sm += bzu * (pv - q5);
    Ap = sm;
  } else {
    const float d = bxl + bxu + byl + byu + bzl + bzu;
    float sm = bxl * q0;
    sm += bxu * q1;
    sm += byl * q2;
    sm += byu * q3;
    sm += bzl * q4;
    sm += bzu * q5;
    Ap = d * pv - sm;
  }
  return L.B[e] - Ap;
}

// in-place relax of slab cell (li, j, k): bt_relax's arithmetic
__device__ __forceinline__ void bc_relax(const DLv& L, int li, int j, int k, float omega, int flux) {
  const int n1 = L.n1, n2 = L.n2, sI = n1 * n2, i = L.i0 + li;
  const int e = (li * n1 + j) * n2 + k, e2 = j * n2 + k;
  const int fyi = (li * (n1 + 1) + j) * n2 + k, fzi = (li * n1 + j) * (n2 + 1) + k;
  const float bxl = L.X[e], bxu = L.X[e + sI], byl = L.Y[fyi], byu = L.Y[fyi + n2], bzl = L.Z[fzi],
              bzu = L.Z[fzi + 1];
  const float d = L.X[e] + L.X[e + sI] + L.Y[fyi] + L.Y[fyi + n2] + L.Z[fzi] + L.Z[fzi + 1];
  if (!(d > 0.f)) return;
  float* P = L.P;
  const float pv = P[e];
  const float q0 = li > 0 ? P[e - sI] : (i > 0 ? L.Plo[e2] : pv);
  const float q1 = li < L.s - 1 ? P[e + sI] : (i < L.n0 - 1 ? L.Phi[e2] : pv);
  const float q2 = P[j > 0 ? e - n2 : e], q3 = P[j < n1 - 1 ? e + n2 : e];
  const float q4 = P[k > 0 ? e - 1 : e], q5 = P[k < n2 - 1 ? e + 1 : e];
  float res;
  if (flux) {
    float sum = bxl * (pv - q0);
    sum += bxu * (pv - q1);
    sum += byl * (pv - q2);
    sum += byu * (pv - q3);
    sum += bzl * (pv - q4);
    sum += bzu * (pv - q5);
    res = L.B[e] - sum;
  } else {
    float sum = bxl * q0;
    sum += bxu * q1;
    sum += byl * q2;
    sum += byu * q3;
    sum += bzl * q4;
    sum += bzu * q5;
    res = L.B[e] - (d * pv - sum);
  }
  P[e] = pv + __fdividef(omega * res, d);  // as gs_update
}

// the cells of `color` in this CTA's slab (n2 even: two cells per k pair);
// shift indexing when n1 and n2 are powers of two
__device__ __forceinline__ void bc_half_sweep(const DLv& L, int color, float omega, int flux, int tid) {
  const int hk = L.n2 >> 1, hn = L.s * L.n1 * hk;
  if (L.s1 >= 0 && L.s2 >= 1) {
    const int sh = L.s2 - 1, hm = hk - 1, jm = L.n1 - 1;
    for (int e = tid; e < hn; e += BC_NT) {
      const int h = e & hm, row = e >> sh, j = row & jm, li = row >> L.s1;
      const int k = 2 * h + ((color - (L.i0 + li) - j) & 1);
      bc_relax(L, li, j, k, omega, flux);
    }
  } else {
    for (int e = tid; e < hn; e += BC_NT) {
      const int h = e % hk, row = e / hk, j = row % L.n1, li = row / L.n1;
      const int k = 2 * h + ((color - (L.i0 + li) - j) & 1);
      bc_relax(L, li, j, k, omega, flux);
    }
  }
}

// dst[e] = src[e] for e < n: FP32 arrays by 4-byte cp.async (completed by the
// caller's cp.async.wait_all), 16-bit arrays widened through registers
template <class S>
__device__ __forceinline__ void bc_load(float* dst, const S* src, int n, int tid) {
  if constexpr (std::is_same<S, float>::value) {
    for (int e = tid; e < n; e += BC_NT)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst + e)),
                   "l"(src + e)
                   : "memory");
  } else {
    bt_load<S, BC_NT>(dst, src, n, 1.f, tid);
  }
}

template <class T, class TB, class AccT>
__global__ void __cluster_dims__(BC_CTAS, 1, 1) __launch_bounds__(BC_NT, 1) k_bottom_cluster(ClusterArgs<T, TB> a) {
  if (is_done(a.st)) return;  // the flag is the same for every CTA of the launch
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char bcsm[];
  __shared__ double sred[40];
  __shared__ double s_mean;
  __shared__ double s_part[BC_CTAS];
  const int tid = threadIdx.x;
  const int rank = (int)cl.block_rank();
  const int nd = a.nd, nl = a.nl;
  float* base = reinterpret_cast<float*>(bcsm);
  float* lbase = base;  // after the slabs (the layout is the same in every CTA)
  for (int l = 0; l < nd; ++l) lbase += bc_level_floats(a.D[l].n0, a.D[l].n1, a.D[l].n2);
  auto align16 = [](float* p) {
    return reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15));
  };
  // dense bottom: the full right-hand side of the level below, this CTA's rows
  // of its solution and the partial sums of the product; otherwise CTA 0's
  // levels and the coarsest solution
  const bool dense = a.M != nullptr;
  float* bfull = align16(lbase);
  float* pd = align16(bfull + a.nb);
  float* red = align16(pd + a.nb / BC_CTAS);
  AccT* Pc;
  {
    float* end = lbase;
    for (int l = 0; l < nl; ++l) end += bottom_level_floats(a.L[l].n0, a.L[l].n1, a.L[l].n2);
    Pc = reinterpret_cast<AccT*>((reinterpret_cast<uintptr_t>(end) + 15) & ~uintptr_t(15));
  }
  const float om = a.omega;

  // ---- load: this CTA's slab of every distributed level, b of the top one;
  // CTA 0 also the faces of its own levels; every P (and B below the top) zero
  for (int l = 0; l < nd; ++l) {
    const BottomLevel& G = a.D[l];
    const DLv L = bc_level(a.D, base, l, rank, cl);
    const int pl = G.n1 * G.n2;
    bc_load(L.X, reinterpret_cast<const T*>(G.bx) + (size_t)L.i0 * pl, (L.s + 1) * pl, tid);
    bc_load(L.Y, reinterpret_cast<const T*>(G.by) + (size_t)L.i0 * (G.n1 + 1) * G.n2, L.s * (G.n1 + 1) * G.n2, tid);
    bc_load(L.Z, reinterpret_cast<const T*>(G.bz) + (size_t)L.i0 * G.n1 * (G.n2 + 1), L.s * G.n1 * (G.n2 + 1), tid);
    for (int e = tid; e < L.s * pl; e += BC_NT) {
      L.P[e] = 0.f;
      if (l > 0) L.B[e] = 0.f;
    }
    for (int e = tid; e < 4 * pl; e += BC_NT) L.H[e] = 0.f;
  }
  {
    const DLv L = bc_level(a.D, base, 0, rank, cl);
    const int cnt = L.s * L.n1 * L.n2;
    const TB* src = a.b + (size_t)L.i0 * L.n1 * L.n2;
    if (a.b_scale) bt_load<TB, BC_NT>(L.B, src, cnt, *a.b_scale, tid);
    else bc_load(L.B, src, cnt, tid);
  }
  if (rank == 0 && !dense) {
    for (int l = 0; l < nl; ++l) {
      const BottomLevel& G = a.L[l];
      const BtPtrs q = bt_ptrs(a.L, lbase, l);
      const int n = G.n0 * G.n1 * G.n2;
      bc_load(q.X, reinterpret_cast<const T*>(G.bx), (G.n0 + 1) * G.n1 * G.n2, tid);
      bc_load(q.Y, reinterpret_cast<const T*>(G.by), G.n0 * (G.n1 + 1) * G.n2, tid);
      bc_load(q.Z, reinterpret_cast<const T*>(G.bz), G.n0 * G.n1 * (G.n2 + 1), tid);
      for (int e = tid; e < n; e += BC_NT) q.P[e] = q.B[e] = 0.f;
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  cl.sync();

  // ---- down the distributed levels: pre-smoothing, residual, restriction
  int cur[BC_MAX_DIST];  // halo slot holding each level's current boundary planes
  for (int l = 0; l < nd; ++l) {
    DLv L = bc_level(a.D, base, l, rank, cl);
    cur[l] = 0;
    for (int sw = 0; sw < a.pre; ++sw)
      for (int cc = 0; cc < 2; ++cc) {
        L.use_slot(cur[l]);
        bc_half_sweep(L, cc, om, a.flux, tid);
        __syncthreads();  // the slab's half-sweep done before its boundary planes go out
        cur[l] ^= 1;
        bc_push(L, cur[l], rank, cl, tid);
        cl.sync();
      }
    L.use_slot(cur[l]);
    // coarse planes rank*s/2 .. : into the next slab, or into CTA 0's first
    // level, or (dense) into every CTA's copy of the full right-hand side
    const int C1 = L.n1 >> 1, C2 = L.n2 >> 1, hs = L.s >> 1, nc = hs * C1 * C2;
    const bool last = l + 1 == nd;
    float* Bc = !last ? bc_level(a.D, base, l + 1, rank, cl).B
                      : dense ? bfull + (size_t)rank * nc : cl.map_shared_rank(bt_ptrs(a.L, lbase, 0).B, 0) + (size_t)rank * nc;
    const bool p2 = L.s1 >= 1 && L.s2 >= 1;
    for (int ec = tid; ec < nc; ec += BC_NT) {
      int I, J, K;
      if (p2) {
        K = ec & (C2 - 1);
        const int t = ec >> (L.s2 - 1);
        J = t & (C1 - 1);
        I = t >> (L.s1 - 1);
      } else {
        K = ec % C2;
        const int t = ec / C2;
        J = t % C1;
        I = t / C1;
      }
      float acc = 0.f;
#pragma unroll
      for (int aa = 0; aa < 2; ++aa)
#pragma unroll
        for (int bb = 0; bb < 2; ++bb)
#pragma unroll
          for (int c2 = 0; c2 < 2; ++c2) acc += bc_residual(L, 2 * I + aa, 2 * J + bb, 2 * K + c2, a.flux);
      const float v = roundT<T>(acc * a.rscale);
      if (last && dense) {
        for (int r = 0; r < BC_CTAS; ++r) cl.map_shared_rank(Bc, r)[ec] = v;
      } else {
        Bc[ec] = v;
      }
    }
    cl.sync();
  }

  // ---- the levels below: the dense operator's rows of this CTA's coarse
  // planes (partial sums over column chunks, added in chunk order), or CTA 0
  if (dense) {
    const int nb = a.nb, R = nb / BC_CTAS, row0 = rank * R;
    const int ch = R >= BC_NT ? 1 : BC_NT / R;  // column chunks per row
    const int cw = (nb + ch - 1) / ch;
    for (int t = tid; t < R * ch; t += BC_NT) {
      const int i = t % R, c = t / R;
      const int m0 = c * cw, m1 = min(nb, m0 + cw);
      float acc = 0.f;
      for (int m = m0; m < m1; ++m) acc = fmaf(__ldg(a.M + (size_t)m * nb + row0 + i), bfull[m], acc);
      red[t] = acc;
    }
    __syncthreads();
    for (int i = tid; i < R; i += BC_NT) {
      float v = 0.f;
      for (int c = 0; c < ch; ++c) v += red[c * R + i];
      pd[i] = v;
    }
    __syncthreads();
  } else {
    if (rank == 0)
      bt_local_vcycle<T, AccT, BC_NT>(a.L, lbase, 0, nl, Pc, om, a.pre, a.post, a.coarsest, a.rscale, a.pscale,
                                      a.flux, sred, &s_mean);
    cl.sync();
  }

  // ---- up the distributed levels: prolongation, post-smoothing with the colours reversed
  for (int l = nd - 1; l >= 0; --l) {
    DLv L = bc_level(a.D, base, l, rank, cl);
    const int h1 = L.n1 >> 1, h2 = L.n2 >> 1, n = L.s * L.n1 * L.n2;
    const float* Pcoarse;
    int cplane0;  // global plane of Pcoarse's first plane
    if (l + 1 < nd) {
      Pcoarse = bc_level(a.D, base, l + 1, rank, cl).P;
      cplane0 = L.i0 >> 1;
    } else if (dense) {
      Pcoarse = pd;
      cplane0 = rank * (L.s >> 1);
    } else {
      Pcoarse = cl.map_shared_rank(bt_ptrs(a.L, lbase, 0).P, 0);
      cplane0 = 0;
    }
    const bool p2 = L.s1 >= 0 && L.s2 >= 0;
    for (int e = tid; e < n; e += BC_NT) {
      int k, j, li;
      if (p2) {
        k = e & (L.n2 - 1);
        const int t = e >> L.s2;
        j = t & (L.n1 - 1);
        li = t >> L.s1;
      } else {
        k = e % L.n2;
        const int t = e / L.n2;
        j = t % L.n1;
        li = t / L.n1;
      }
      const int I = ((L.i0 + li) >> 1) - cplane0;
      L.P[e] += Pcoarse[(I * h1 + (j >> 1)) * h2 + (k >> 1)] * a.pscale;
    }
    __syncthreads();  // the whole slab prolongated before its boundary planes go out
    cur[l] ^= 1;
    bc_push(L, cur[l], rank, cl, tid);
    cl.sync();
    for (int sw = 0; sw < a.post; ++sw)
      for (int cc = 0; cc < 2; ++cc) {
        L.use_slot(cur[l]);
        bc_half_sweep(L, 1 ^ cc, om, a.flux, tid);
        __syncthreads();
        cur[l] ^= 1;
        bc_push(L, cur[l], rank, cl, tid);
        cl.sync();
      }
  }

  // ---- output (and the mean when the top level is level 0)
  {
    const DLv L = bc_level(a.D, base, 0, rank, cl);
    const int cnt = L.s * L.n1 * L.n2;
    T* out = a.p_out + (size_t)L.i0 * L.n1 * L.n2;
    double ls = 0.0;
    for (int e = tid; e < cnt; e += BC_NT) {
      stT(out + e, L.P[e]);
      ls += (double)roundT<T>(L.P[e]);
    }
    if (a.want_mean) {
      const double bs = block_sum<BC_NT>(ls, sred);
      if (tid == 0) *cl.map_shared_rank(&s_part[rank], 0) = bs;
    }
  }
  cl.sync();  // also: no CTA leaves while another may still read its shared memory
  if (a.want_mean && rank == 0 && tid == 0) {
    double tot = 0.0;
    for (int r = 0; r < BC_CTAS; ++r) tot += s_part[r];
    const int n = a.D[0].n0 * a.D[0].n1 * a.D[0].n2;
    a.st->sum_last = tot;
    a.st->c_shift = (float)(-(tot / (double)n) * (a.mixed ? (double)a.st->zscale : 1.0));
  }
}

// ---- the dense bottom operator, one column per CTA: the V-cycle of the
// levels below the cluster's slabs (bt_local_vcycle, DB_NT threads) applied to
// the unit right-hand side e_m, written to M[m * nb + i]
constexpr int DB_NT = 128;

template <class T> struct DenseBuildArgs {
  int nl;
  BottomLevel L[PF_MG_MAX_LEVELS];
  float* M;
  float omega;
  int pre, post, coarsest;
  float rscale, pscale;
  int flux;
};

template <class T, class AccT>
__global__ void __launch_bounds__(DB_NT) k_bottom_dense_build(const __grid_constant__ DenseBuildArgs<T> a) {
  extern __shared__ __align__(16) unsigned char dbsm[];
  __shared__ double sred[40];
  __shared__ double s_mean;
  const int tid = threadIdx.x, m = blockIdx.x;
  float* base = reinterpret_cast<float*>(dbsm);
  AccT* Pc;
  {
    float* end = base;
    for (int l = 0; l < a.nl; ++l) end += bottom_level_floats(a.L[l].n0, a.L[l].n1, a.L[l].n2);
    Pc = reinterpret_cast<AccT*>((reinterpret_cast<uintptr_t>(end) + 15) & ~uintptr_t(15));
  }
  for (int l = 0; l < a.nl; ++l) {
    const BottomLevel& G = a.L[l];
    const BtPtrs q = bt_ptrs(a.L, base, l);
    const int n = G.n0 * G.n1 * G.n2;
    bt_load<T, DB_NT>(q.X, reinterpret_cast<const T*>(G.bx), (G.n0 + 1) * G.n1 * G.n2, 1.f, tid);
    bt_load<T, DB_NT>(q.Y, reinterpret_cast<const T*>(G.by), G.n0 * (G.n1 + 1) * G.n2, 1.f, tid);
    bt_load<T, DB_NT>(q.Z, reinterpret_cast<const T*>(G.bz), G.n0 * G.n1 * (G.n2 + 1), 1.f, tid);
    for (int e = tid; e < n; e += DB_NT) {
      q.P[e] = 0.f;
      q.B[e] = (l == 0 && e == m) ? 1.f : 0.f;
    }
  }
  __syncthreads();
  bt_local_vcycle<T, AccT, DB_NT>(a.L, base, 0, a.nl, Pc, a.omega, a.pre, a.post, a.coarsest, a.rscale, a.pscale,
                                  a.flux, sred, &s_mean);
  const float* P0 = bt_ptrs(a.L, base, 0).P;
  const int nb = a.L[0].n0 * a.L[0].n1 * a.L[0].n2;
  for (int i = tid; i < nb; i += DB_NT) a.M[(size_t)m * nb + i] = P0[i];
}

// --------------------------------------------------------------- CG vector kernels
// Sum of b (for the mean); last CTA stores c_shift = float(-sum/n).
__global__ void __launch_bounds__(RED_NT) k_sum_mean(long long n, const float* __restrict__ x, double* partials,
                                                     unsigned* counter, MGState* st) {
  __shared__ double sh[40];
  double s = 0.0;
  for (long long e = blockIdx.x * (long long)RED_NT + threadIdx.x; e < n; e += (long long)gridDim.x * RED_NT)
    s += (double)x[e];
  s = block_sum<RED_NT>(s, sh);
  double tot;
  if (grid_sum_last<RED_NT>(s, partials, counter, &tot, sh) && threadIdx.x == 0) {
    st->sum_last = tot;
    st->c_shift = (float)(-(tot / (double)n));
  }
}

// r = rhs = b + c_shift; x = 0; bnorm = max|r|; stop if bnorm == 0
// (pfflip/poisson.py:363-372)
__global__ void __launch_bounds__(RED_NT) k_init_r(long long n, const float* __restrict__ b, float* __restrict__ rhs,
                                                   float* __restrict__ r, float* __restrict__ x, double* partials,
                                                   unsigned* counter, MGState* st) {
  __shared__ float shf[40];
  const float c = st->c_shift;
  float m = 0.f;
  for (long long e = blockIdx.x * (long long)RED_NT + threadIdx.x; e < n; e += (long long)gridDim.x * RED_NT) {
    const float v = b[e] + c;
    if (rhs) rhs[e] = v;
    r[e] = v;
    x[e] = 0.f;
    m = fmaxf(m, isfinite(v) ? fabsf(v) : INFINITY);
  }
  m = block_max<RED_NT>(m, shf);
  float tot;
  if (grid_max_last<RED_NT>(m, partials, counter, &tot, shf) && threadIdx.x == 0) {
    st->bnorm = (double)tot;
    st->rel = 1.0;
    st->it = 0;
    st->status = ST_RUNNING;
    st->done = 0;
    if (!(tot > 0.f) || isinf(tot)) {
      st->done = 1;
      st->status = (tot == 0.f) ? ST_ZERO_RHS : ST_NONFINITE;
      st->rel = (tot == 0.f) ? 0.0 : 1.0;
    }
    // 16-bit hierarchy: b of level 0 is r * scale_r, a power of two putting max|r| in [0.5, 1)
    int ex = 0;
    frexpf(tot > 0.f ? tot : 1.f, &ex);
    st->scale_r = ldexpf(1.f, -ex);
  }
}

// z = p*zscale + c_shift, the preconditioned residual (pfflip/poisson.py:351-352)
template <class T>
__device__ __forceinline__ float zval(const T* p, long long e, float zs, float c) {
  return ldT(p + e) * zs + c;
}

// 4-wide loads/stores of the CG vectors (16-byte float4, 8-byte 16-bit quads)
__device__ __forceinline__ float4 ld4(const float* p, long long i4) { return reinterpret_cast<const float4*>(p)[i4]; }
__device__ __forceinline__ float4 ld4(const __half* p, long long i4) {
  const uint2 u = reinterpret_cast<const uint2*>(p)[i4];
  const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 ld4(const __nv_bfloat16* p, long long i4) {
  const uint2 u = reinterpret_cast<const uint2*>(p)[i4];
  const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
  const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void st4(float* p, long long i4, float4 v) { reinterpret_cast<float4*>(p)[i4] = v; }

// q = z; rz = <r, z>   (pfflip/poisson.py:378-380)
template <class T>
__global__ void __launch_bounds__(RED_NT) k_init_q(long long n, const T* __restrict__ p, const float* __restrict__ r,
                                                   float* __restrict__ q, float* __restrict__ zout, double* partials,
                                                   unsigned* counter, MGState* st, int mixed) {
  if (is_done(st)) return;
  __shared__ double sh[40];
  const float c = st->c_shift, zs = mixed ? st->zscale : 1.f;
  double s = 0.0;
  for (long long e = blockIdx.x * (long long)RED_NT + threadIdx.x; e < n; e += (long long)gridDim.x * RED_NT) {
    const float z = zval(p, e, zs, c);
    q[e] = z;
    if (zout) zout[e] = z;
    s += (double)r[e] * (double)z;
  }
  s = block_sum<RED_NT>(s, sh);
  double tot;
  if (grid_sum_last<RED_NT>(s, partials, counter, &tot, sh) && threadIdx.x == 0) st->rz = tot;
}

// Ap = A q; qAq = <q, Ap>; it += 1; alpha = rz/qAq or stop when qAq <= 0
// (pfflip/poisson.py:384-389)
__global__ void __launch_bounds__(C3_NT) k_apply_dot(int nx, int ny, int nz, const float* __restrict__ q,
                                                     const float* __restrict__ bx, const float* __restrict__ by,
                                                     const float* __restrict__ bz, const float* __restrict__ diag,
                                                     float* __restrict__ Ap, double* partials, unsigned* counter,
                                                     MGState* st, int flux) {
  if (is_done(st)) return;
  __shared__ double sh[40];
  const Cell3 c = cell_here();  // blockIdx.z counts groups of 4 i-planes
  double s = 0.0;
  if (c.j < ny && c.k < nz) {
#pragma unroll
    for (int di = 0; di < 4; ++di) {
      const int i = 4 * c.i + di;
      if (i >= nx) break;
      const long long e = ((long long)i * ny + c.j) * nz + c.k;
      const float v = apply_row(q, bx, by, bz, diag, nx, ny, nz, i, c.j, c.k, flux);
      Ap[e] = v;
      s += (double)q[e] * (double)v;
    }
  }
  s = block_sum<C3_NT>(s, sh);
  double tot;
  if (grid_sum_last<C3_NT>(s, partials, counter, &tot, sh) && threadIdx.x == 0) {
    st->it += 1;
    st->qAq = tot;
    if (!(tot > 0.0)) {
      st->done = 1;
      st->status = (tot <= 0.0) ? ST_BREAKDOWN : ST_NONFINITE;
    } else {
      st->alpha = st->rz / tot;
      st->alpha_f = (float)st->alpha;
      st->neg_alpha_f = (float)(-st->alpha);
    }
  }
}

// x += alpha q; r_new = r - alpha Ap (r kept as r_prev); rel = max|r_new|/bnorm
// (pfflip/poisson.py:390-398).  4-wide, grid-stride.
__global__ void __launch_bounds__(RED_NT) k_update_xr(long long n, const float* __restrict__ q,
                                                      const float* __restrict__ Ap, const float* __restrict__ r,
                                                      float* __restrict__ r_new, float* __restrict__ x,
                                                      double* partials, unsigned* counter, MGState* st) {
  if (is_done(st)) return;
  __shared__ float shf[40];
  const float af = st->alpha_f, naf = st->neg_alpha_f;
  float m = 0.f;
  const long long n4 = n >> 2, stride = (long long)gridDim.x * RED_NT;
  auto one = [&](float qv, float av, float rv, float& xv, float& rn) {
    xv += af * qv;
    rn = rv + naf * av;
    m = fmaxf(m, isfinite(rn) ? fabsf(rn) : INFINITY);
  };
  for (long long i = blockIdx.x * (long long)RED_NT + threadIdx.x; i < n4; i += stride) {
    const float4 qv = ld4(q, i), av = ld4(Ap, i), rv = ld4(r, i);
    float4 xv = ld4(x, i), rn;
    one(qv.x, av.x, rv.x, xv.x, rn.x);
    one(qv.y, av.y, rv.y, xv.y, rn.y);
    one(qv.z, av.z, rv.z, xv.z, rn.z);
    one(qv.w, av.w, rv.w, xv.w, rn.w);
    st4(x, i, xv);
    st4(r_new, i, rn);
  }
  for (long long e = 4 * n4 + blockIdx.x * (long long)RED_NT + threadIdx.x; e < n; e += stride) {
    float xv = x[e], rn;
    one(q[e], Ap[e], r[e], xv, rn);
    x[e] = xv;
    r_new[e] = rn;
  }
  m = block_max<RED_NT>(m, shf);
  float tot;
  if (grid_max_last<RED_NT>(m, partials, counter, &tot, shf) && threadIdx.x == 0) {
    const double rel = (double)tot / st->bnorm;
    st->rel = rel;
    st->maxabs_last = tot;
    if (!(rel == rel) || isinf(rel)) {
      st->done = 1;
      st->status = ST_NONFINITE;
    } else if (rel < (double)st->tol) {
      st->done = 1;
      st->status = ST_CONVERGED;
    }
    int ex = 0;
    frexpf(tot > 0.f ? tot : 1.f, &ex);
    st->scale_r = ldexpf(1.f, -ex);
  }
}

// rz_new = <r, z>, rpz = <r_prev, z>, beta = max((rz_new - rpz)/rz, 0), rz = rz_new
// (pfflip/poisson.py:402-406).  4-wide, grid-stride.
template <class T>
__global__ void __launch_bounds__(RED_NT) k_dots(long long n, const T* __restrict__ p, const float* __restrict__ r,
                                                 const float* __restrict__ r_prev, double* partials,
                                                 unsigned* counter, MGState* st, int mixed) {
  if (is_done(st)) return;
  __shared__ double sh[40];
  const float c = st->c_shift, zs = mixed ? st->zscale : 1.f;
  double s1 = 0.0, s2 = 0.0;
  const long long n4 = n >> 2, stride = (long long)gridDim.x * RED_NT;
  auto one = [&](float pv, float rv, float qv) {
    const double z = (double)(pv * zs + c);
    s1 += (double)rv * z;
    s2 += (double)qv * z;
  };
  for (long long i = blockIdx.x * (long long)RED_NT + threadIdx.x; i < n4; i += stride) {
    const float4 pv = ld4(p, i), rv = ld4(r, i), qv = ld4(r_prev, i);
    one(pv.x, rv.x, qv.x);
    one(pv.y, rv.y, qv.y);
    one(pv.z, rv.z, qv.z);
    one(pv.w, rv.w, qv.w);
  }
  for (long long e = 4 * n4 + blockIdx.x * (long long)RED_NT + threadIdx.x; e < n; e += stride)
    one(ldT(p + e), r[e], r_prev[e]);
  s1 = block_sum<RED_NT>(s1, sh);
  s2 = block_sum<RED_NT>(s2, sh);
  double t1, t2;
  if (grid_sum2_last<RED_NT>(s1, s2, partials, counter, &t1, &t2, sh) && threadIdx.x == 0) {
    const double num = t1 - t2;
    const double beta = (st->rz != 0.0) ? fmax(num / st->rz, 0.0) : 0.0;
    st->rz_new = t1;
    st->rpz = t2;
    st->beta = beta;
    st->beta_f = (float)beta;
    st->rz = t1;
  }
}

// q = z + beta q   (pfflip/poisson.py:405, scale_add).  4-wide, grid-stride.
template <class T>
__global__ void __launch_bounds__(RED_NT) k_update_q(long long n, const T* __restrict__ p, float* __restrict__ q,
                                                     MGState* st, int mixed) {
  if (is_done(st)) return;
  const float c = st->c_shift, zs = mixed ? st->zscale : 1.f, bf = st->beta_f;
  const long long n4 = n >> 2, stride = (long long)gridDim.x * RED_NT;
  for (long long i = blockIdx.x * (long long)RED_NT + threadIdx.x; i < n4; i += stride) {
    const float4 pv = ld4(p, i);
    float4 qv = ld4(q, i);
    qv.x = (pv.x * zs + c) + bf * qv.x;
    qv.y = (pv.y * zs + c) + bf * qv.y;
    qv.z = (pv.z * zs + c) + bf * qv.z;
    qv.w = (pv.w * zs + c) + bf * qv.w;
    st4(q, i, qv);
  }
  for (long long e = 4 * n4 + blockIdx.x * (long long)RED_NT + threadIdx.x; e < n; e += stride)
    q[e] = zval(p, e, zs, c) + bf * q[e];
}

// z = p*zscale + c_shift written out (precondition entry point)
template <class T>
__global__ void k_write_z(long long n, const T* __restrict__ p, float* __restrict__ z, const MGState* st, int mixed) {
  const float c = st->c_shift, zs = mixed ? st->zscale : 1.f;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    z[e] = zval(p, e, zs, c);
}

// final mean removal of x written into the caller's output (pfflip/poisson.py:408)
__global__ void k_shift_out(long long n, const float* __restrict__ x, float* __restrict__ out, const MGState* st) {
  const float c = st->c_shift;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    out[e] = x[e] + c;
}

__global__ void k_set_state(MGState* st, float tol, int max_iter, float zscale_base) {
  st->tol = tol;
  st->max_iter = max_iter;
  st->done = 0;
  st->status = ST_RUNNING;
  st->it = 0;
  st->rel = 1.0;
  st->zscale = zscale_base;  // multiplied by 1/scale_r where used
}

// zscale = zscale_base / scale_r (16-bit hierarchy)
__global__ void k_update_zscale(MGState* st, float coef_scale) {
  st->zscale = coef_scale / st->scale_r;
}

__global__ void k_copy_f(long long n, const float* __restrict__ a, float* __restrict__ b) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    b[e] = a[e];
}


// generic mean of a level-0 vector stored as T: c_shift = float(-mean * zscale)
template <class T>
__global__ void __launch_bounds__(RED_NT) k_mean_of(long long n, const T* __restrict__ p, double* partials,
                                                    unsigned* counter, MGState* st, int mixed) {
  __shared__ double sh[40];
  double s = 0.0;
  for (long long e = blockIdx.x * (long long)RED_NT + threadIdx.x; e < n; e += (long long)gridDim.x * RED_NT)
    s += (double)ldT(p + e);
  s = block_sum<RED_NT>(s, sh);
  double tot;
  if (grid_sum_last<RED_NT>(s, partials, counter, &tot, sh) && threadIdx.x == 0) {
    st->sum_last = tot;
    st->c_shift = (float)(-(tot / (double)n) * (mixed ? (double)st->zscale : 1.0));
  }
}

// p += float(-mean(p)) in place (mean from st->sum_last; coarsest-level fallback)
template <class T>
__global__ void k_shift_mean_inplace(long long n, T* __restrict__ p, const MGState* st) {
  const float c = (float)(-(st->sum_last / (double)n));
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    stT(p + e, ldT(p + e) + c);
}

// fine p += pscale * coarse p[i/2, j/2, k/2]   (pfflip/poisson.py:178-182)
template <class T>
__global__ void k_prolong_add(int n0, int n1, int n2, const T* __restrict__ pc, T* __restrict__ p, float pscale,
                              const MGState* st) {
  if (is_done(st)) return;
  const long long n = (long long)n0 * n1 * n2;
  const int h1 = n1 >> 1, h2 = n2 >> 1;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(e % n2);
    const long long t = e / n2;
    const int j = (int)(t % n1), i = (int)(t / n1);
    stT(p + e, ldT(p + e) + ldT(pc + ((long long)(i >> 1) * h1 + (j >> 1)) * h2 + (k >> 1)) * pscale);
  }
}

// max|r| -> scale_r and zscale (precondition entry point, 16-bit hierarchy)
__global__ void __launch_bounds__(RED_NT) k_scale_of(long long n, const float* __restrict__ r, double* partials,
                                                     unsigned* counter, MGState* st, float coef_scale) {
  __shared__ float shf[40];
  float m = 0.f;
  for (long long e = blockIdx.x * (long long)RED_NT + threadIdx.x; e < n; e += (long long)gridDim.x * RED_NT)
    m = fmaxf(m, fabsf(r[e]));
  m = block_max<RED_NT>(m, shf);
  float tot;
  if (grid_max_last<RED_NT>(m, partials, counter, &tot, shf) && threadIdx.x == 0) {
    int ex = 0;
    frexpf(tot > 0.f && isfinite(tot) ? tot : 1.f, &ex);
    st->scale_r = ldexpf(1.f, -ex);
    st->zscale = coef_scale / st->scale_r;
  }
}

__global__ void k_clear_done(MGState* st) {
  st->done = 0;
  st->status = ST_RUNNING;
}

// =============================================================== host side
void count_suppress(bool on);

}  // namespace pf

struct pf_mg_plan {
  pf_mg_desc d;
  int prec;
  float lp_scale[PF_MG_MAX_LEVELS];
  int lb;              // first level solved by the single-CTA bottom kernel (nlev = none)
  bool use_tma;        // stage fp32 smoother tiles with TMA where the level allows it
  int sms;             // multiprocessors of the plan's device (persistent sweep grid)
  size_t bottom_smem;  // dynamic shared memory of the bottom kernel
  bool bottom_stage;   // bottom_smem includes the 16-bit staging area
  int bc_nd;           // > 0: levels lb .. lb+bc_nd-1 run distributed on a CTA cluster (k_bottom_cluster)
  size_t bc_smem;      // dynamic shared memory per CTA of the cluster kernel
  int dense_nb;        // > 0: the levels below the slabs run as a dense nb x nb operator in bottom_op
  float* bottom_op;
  cudaStream_t cap_stream;
  cudaGraphExec_t exec[2];
  size_t exec_nodes[2];
  bool graphs_ready;
  pf::MGState* h_state[2];
  cudaEvent_t ev[2];
};

namespace {
using namespace pf;

inline MGState* ST(pf_mg_plan* P) { return reinterpret_cast<MGState*>(P->d.state); }
inline unsigned* CNT(pf_mg_plan* P, int k) { return P->d.counters + k; }
inline float* scale_r_ptr(pf_mg_plan* P) { return &ST(P)->scale_r; }
inline long long ncells(const pf_mg_level& L) { return (long long)L.nx * L.ny * L.nz; }
inline bool mixed(const pf_mg_plan* P) { return P->prec != PF_PREC_FP32; }
inline int FLUX(const pf_mg_plan* P) { return P->d.stencil == PF_STENCIL_FLUX ? 1 : 0; }

template <class T> struct LV { T *bx, *by, *bz, *p0, *p1, *b; };

template <class T> LV<T> view(pf_mg_plan* P, int lv) {
  const pf_mg_level& L = P->d.lev[lv];
  if (P->prec == PF_PREC_FP32)
    return LV<T>{(T*)L.bx, (T*)L.by, (T*)L.bz, (T*)L.p, (T*)L.p_alt, (T*)L.b};
  return LV<T>{(T*)L.bx_lp, (T*)L.by_lp, (T*)L.bz_lp, (T*)L.p_lp, (T*)L.p_lp_alt, (T*)L.b_lp};
}

// about 8 CTAs per SM: each thread runs several elements of a grid-stride
// loop, so several loads are in flight per thread
int red_grid(long long n) { return grid_for(n, RED_NT, kNumSMs * 8); }
// 4-wide grid-stride kernels of the CG iteration (k_update_xr, k_dots,
// k_update_q): about 4 CTAs per SM, so the last CTA of a reduction sums half
// as many partials (128^3 solve 9.12 -> 8.90 ms against 8 CTAs per SM)
int vec_grid(long long n) { return grid_for((n + 3) / 4, RED_NT, kNumSMs * 4); }
int ew_grid(long long n) { return grid_for(n, 256, 1 << 20); }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(ptr);
    cudaGetLastError();
  }
  return fn;
}

// 3D tensor of dtype (esize bytes per element): extents (d0 innermost, d1,
// d2), row pitch and plane pitch in elements
bool encode3d_t(CUtensorMap* m, CUtensorMapDataType dtype, uint32_t esize, const void* base, uint64_t d0, uint64_t d1,
                uint64_t d2, uint64_t row_pitch, uint64_t plane_pitch, uint32_t b0, uint32_t b1, uint32_t b2) {
  EncodeTiledFn fn = encode_fn();
  if (!fn || !aligned16(base) || (row_pitch * esize) % 16 || (plane_pitch * esize) % 16 || (b0 * esize) % 16)
    return false;
  cuuint64_t dims[3] = {d0, d1, d2};
  cuuint64_t strides[2] = {row_pitch * esize, plane_pitch * esize};
  cuuint32_t box[3] = {b0, b1, b2};
  cuuint32_t es[3] = {1, 1, 1};
  return fn(m, dtype, 3, const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 3D fp32 tensor: extents (d0 innermost, d1, d2), row pitch and plane pitch in floats
bool encode3d(CUtensorMap* m, const void* base, uint64_t d0, uint64_t d1, uint64_t d2, uint64_t row_pitch,
              uint64_t plane_pitch, uint32_t b0, uint32_t b1, uint32_t b2) {
  return encode3d_t(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, d0, d1, d2, row_pitch, plane_pitch, b0, b1, b2);
}

// TMA staging of a level: fp32 storage, rows a multiple of 4 floats, padded z-faces
template <int TI, class T, class TB>
bool tma_maps(pf_mg_plan* P, int lv, const T* p_in, const TB* b, const float* b_scale, const LV<T>& V, TileMaps* m) {
  if constexpr (!std::is_same<T, float>::value || !std::is_same<TB, float>::value) {
    return false;
  } else {
    const pf_mg_level& L = P->d.lev[lv];
    if (b_scale || !L.bz_pad || L.nz % 4 != 0 || L.bz_pitch % 8 != 0) return false;
    const uint64_t n0 = L.nx, n1 = L.ny, n2 = L.nz;
    const float* pm = p_in ? p_in : V.p0;
    return encode3d(&m->p, pm, n2, n1, n0, n2, n1 * n2, TM_W, SW_TJ + 4, TI + 4) &&
           encode3d(&m->b, b, n2, n1, n0, n2, n1 * n2, TM_W, SW_TJ + 2, TI + 2) &&
           encode3d(&m->x, V.bx, n2, n1, n0 + 1, n2, n1 * n2, TM_W, SW_TJ + 2, TI + 3) &&
           encode3d(&m->y, V.by, n2, n1 + 1, n0, n2, (n1 + 1) * n2, TM_W, SW_TJ + 3, TI + 2) &&
           encode3d(&m->z, L.bz_pad, n2 + 1, n1, n0, (uint64_t)L.bz_pitch, n1 * (uint64_t)L.bz_pitch, TM_W,
                    SW_TJ + 2, TI + 2);
  }
}

// TMA staging of a 16-bit level: rows a multiple of 8 elements (16 bytes), the
// padded 16-bit z-faces in bz_pad; b is the fp32 residual (finest level, with
// its scale) or 16-bit
template <int TI, class T, class TB>
bool tma_maps16(pf_mg_plan* P, int lv, const T* p_in, const TB* b, const LV<T>& V, TileMaps* m) {
  if constexpr (std::is_same<T, float>::value) {
    return false;
  } else {
    const pf_mg_level& L = P->d.lev[lv];
    if (!L.bz_pad || L.nz % 8 != 0 || L.bz_pitch % 8 != 0) return false;
    const CUtensorMapDataType dt =
        std::is_same<T, __half>::value ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    const uint64_t n0 = L.nx, n1 = L.ny, n2 = L.nz;
    const T* pm = p_in ? p_in : V.p0;
    bool ok = encode3d_t(&m->p, dt, 2, pm, n2, n1, n0, n2, n1 * n2, TM16_W, SW_TJ + 4, TI + 4);
    if constexpr (std::is_same<TB, float>::value)
      ok = ok && encode3d(&m->b, b, n2, n1, n0, n2, n1 * n2, TM_W, SW_TJ + 2, TI + 2);
    else
      ok = ok && encode3d_t(&m->b, dt, 2, b, n2, n1, n0, n2, n1 * n2, TM16_W, SW_TJ + 2, TI + 2);
    return ok && encode3d_t(&m->x, dt, 2, V.bx, n2, n1, n0 + 1, n2, n1 * n2, TM16_W, SW_TJ + 2, TI + 3) &&
           encode3d_t(&m->y, dt, 2, V.by, n2, n1 + 1, n0, n2, (n1 + 1) * n2, TM16_W, SW_TJ + 3, TI + 2) &&
           encode3d_t(&m->z, dt, 2, L.bz_pad, n2 + 1, n1, n0, (uint64_t)L.bz_pitch, n1 * (uint64_t)L.bz_pitch,
                      TM16_W, SW_TJ + 2, TI + 2);
  }
}

// launch that may overlap the end of the kernel before it on the stream
// (programmatic dependent launch); the kernel must call griddepcontrol.wait
// before it reads anything an earlier kernel writes
template <class... KArgs, class... Args>
cudaError_t launch_overlapped(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

template <class T, class TB>
int launch_sweep(pf_mg_plan* P, int lv, const T* p_in, bool zero_in, T* p_out, const TB* b, const float* b_scale,
                 const LV<T>& V, const T* pc, float pc_scale, int first_color, bool mean, bool use_state,
                 cudaStream_t s) {
  const pf_mg_level& L = P->d.lev[lv];
  SweepArgs<T, TB> a;
  a.n0 = L.nx; a.n1 = L.ny; a.n2 = L.nz;
  a.p_in = p_in; a.zero_in = zero_in ? 1 : 0; a.p_out = p_out;
  a.b = b; a.b_scale = b_scale;
  a.bx = V.bx; a.by = V.by; a.bz = V.bz;
  a.pc = pc; a.pc_scale = pc_scale;
  a.omega = P->d.omega;
  a.first_color = first_color;
  a.partials = mean ? P->d.partials : nullptr;
  a.counter = CNT(P, CNT_SWEEP_MEAN);
  a.st = use_state ? ST(P) : nullptr;
  a.n_total = (int)ncells(L);
  a.mixed = mixed(P) ? 1 : 0;
  a.flux = P->d.stencil == PF_STENCIL_FLUX ? 1 : 0;
  constexpr int TI = 4;
  dim3 grid((L.nz + SW_TK - 1) / SW_TK, (L.ny + SW_TJ - 1) / SW_TJ, (L.nx + TI - 1) / TI);
  if constexpr (std::is_same<T, float>::value && std::is_same<TB, float>::value) {
    TileMaps maps;
    // levels of 128+ planes: 6-plane tiles (73.5 KB of shared memory), so
    // that three CTAs of 512 threads share an SM and one CTA's staging
    // overlaps the others' relaxations (1.39 relaxations and 48 staged bytes
    // per cell); 2% faster per solve than 8-plane tiles at two CTAs per SM
    if (P->use_tma && L.nx >= 128 && tma_maps<6, T, TB>(P, lv, p_in, b, b_scale, V, &maps)) {
      const dim3 g6(grid.x, grid.y, (L.nx + 5) / 6);
      PF_CUDA_TRY(launch_overlapped(k_rb_tile_tma<6, 512>, g6, dim3(512), TmaDims<6>::SMEM, s, maps, a));
      PF_LAUNCHED();
      return PF_OK;
    }
    // levels of 64 planes: 8-plane tiles (1.33 relaxations and 44 staged bytes
    // per cell instead of 1.5 and 55), 512 threads, two CTAs per SM: one wave
    // of 256 CTAs, which six-plane tiles (352 CTAs) do not beat
    if (P->use_tma && L.nx >= 64 && tma_maps<8, T, TB>(P, lv, p_in, b, b_scale, V, &maps)) {
      const dim3 g8(grid.x, grid.y, (L.nx + 7) / 8);
      PF_CUDA_TRY(launch_overlapped(k_rb_tile_tma<8, 512>, g8, dim3(512), TmaDims<8>::SMEM, s, maps, a));
      PF_LAUNCHED();
      return PF_OK;
    }
    if (P->use_tma && tma_maps<TI, T, TB>(P, lv, p_in, b, b_scale, V, &maps)) {
      PF_CUDA_TRY(launch_overlapped(k_rb_tile_tma<TI, SW_NT>, grid, dim3(SW_NT), TmaDims<TI>::SMEM, s, maps, a));
      PF_LAUNCHED();
      return PF_OK;
    }
  }
  if constexpr (!std::is_same<T, float>::value) {
    TileMaps maps;
    constexpr bool B32 = std::is_same<TB, float>::value;
    // as in FP32: six-plane tiles at 128+ planes (68 KB with the FP32 b rows
    // of the finest level: three CTAs per SM), eight-plane tiles at 64 planes
    if (P->use_tma && L.nx >= 128 && tma_maps16<6, T, TB>(P, lv, p_in, b, V, &maps)) {
      const dim3 g6(grid.x, grid.y, (L.nx + 5) / 6);
      PF_CUDA_TRY(launch_overlapped(k_rb_tile_tma16<6, 512, T, TB>, g6, dim3(512), Tma16Dims<6, B32>::SMEM, s, maps,
                                    a));
      PF_LAUNCHED();
      return PF_OK;
    }
    if (P->use_tma && L.nx >= 64 && tma_maps16<8, T, TB>(P, lv, p_in, b, V, &maps)) {
      const dim3 g8(grid.x, grid.y, (L.nx + 7) / 8);
      PF_CUDA_TRY(launch_overlapped(k_rb_tile_tma16<8, 512, T, TB>, g8, dim3(512), Tma16Dims<8, B32>::SMEM, s, maps,
                                    a));
      PF_LAUNCHED();
      return PF_OK;
    }
    if (P->use_tma && tma_maps16<TI, T, TB>(P, lv, p_in, b, V, &maps)) {
      PF_CUDA_TRY(launch_overlapped(k_rb_tile_tma16<TI, SW_NT, T, TB>, grid, dim3(SW_NT), Tma16Dims<TI, B32>::SMEM, s,
                                    maps, a));
      PF_LAUNCHED();
      return PF_OK;
    }
  }
  k_rb_tile<T, TB, TI><<<grid, SW_NT, TileDims<TI>::SMEM, s>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}

int lg2_exact(int v) {
  int s = 0;
  while ((1 << s) < v) ++s;
  return (1 << s) == v ? s : -1;
}

template <class T> BottomLevel bottom_level(pf_mg_plan* P, int lv) {
  const pf_mg_level& L = P->d.lev[lv];
  LV<T> V = view<T>(P, lv);
  const int s1 = lg2_exact(L.ny), s2 = lg2_exact(L.nz);
  const bool p2 = s1 >= 0 && s2 >= 0;
  return BottomLevel{L.nx, L.ny, L.nz, p2 ? s1 : -1, p2 ? s2 : -1, V.bx, V.by, V.bz};
}

template <class T, class TB>
int launch_bottom_cluster(pf_mg_plan* P, const TB* b, const float* b_scale, bool want_mean, cudaStream_t s, T** out) {
  ClusterArgs<T, TB> a;
  const int lb = P->lb, nlev = P->d.nlev;
  a.nd = P->bc_nd;
  for (int l = 0; l < a.nd; ++l) a.D[l] = bottom_level<T>(P, lb + l);
  a.nl = nlev - lb - a.nd;
  for (int l = 0; l < a.nl; ++l) a.L[l] = bottom_level<T>(P, lb + a.nd + l);
  LV<T> V0 = view<T>(P, lb);
  a.b = b;
  a.b_scale = b_scale;
  a.p_out = V0.p0;
  a.omega = P->d.omega;
  a.pre = P->d.pre;
  a.post = P->d.post;
  a.coarsest = P->d.coarsest;
  a.rscale = mixed(P) ? 0.125f : 1.f;
  a.pscale = mixed(P) ? 2.f : 1.f;
  a.flux = FLUX(P);
  a.st = ST(P);
  a.want_mean = want_mean ? 1 : 0;
  a.mixed = mixed(P) ? 1 : 0;
  a.M = P->dense_nb ? P->bottom_op : nullptr;
  a.nb = P->dense_nb;
  if (mixed(P)) k_bottom_cluster<T, TB, double><<<BC_CTAS, BC_NT, P->bc_smem, s>>>(a);
  else k_bottom_cluster<T, TB, float><<<BC_CTAS, BC_NT, P->bc_smem, s>>>(a);
  PF_LAUNCHED();
  *out = V0.p0;
  return PF_OK;
}

template <class T, class TB>
int launch_bottom(pf_mg_plan* P, const TB* b, const float* b_scale, bool want_mean, cudaStream_t s, T** out) {
  if (P->bc_nd > 0) return launch_bottom_cluster<T, TB>(P, b, b_scale, want_mean, s, out);
  BottomArgs<T, TB> a;
  const int lb = P->lb;
  a.nl = P->d.nlev - lb;
  for (int l = 0; l < a.nl; ++l) {
    const pf_mg_level& L = P->d.lev[lb + l];
    LV<T> V = view<T>(P, lb + l);
    auto lg = [](int v) {
      int s = 0;
      while ((1 << s) < v) ++s;
      return (1 << s) == v ? s : -1;
    };
    const int s1 = lg(L.ny), s2 = lg(L.nz);
    const bool p2 = s1 >= 0 && s2 >= 0;
    a.L[l] = BottomLevel{L.nx, L.ny, L.nz, p2 ? s1 : -1, p2 ? s2 : -1, V.bx, V.by, V.bz};
  }
  LV<T> V0 = view<T>(P, lb);
  a.b = b;
  a.b_scale = b_scale;
  a.p_out = V0.p0;
  a.omega = P->d.omega;
  a.pre = P->d.pre;
  a.post = P->d.post;
  a.coarsest = P->d.coarsest;
  a.rscale = mixed(P) ? 0.125f : 1.f;
  a.pscale = mixed(P) ? 2.f : 1.f;
  a.flux = FLUX(P);
  a.st = ST(P);
  a.want_mean = want_mean ? 1 : 0;
  a.mixed = mixed(P) ? 1 : 0;
  a.bulk = 0;
  if constexpr (std::is_same<T, float>::value && std::is_same<TB, float>::value) {
    bool ok = b_scale == nullptr && aligned16(b) && ((size_t)ncells(P->d.lev[lb]) * 4) % 16 == 0;
    for (int l = 0; l < a.nl && ok; ++l) {
      const BottomLevel& L = a.L[l];
      const long long nf[3] = {(long long)(L.n0 + 1) * L.n1 * L.n2, (long long)L.n0 * (L.n1 + 1) * L.n2,
                               (long long)L.n0 * L.n1 * (L.n2 + 1)};
      const void* ptr[3] = {L.bx, L.by, L.bz};
      ok = ok && ((long long)L.n0 * L.n1 * L.n2) % 4 == 0;  // P and B keep every shared offset 16-byte aligned
      for (int c = 0; c < 3; ++c) ok = ok && aligned16(ptr[c]) && (nf[c] * 4) % 16 == 0;
    }
    a.bulk = ok ? 1 : 0;
  } else {
    bool ok = aligned16(b) && ((size_t)ncells(P->d.lev[lb]) * sizeof(TB)) % 16 == 0 && P->bottom_stage;
    for (int l = 0; l < a.nl && ok; ++l) {
      const BottomLevel& L = a.L[l];
      const long long nf[3] = {(long long)(L.n0 + 1) * L.n1 * L.n2, (long long)L.n0 * (L.n1 + 1) * L.n2,
                               (long long)L.n0 * L.n1 * (L.n2 + 1)};
      const void* ptr[3] = {L.bx, L.by, L.bz};
      for (int c = 0; c < 3; ++c) ok = ok && aligned16(ptr[c]) && (nf[c] * (long long)sizeof(T)) % 16 == 0;
    }
    a.bulk = ok ? 2 : 0;
  }
  if (mixed(P)) k_bottom<T, TB, double><<<1, BT_NT, P->bottom_smem, s>>>(a);
  else k_bottom<T, TB, float><<<1, BT_NT, P->bottom_smem, s>>>(a);
  PF_LAUNCHED();
  *out = V0.p0;
  return PF_OK;
}

#define PF_TRY(x)              \
  do {                         \
    int rc_ = (x);             \
    if (rc_ != PF_OK) return rc_; \
  } while (0)

// One V-cycle on level lv with right-hand side b (storage TB, times *b_scale);
// the level's final p is returned in *out.  want_mean: the mean of the final p
// goes to st->c_shift (level 0 only).
template <class T, class TB>
int vcycle(pf_mg_plan* P, int lv, const TB* b, const float* b_scale, bool want_mean, cudaStream_t s, T** out) {
  const pf_mg_level& L = P->d.lev[lv];
  LV<T> V = view<T>(P, lv);
  const int nlev = P->d.nlev;
  const long long n = ncells(L);
  if (lv == P->lb) return launch_bottom<T, TB>(P, b, b_scale, want_mean, s, out);
  if (lv == nlev - 1) {
    // coarsest level too large for one CTA: `coarsest` tile sweeps from zero, mean removed
    T* cur = nullptr;
    for (int it = 0; it < P->d.coarsest; ++it) {
      T* o = (it & 1) ? V.p1 : V.p0;
      PF_TRY((launch_sweep<T, TB>(P, lv, cur, it == 0, o, b, b_scale, V, nullptr, 1.f, 0, false, true, s)));
      cur = o;
    }
    if (!cur) {
      PF_CUDA_TRY(cudaMemsetAsync(V.p0, 0, sizeof(T) * n, s));
      cur = V.p0;
    }
    k_mean_of<T><<<red_grid(n), RED_NT, 0, s>>>(n, cur, P->d.partials, CNT(P, CNT_COARSE), ST(P), 0);
    PF_LAUNCHED();
    k_shift_mean_inplace<T><<<ew_grid(n), 256, 0, s>>>(n, cur, ST(P));
    PF_LAUNCHED();
    if (want_mean) {
      k_mean_of<T><<<red_grid(n), RED_NT, 0, s>>>(n, cur, P->d.partials, CNT(P, CNT_SWEEP_MEAN), ST(P),
                                                  mixed(P) ? 1 : 0);
      PF_LAUNCHED();
    }
    *out = cur;
    return PF_OK;
  }
  const float rscale = mixed(P) ? 0.125f : 1.f;
  const float pscale = mixed(P) ? 2.f : 1.f;
  T* cur = nullptr;
  for (int it = 0; it < P->d.pre; ++it) {
    T* o = (it & 1) ? V.p1 : V.p0;
    PF_TRY((launch_sweep<T, TB>(P, lv, cur, it == 0, o, b, b_scale, V, nullptr, 1.f, 0, false, true, s)));
    cur = o;
  }
  if (!cur) {
    PF_CUDA_TRY(cudaMemsetAsync(V.p0, 0, sizeof(T) * n, s));
    cur = V.p0;
  }
  LV<T> C = view<T>(P, lv + 1);
  const pf_mg_level& CL = P->d.lev[lv + 1];
  k_residual_restrict<T, TB><<<grid_cells(CL.nx, CL.ny, CL.nz), C3_NT, 0, s>>>(
      L.nx, L.ny, L.nz, cur, b, b_scale, V.bx, V.by, V.bz, C.b, rscale, nullptr, ST(P), FLUX(P));
  PF_LAUNCHED();
  T* pc = nullptr;
  PF_TRY((vcycle<T, T>(P, lv + 1, C.b, nullptr, false, s, &pc)));
  if (P->d.post == 0) {
    k_prolong_add<T><<<ew_grid(n), 256, 0, s>>>(L.nx, L.ny, L.nz, pc, cur, pscale, ST(P));
    PF_LAUNCHED();
    if (want_mean) {
      k_mean_of<T><<<red_grid(n), RED_NT, 0, s>>>(n, cur, P->d.partials, CNT(P, CNT_SWEEP_MEAN), ST(P),
                                                  mixed(P) ? 1 : 0);
      PF_LAUNCHED();
    }
  } else {
    for (int it = 0; it < P->d.post; ++it) {
      T* o = (cur == V.p0) ? V.p1 : V.p0;
      PF_TRY((launch_sweep<T, TB>(P, lv, cur, false, o, b, b_scale, V, it == 0 ? pc : nullptr, pscale, 1,
                                  want_mean && it == P->d.post - 1, true, s)));
      cur = o;
    }
  }
  *out = cur;
  return PF_OK;
}

template <class T> int vcycle0(pf_mg_plan* P, const float* r, cudaStream_t s, T** out) {
  return vcycle<T, float>(P, 0, r, mixed(P) ? scale_r_ptr(P) : nullptr, true, s, out);
}

template <class T> int enqueue_setup(pf_mg_plan* P, const float* b, float tol, int max_iter, cudaStream_t s) {
  const pf_mg_level& L0 = P->d.lev[0];
  const long long n = ncells(L0);
  k_set_state<<<1, 1, 0, s>>>(ST(P), tol, max_iter, P->d.coef_scale);
  PF_LAUNCHED();
  k_sum_mean<<<red_grid(n), RED_NT, 0, s>>>(n, b, P->d.partials, CNT(P, CNT_SUM_B), ST(P));
  PF_LAUNCHED();
  k_init_r<<<red_grid(n), RED_NT, 0, s>>>(n, b, P->d.rhs, P->d.res_v, P->d.x, P->d.partials, CNT(P, CNT_INIT_R),
                                          ST(P));
  PF_LAUNCHED();
  if (mixed(P)) {
    k_update_zscale<<<1, 1, 0, s>>>(ST(P), P->d.coef_scale);
    PF_LAUNCHED();
  }
  T* p0 = nullptr;
  PF_TRY(vcycle0<T>(P, P->d.res_v, s, &p0));
  k_init_q<T><<<red_grid(n), RED_NT, 0, s>>>(n, p0, P->d.res_v, P->d.q, P->d.z, P->d.partials, CNT(P, CNT_INIT_Q),
                                             ST(P), mixed(P) ? 1 : 0);
  PF_LAUNCHED();
  return PF_OK;
}

template <class T> int enqueue_iteration(pf_mg_plan* P, int par, cudaStream_t s) {
  const pf_mg_level& L0 = P->d.lev[0];
  const long long n = ncells(L0);
  float* r_cur = par ? P->d.res_alt : P->d.res_v;
  float* r_new = par ? P->d.res_v : P->d.res_alt;
  k_apply_dot<<<grid_cells((L0.nx + 3) / 4, L0.ny, L0.nz), C3_NT, 0, s>>>(L0.nx, L0.ny, L0.nz, P->d.q, L0.bx, L0.by, L0.bz,
                                                                nullptr, P->d.Ap, P->d.partials,
                                                                CNT(P, CNT_APPLY_DOT), ST(P), FLUX(P));
  PF_LAUNCHED();
  k_update_xr<<<vec_grid(n), RED_NT, 0, s>>>(n, P->d.q, P->d.Ap, r_cur, r_new, P->d.x, P->d.partials,
                                             CNT(P, CNT_UPDATE_XR), ST(P));
  PF_LAUNCHED();
  if (mixed(P)) {
    k_update_zscale<<<1, 1, 0, s>>>(ST(P), P->d.coef_scale);
    PF_LAUNCHED();
  }
  T* p0 = nullptr;
  PF_TRY(vcycle0<T>(P, r_new, s, &p0));
  k_dots<T><<<vec_grid(n), RED_NT, 0, s>>>(n, p0, r_new, r_cur, P->d.partials, CNT(P, CNT_DOTS), ST(P),
                                           mixed(P) ? 1 : 0);
  PF_LAUNCHED();
  k_update_q<T><<<vec_grid(n), RED_NT, 0, s>>>(n, p0, P->d.q, ST(P), mixed(P) ? 1 : 0);
  PF_LAUNCHED();
  return PF_OK;
}

int enqueue_final(pf_mg_plan* P, float* x_out, cudaStream_t s) {
  const long long n = ncells(P->d.lev[0]);
  k_sum_mean<<<red_grid(n), RED_NT, 0, s>>>(n, P->d.x, P->d.partials, CNT(P, CNT_FINAL_SUM), ST(P));
  PF_LAUNCHED();
  k_shift_out<<<ew_grid(n), 256, 0, s>>>(n, P->d.x, x_out, ST(P));
  PF_LAUNCHED();
  return PF_OK;
}

template <class T> int capture_graphs(pf_mg_plan* P) {
  for (int par = 0; par < 2; ++par) {
    cudaGraph_t g = nullptr;
    PF_CUDA_TRY(cudaStreamBeginCapture(P->cap_stream, cudaStreamCaptureModeThreadLocal));
    count_suppress(true);
    int rc = enqueue_iteration<T>(P, par, P->cap_stream);
    count_suppress(false);
    cudaError_t e = cudaStreamEndCapture(P->cap_stream, &g);
    if (rc != PF_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) {
      set_cuda_error(e, "cudaStreamEndCapture");
      return PF_ERR_CUDA;
    }
    size_t nn = 0;
    cudaGraphGetNodes(g, nullptr, &nn);
    P->exec_nodes[par] = nn;
    e = cudaGraphInstantiate(&P->exec[par], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      set_cuda_error(e, "cudaGraphInstantiate");
      return PF_ERR_CUDA;
    }
  }
  P->graphs_ready = true;
  return PF_OK;
}

template <class T>
int solve_impl(pf_mg_plan* P, const float* b, float* x, float tol, int max_iter, int use_graphs, int verbose,
               int* iters_out, double* rel_out, cudaStream_t s) {
  PF_TRY(enqueue_setup<T>(P, b, tol, max_iter, s));
  if (use_graphs && !P->graphs_ready) PF_TRY(capture_graphs<T>(P));
  for (int k = 1; k <= max_iter; ++k) {
    const int par = (k - 1) & 1;
    if (use_graphs) {
      PF_CUDA_TRY(cudaGraphLaunch(P->exec[par], s));
      count_launch(P->exec_nodes[par]);
    } else {
      PF_TRY(enqueue_iteration<T>(P, par, s));
    }
    PF_CUDA_TRY(cudaMemcpyAsync(P->h_state[k & 1], P->d.state, sizeof(MGState), cudaMemcpyDeviceToHost, s));
    PF_CUDA_TRY(cudaEventRecord(P->ev[k & 1], s));
    if (verbose) {
      PF_CUDA_TRY(cudaEventSynchronize(P->ev[k & 1]));
      const MGState* h = P->h_state[k & 1];
      if (h->it == k) std::printf("    pcg it=%3d  |r|inf/|b|inf = %.3e\n", h->it, h->rel);
      if (h->done) break;
      continue;
    }
    if (k >= 2) {
      PF_CUDA_TRY(cudaEventSynchronize(P->ev[(k - 1) & 1]));
      if (P->h_state[(k - 1) & 1]->done) break;
    }
  }
  PF_TRY(enqueue_final(P, x, s));
  PF_CUDA_TRY(cudaMemcpyAsync(P->h_state[0], P->d.state, sizeof(MGState), cudaMemcpyDeviceToHost, s));
  PF_CUDA_TRY(cudaStreamSynchronize(s));
  const MGState* h = P->h_state[0];
  *iters_out = h->it;
  *rel_out = h->rel;
  if (h->status == ST_NONFINITE) {
    set_error(PF_ERR_NONFINITE, "non-finite residual in the CG iteration %d", h->it);
    return PF_ERR_NONFINITE;
  }
  if (h->status == ST_TMA_TIMEOUT) {
    set_error(PF_ERR_CUDA, "a TMA staging wait timed out in the CG iteration %d; the solve was stopped", h->it);
    return PF_ERR_CUDA;
  }
  if (h->status == ST_RUNNING) {
    set_error(PF_ERR_NOT_CONVERGED, "tolerance %g not reached in %d iterations (rel %g)", (double)tol, h->it, h->rel);
    return PF_ERR_NOT_CONVERGED;
  }
  return PF_OK;
}

// the dense operator of the levels below the cluster's slabs, one column per CTA
template <class T> int launch_dense_build(pf_mg_plan* P, cudaStream_t s) {
  DenseBuildArgs<T> a;
  const int l0 = P->lb + P->bc_nd;
  a.nl = P->d.nlev - l0;
  size_t floats = 0;
  for (int l = 0; l < a.nl; ++l) {
    a.L[l] = bottom_level<T>(P, l0 + l);
    floats += bottom_level_floats(a.L[l].n0, a.L[l].n1, a.L[l].n2);
  }
  a.M = P->bottom_op;
  a.omega = P->d.omega;
  a.pre = P->d.pre;
  a.post = P->d.post;
  a.coarsest = P->d.coarsest;
  a.rscale = mixed(P) ? 0.125f : 1.f;
  a.pscale = mixed(P) ? 2.f : 1.f;
  a.flux = FLUX(P);
  const BottomLevel& Lc = a.L[a.nl - 1];
  const size_t smem = floats * sizeof(float) + 16 + (size_t)Lc.n0 * Lc.n1 * Lc.n2 * sizeof(double);
  if (mixed(P)) k_bottom_dense_build<T, double><<<P->dense_nb, DB_NT, smem, s>>>(a);
  else k_bottom_dense_build<T, float><<<P->dense_nb, DB_NT, smem, s>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}

template <class T> int build_impl(pf_mg_plan* P, cudaStream_t s) {
  for (int lv = 0; lv < P->d.nlev; ++lv) {
    const pf_mg_level& L = P->d.lev[lv];
    const long long n = ncells(L);
    const long long nf = (long long)(L.nx + 1) * L.ny * L.nz + (long long)L.nx * (L.ny + 1) * L.nz +
                         (long long)L.nx * L.ny * (L.nz + 1);
    T* lpx = mixed(P) ? (T*)L.bx_lp : nullptr;
    k_level_coefs<T><<<ew_grid(n + (lpx ? nf : 0)), 256, 0, s>>>(L.nx, L.ny, L.nz, L.bx, L.by, L.bz, L.diag, lpx,
                                                                 (T*)L.by_lp, (T*)L.bz_lp, P->lp_scale[lv],
                                                                 L.bz_pad, L.bz_pitch);
    PF_LAUNCHED();
    if (lv + 1 < P->d.nlev) {
      const pf_mg_level& C = P->d.lev[lv + 1];
      const long long ncf = (long long)(C.nx + 1) * C.ny * C.nz + (long long)C.nx * (C.ny + 1) * C.nz +
                            (long long)C.nx * C.ny * (C.nz + 1);
      k_coarsen_faces<<<ew_grid(ncf), 256, 0, s>>>(L.nx, L.ny, L.nz, C.nx, C.ny, C.nz, L.bx, L.by, L.bz, C.bx, C.by,
                                                    C.bz);
      PF_LAUNCHED();
    }
  }
  if (P->dense_nb) {
    const int rc = launch_dense_build<T>(P, s);
    if (rc != PF_OK) return rc;
  }
  return PF_OK;
}

template <class T> int precondition_impl(pf_mg_plan* P, const float* r, float* z, cudaStream_t s) {
  const long long n = ncells(P->d.lev[0]);
  k_clear_done<<<1, 1, 0, s>>>(ST(P));
  PF_LAUNCHED();
  if (mixed(P)) {
    k_scale_of<<<red_grid(n), RED_NT, 0, s>>>(n, r, P->d.partials, CNT(P, CNT_SCALE), ST(P), P->d.coef_scale);
    PF_LAUNCHED();
  }
  T* p0 = nullptr;
  PF_TRY(vcycle0<T>(P, r, s, &p0));
  k_write_z<T><<<ew_grid(n), 256, 0, s>>>(n, p0, z, ST(P), mixed(P) ? 1 : 0);
  PF_LAUNCHED();
  return PF_OK;
}

template <class T> cudaError_t set_smem_attrs() {
  const int mx = 220 * 1024, tile = (int)TileDims<4>::SMEM;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t r) {
    if (e == cudaSuccess) e = r;
  };
  chk(cudaFuncSetAttribute(k_bottom<T, float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  chk(cudaFuncSetAttribute(k_bottom<T, T, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  chk(cudaFuncSetAttribute(k_bottom<T, float, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  chk(cudaFuncSetAttribute(k_bottom<T, T, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  chk(cudaFuncSetAttribute(k_bottom_cluster<T, float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  chk(cudaFuncSetAttribute(k_bottom_cluster<T, T, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  chk(cudaFuncSetAttribute(k_bottom_cluster<T, float, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  chk(cudaFuncSetAttribute(k_bottom_cluster<T, T, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  chk(cudaFuncSetAttribute(k_bottom_dense_build<T, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  chk(cudaFuncSetAttribute(k_bottom_dense_build<T, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  chk(cudaFuncSetAttribute(k_rb_tile<T, float, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, tile));
  chk(cudaFuncSetAttribute(k_rb_tile<T, T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, tile));
  chk(cudaFuncSetAttribute(k_rb_tile_tma<4, SW_NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)TmaDims<4>::SMEM));
  chk(cudaFuncSetAttribute(k_rb_tile_tma<8, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TmaDims<8>::SMEM));
  chk(cudaFuncSetAttribute(k_rb_tile_tma<6, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TmaDims<6>::SMEM));
  if constexpr (!std::is_same<T, float>::value) {
    chk(cudaFuncSetAttribute(k_rb_tile_tma16<4, SW_NT, T, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Tma16Dims<4, true>::SMEM));
    chk(cudaFuncSetAttribute(k_rb_tile_tma16<4, SW_NT, T, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Tma16Dims<4, false>::SMEM));
    chk(cudaFuncSetAttribute(k_rb_tile_tma16<6, 512, T, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Tma16Dims<6, true>::SMEM));
    chk(cudaFuncSetAttribute(k_rb_tile_tma16<6, 512, T, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Tma16Dims<6, false>::SMEM));
    chk(cudaFuncSetAttribute(k_rb_tile_tma16<8, 512, T, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Tma16Dims<8, true>::SMEM));
    chk(cudaFuncSetAttribute(k_rb_tile_tma16<8, 512, T, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Tma16Dims<8, false>::SMEM));
  }
  return e;
}

}  // namespace

struct BottomSel {
  int lb = 0;              // first level of the bottom kernel
  size_t bottom_smem = 0;  // single-CTA kernel
  bool bottom_stage = false;
  int bc_nd = 0;           // cluster kernel: distributed levels
  size_t bc_smem = 0;
  int dense_nb = 0;        // dense operator of the levels below the slabs: its size (cells)
  size_t bc_smem_dense = 0;
};

// The bottom of a plan's V-cycle (pf_mg_plan_create, pf_mg_bottom_op_floats).
BottomSel select_bottom(const pf_mg_desc* desc) {
  BottomSel r;
  // bottom kernel: the deepest run of levels that each fit kBottomMaxCells and
  // together fit the shared memory of one CTA
  r.lb = desc->nlev;
  r.bottom_smem = 0;
  r.bottom_stage = desc->precision != PF_PREC_FP32;
  {
    // 16-bit hierarchy: a staging area for the raw 16-bit faces (and b, at
    // most 4 bytes a cell) behind the coarsest solution
    size_t floats = 0, faces = 0;
    const pf_mg_level& Lc = desc->lev[desc->nlev - 1];
    for (int lv = desc->nlev - 1; lv >= 0; --lv) {
      const pf_mg_level& L = desc->lev[lv];
      const long long n = (long long)L.nx * L.ny * L.nz;
      const size_t f2 = floats + bottom_level_floats(L.nx, L.ny, L.nz);
      const size_t fc2 = faces + bottom_level_floats(L.nx, L.ny, L.nz) - 2 * (size_t)n;
      const size_t stage = r.bottom_stage ? 16 + 2 * fc2 + 4 * (size_t)n : 0;
      const size_t bytes = f2 * sizeof(float) + 16 + (size_t)Lc.nx * Lc.ny * Lc.nz * sizeof(double) + stage;
      if (n > kBottomMaxCells || bytes > 200 * 1024) break;
      floats = f2;
      faces = fc2;
      r.lb = lv;
      r.bottom_smem = bytes;
    }
  }
  // cluster bottom (k_bottom_cluster): the finest start level lv < lb such
  // that lv .. lv+nd-1 halve exactly and split into even slabs over BC_CTAS
  // CTAs (n0 a multiple of 2*BC_CTAS, n1 and n2 even), at least one level is
  // left for CTA 0, and slabs, CTA 0's levels and the FP64 coarsest fit one
  // CTA's shared memory.  PFFLIP_MG_BOTTOM=cta keeps the single-CTA bottom.
  r.bc_nd = 0;
  r.bc_smem = 0;
  {
    const char* env = std::getenv("PFFLIP_MG_BOTTOM");
    const bool allow = !(env && std::strcmp(env, "cta") == 0);
    const bool allow_dense = !(env && (std::strcmp(env, "cta") == 0 || std::strcmp(env, "cluster") == 0));
    const int nlev = desc->nlev;
    const pf_mg_level& Lc = desc->lev[nlev - 1];
    for (int lv = 0; allow && lv < r.lb; ++lv) {
      auto halves = [&](int l) {
        const pf_mg_level& F = desc->lev[l];
        const pf_mg_level& C = desc->lev[l + 1];
        return C.nx * 2 == F.nx && C.ny * 2 == F.ny && C.nz * 2 == F.nz;
      };
      int nd = 0;
      size_t floats = 0;
      while (lv + nd < nlev - 1 && nd < BC_MAX_DIST) {
        const pf_mg_level& L = desc->lev[lv + nd];
        if (L.nx % (2 * BC_CTAS) != 0 || L.ny % 2 != 0 || L.nz % 2 != 0 || !halves(lv + nd)) break;
        floats += bc_level_floats(L.nx, L.ny, L.nz);
        ++nd;
      }
      if (nd == 0) continue;
      for (int l = lv + nd; l < nlev; ++l)
        floats += bottom_level_floats(desc->lev[l].nx, desc->lev[l].ny, desc->lev[l].nz);
      const size_t bytes = floats * sizeof(float) + 16 + (size_t)Lc.nx * Lc.ny * Lc.nz * sizeof(double);
      if (bytes > 200 * 1024) continue;
      r.bc_nd = nd;
      r.bc_smem = bytes;
      r.lb = lv;
      // dense bottom: the levels below the slabs as one operator on the first of
      // them, each CTA applying the rows of its own coarse planes
      const pf_mg_level& F = desc->lev[lv + nd];
      const int nb = F.nx * F.ny * F.nz;
      if (allow_dense && nb <= kDenseMaxCells && F.nx % BC_CTAS == 0) {
        size_t dfl = 0;
        for (int l = lv; l < lv + nd; ++l) dfl += bc_level_floats(desc->lev[l].nx, desc->lev[l].ny, desc->lev[l].nz);
        r.dense_nb = nb;
        r.bc_smem_dense = (dfl + 4 + (size_t)nb + 4 + (size_t)(nb / BC_CTAS) + 4 + BC_NT) * sizeof(float);
      }
      break;
    }
  }
  return r;
}

extern "C" {

int64_t pf_mg_partials_count(void) { return pf::kPartials; }

int32_t pf_mg_level_count(int32_t nx, int32_t ny, int32_t nz, int32_t min_dim, int32_t* dims_out) {
  int r[3] = {nx, ny, nz};
  int n = 0;
  while (n < PF_MG_MAX_LEVELS) {
    if (dims_out) { dims_out[3 * n] = r[0]; dims_out[3 * n + 1] = r[1]; dims_out[3 * n + 2] = r[2]; }
    ++n;
    const int mn = r[0] < r[1] ? (r[0] < r[2] ? r[0] : r[2]) : (r[1] < r[2] ? r[1] : r[2]);
    if (mn / 2 < min_dim || (r[0] % 2) || (r[1] % 2) || (r[2] % 2)) break;
    r[0] /= 2; r[1] /= 2; r[2] /= 2;
  }
  return n;
}

int pf_mg_plan_create(const pf_mg_desc* desc, pf_mg_plan** out) {
  PF_REQUIRE(desc && out, "null argument");
  PF_REQUIRE(desc->nlev >= 1 && desc->nlev <= PF_MG_MAX_LEVELS, "nlev %d out of range", desc->nlev);
  PF_REQUIRE(desc->precision >= PF_PREC_FP32 && desc->precision <= PF_PREC_BF16, "bad precision");
  PF_REQUIRE(desc->stencil == PF_STENCIL_REFERENCE || desc->stencil == PF_STENCIL_FLUX, "bad stencil");
  PF_REQUIRE(desc->state && desc->partials && desc->counters, "state/partials/counters required");
  PF_REQUIRE(desc->res_v && desc->res_alt && desc->q && desc->Ap && desc->x, "CG vectors required");
  for (int lv = 0; lv < desc->nlev; ++lv) {
    const pf_mg_level& L = desc->lev[lv];
    PF_REQUIRE(L.nx > 0 && L.ny > 0 && L.nz > 0, "level %d dims", lv);
    PF_REQUIRE(L.bx && L.by && L.bz && L.diag && L.p && L.p_alt && L.b, "level %d fp32 arrays", lv);
    if (desc->precision != PF_PREC_FP32)
      PF_REQUIRE(L.bx_lp && L.by_lp && L.bz_lp && L.p_lp && L.p_lp_alt && L.b_lp, "level %d 16-bit arrays", lv);
    if (lv > 0) {
      const pf_mg_level& F = desc->lev[lv - 1];
      PF_REQUIRE(F.nx == 2 * L.nx && F.ny == 2 * L.ny && F.nz == 2 * L.nz, "level %d is not half of level %d", lv,
                 lv - 1);
    }
    const long long tiles = (long long)((L.nz + SW_TK - 1) / SW_TK) * ((L.ny + SW_TJ - 1) / SW_TJ) * ((L.nx + 3) / 4);
    PF_REQUIRE(tiles <= pf::kPartials, "level %d too large for the sweep reduction", lv);
  }
  pf_mg_plan* P = new pf_mg_plan();
  std::memset(P, 0, sizeof(*P));
  P->d = *desc;
  P->prec = desc->precision;
  {
    const char* env = std::getenv("PFFLIP_NO_TMA");
    P->use_tma = !(env && env[0] == '1');
  }
  {
    int dev = 0;
    P->sms = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&P->sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    if (P->sms <= 0) P->sms = kNumSMs;
  }
  for (int lv = 0; lv < desc->nlev; ++lv) {
    P->lp_scale[lv] = std::ldexp(desc->coef_scale > 0.f ? desc->coef_scale : 1.f, -2 * lv);
  }
  {
    const BottomSel sel = select_bottom(desc);
    P->lb = sel.lb;
    P->bottom_smem = sel.bottom_smem;
    P->bottom_stage = sel.bottom_stage;
    P->bc_nd = sel.bc_nd;
    P->bc_smem = sel.bc_smem;
    P->dense_nb = (sel.dense_nb > 0 && desc->bottom_op) ? sel.dense_nb : 0;
    if (P->dense_nb) P->bc_smem = sel.bc_smem_dense;
    P->bottom_op = desc->bottom_op;
  }
  cudaError_t e = cudaStreamCreateWithFlags(&P->cap_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&P->h_state[0], sizeof(pf::MGState) * 2, cudaHostAllocDefault);
  if (e == cudaSuccess) {
    P->h_state[1] = P->h_state[0] + 1;
    e = cudaEventCreateWithFlags(&P->ev[0], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->ev[1], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    pf::set_cuda_error(e, "pf_mg_plan_create");
    pf_mg_plan_destroy(P);
    return PF_ERR_CUDA;
  }
  e = set_smem_attrs<float>();
  if (e == cudaSuccess) e = set_smem_attrs<__half>();
  if (e == cudaSuccess) e = set_smem_attrs<__nv_bfloat16>();
  if (e != cudaSuccess) {
    pf::set_cuda_error(e, "cudaFuncSetAttribute (shared memory)");
    pf_mg_plan_destroy(P);
    return PF_ERR_CUDA;
  }
  *out = P;
  return PF_OK;
}

int pf_mg_plan_destroy(pf_mg_plan* P) {
  if (!P) return PF_OK;
  for (int i = 0; i < 2; ++i) {
    if (P->exec[i]) cudaGraphExecDestroy(P->exec[i]);
    if (P->ev[i]) cudaEventDestroy(P->ev[i]);
  }
  if (P->h_state[0]) cudaFreeHost(P->h_state[0]);
  if (P->cap_stream) cudaStreamDestroy(P->cap_stream);
  delete P;
  return PF_OK;
}

int pf_mg_bottom_info(const pf_mg_plan* P, int32_t* first_level, int32_t* cluster_levels, int32_t* dense) {
  PF_REQUIRE(P && first_level && cluster_levels && dense, "null argument");
  *first_level = P->lb;
  *cluster_levels = P->bc_nd;
  *dense = P->dense_nb > 0 ? 1 : 0;
  return PF_OK;
}

int64_t pf_mg_bottom_op_floats(const pf_mg_desc* desc) {
  if (!desc || desc->nlev < 1 || desc->nlev > PF_MG_MAX_LEVELS) return 0;
  const BottomSel sel = select_bottom(desc);
  return sel.dense_nb > 0 ? (int64_t)sel.dense_nb * sel.dense_nb : 0;
}

int pf_mg_build_hierarchy(pf_mg_plan* P, const float* bx, const float* by, const float* bz, void* stream) {
  PF_REQUIRE(P && bx && by && bz, "null argument");
  cudaStream_t s = S(stream);
  const pf_mg_level& L0 = P->d.lev[0];
  const size_t nfx = (size_t)(L0.nx + 1) * L0.ny * L0.nz, nfy = (size_t)L0.nx * (L0.ny + 1) * L0.nz,
               nfz = (size_t)L0.nx * L0.ny * (L0.nz + 1);
  if (bx != L0.bx) PF_CUDA_TRY(cudaMemcpyAsync(L0.bx, bx, nfx * 4, cudaMemcpyDeviceToDevice, s));
  if (by != L0.by) PF_CUDA_TRY(cudaMemcpyAsync(L0.by, by, nfy * 4, cudaMemcpyDeviceToDevice, s));
  if (bz != L0.bz) PF_CUDA_TRY(cudaMemcpyAsync(L0.bz, bz, nfz * 4, cudaMemcpyDeviceToDevice, s));
  switch (P->prec) {
    case PF_PREC_FP16: return build_impl<__half>(P, s);
    case PF_PREC_BF16: return build_impl<__nv_bfloat16>(P, s);
    default: return build_impl<float>(P, s);
  }
}

int pf_mg_precondition(pf_mg_plan* P, const float* r, float* z, void* stream) {
  PF_REQUIRE(P && r && z, "null argument");
  switch (P->prec) {
    case PF_PREC_FP16: return precondition_impl<__half>(P, r, z, S(stream));
    case PF_PREC_BF16: return precondition_impl<__nv_bfloat16>(P, r, z, S(stream));
    default: return precondition_impl<float>(P, r, z, S(stream));
  }
}

int pf_mg_smooth(pf_mg_plan* P, int32_t lv, int32_t nsweeps, int32_t reverse, void* stream) {
  PF_REQUIRE(P && lv >= 0 && lv < P->d.nlev && nsweeps >= 0, "bad argument");
  cudaStream_t s = S(stream);
  const pf_mg_level& L = P->d.lev[lv];
  LV<float> V{L.bx, L.by, L.bz, L.p, L.p_alt, L.b};
  const int saved = P->prec;
  P->prec = PF_PREC_FP32;  // this entry point runs on the fp32 level arrays
  float* cur = L.p;
  int rc = PF_OK;
  for (int it = 0; it < nsweeps && rc == PF_OK; ++it) {
    float* o = (cur == L.p) ? L.p_alt : L.p;
    rc = launch_sweep<float, float>(P, lv, cur, false, o, L.b, nullptr, V, nullptr, 1.f, reverse ? 1 : 0, false,
                                    false, s);
    cur = o;
  }
  P->prec = saved;
  if (rc != PF_OK) return rc;
  if (cur != L.p) PF_CUDA_TRY(cudaMemcpyAsync(L.p, cur, sizeof(float) * ncells(L), cudaMemcpyDeviceToDevice, s));
  return PF_OK;
}

int pf_mg_solve(pf_mg_plan* P, const float* b, float* x, float tol, int32_t max_iter, int32_t use_graphs,
                int32_t verbose, int32_t* iters_out, double* rel_out, void* stream) {
  PF_REQUIRE(P && b && x && iters_out && rel_out, "null argument");
  PF_REQUIRE(max_iter >= 0, "max_iter < 0");
  cudaStream_t s = S(stream);
  switch (P->prec) {
    case PF_PREC_FP16: return solve_impl<__half>(P, b, x, tol, max_iter, use_graphs, verbose, iters_out, rel_out, s);
    case PF_PREC_BF16:
      return solve_impl<__nv_bfloat16>(P, b, x, tol, max_iter, use_graphs, verbose, iters_out, rel_out, s);
    default: return solve_impl<float>(P, b, x, tol, max_iter, use_graphs, verbose, iters_out, rel_out, s);
  }
}

int pf_apply_A(const pf_grid* g, const float* p, const float* bx, const float* by, const float* bz,
               const float* diag, float* out, int32_t stencil, void* stream) {
  PF_REQUIRE(g && p && bx && by && bz && out, "null argument");
  PF_REQUIRE(stencil == PF_STENCIL_REFERENCE || stencil == PF_STENCIL_FLUX, "bad stencil");
  k_apply_A<<<grid_cells(g->nx, g->ny, g->nz), C3_NT, 0, S(stream)>>>(g->nx, g->ny, g->nz, p, bx, by, bz, diag, out,
                                                                      stencil == PF_STENCIL_FLUX ? 1 : 0);
  PF_LAUNCHED();
  return PF_OK;
}

}  // extern "C"
