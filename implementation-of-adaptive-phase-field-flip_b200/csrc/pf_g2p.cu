// Grid-to-particle transfer and advection in one particle pass on sm_100a.
//
// The reference runs field_difference x3 (pfflip/kernels.py:499-502), g2p
// (:468-496), the liquid extrapolation, advect_rk3 (:508-549) and
// reflect_at_walls (:567-595) as separate launches (pfflip/sim.py:316-341,
// :408-420).  The extrapolation only reads grid fields, so it runs first and
// a single kernel then does, per particle, the FLIP/PIC update, the Ralston
// RK3 trace through the extrapolated (liquid) or raw (air) field, the clamp
// and the wall reflection.  u - u* is formed per interpolation tap, which is
// the reference's interpolation of the difference field, value for value.
// Interpolation coordinates are x * (1/dx): identical to the reference's x/dx
// for power-of-two dx, within an ulp otherwise.
// Particles are in cell order, so neighbouring threads gather neighbouring
// taps from L1/L2.
#include "pf_faces.cuh"

namespace pf {

struct G2PArgs {
  long long n;
  int nx, ny, nz;
  float dx, inv_dx, dt, a_liq, a_air;
  float lo[3], hi[3];
  float4* pos;
  float4* vel;
  const float* u[3];
  const float* us[3];
  const float* ul[3];
  const int* solid;
  int do_g2p, do_advect;
};

// Per-position interpolation frame: for each axis d and node offset o in
// {0, 0.5}, the clamped lower/upper tap indices and the upper weight of
// g = x/dx - o (pfflip/kernels.py:52-79).  Face grid c uses offset 0 on axis c
// and 0.5 on the other axes, so all three components share one frame.
struct Frame {
  int lo[3][2], hi[3][2];
  float t[3][2];
};

__device__ __forceinline__ void make_frame(const float x[3], float inv_dx, int nx, int ny, int nz, Frame& f) {
  const int n[3] = {nx, ny, nz};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float q = x[d] * inv_dx;
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      // v = 0: offset 0 (normal axis, extent n+1); v = 1: offset 0.5 (extent n)
      const float g = v == 0 ? q : q - 0.5f;
      const int i0 = (int)floorf(g);
      const int last = v == 0 ? n[d] : n[d] - 1;
      f.t[d][v] = g - (float)i0;
      f.lo[d][v] = min(max(i0, 0), last);
      f.hi[d][v] = min(max(i0 + 1, 0), last);
    }
  }
}

// trilinear sample of face grid c (DIFF: of f - fs, tap by tap), taps and sums
// in the reference's order
template <bool DIFF>
__device__ __forceinline__ float sample_c(const float* __restrict__ f, const float* __restrict__ fs, int c,
                                          const Frame& fr, int ny, int nz) {
  const int vi = c == 0 ? 0 : 1, vj = c == 1 ? 0 : 1, vk = c == 2 ? 0 : 1;
  const int n1 = ny + (c == 1), n2 = nz + (c == 2);
  const float tx = fr.t[0][vi], ty = fr.t[1][vj], tz = fr.t[2][vk];
  const int I[2] = {fr.lo[0][vi], fr.hi[0][vi]}, J[2] = {fr.lo[1][vj], fr.hi[1][vj]};
  const int K[2] = {fr.lo[2][vk], fr.hi[2][vk]};
  const float wi[2] = {1.f - tx, tx}, wj[2] = {1.f - ty, ty}, wk[2] = {1.f - tz, tz};
  float acc = 0.f;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj) {
      const int row = (I[di] * n1 + J[dj]) * n2;  // face arrays hold < 2^31 entries
      const float wij = wi[di] * wj[dj];
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) {
        float v = __ldg(f + row + K[dk]);
        if (DIFF) v = v - __ldg(fs + row + K[dk]);
        acc += wij * wk[dk] * v;
      }
    }
  return acc;
}

__device__ __forceinline__ void sample_vel(const float* const f[3], const float x[3], float inv_dx, int nx, int ny,
                                           int nz, float out[3]) {
  Frame fr;
  make_frame(x, inv_dx, nx, ny, nz, fr);
#pragma unroll
  for (int c = 0; c < 3; ++c) out[c] = sample_c<false>(f[c], nullptr, c, fr, ny, nz);
}

// pfflip/kernels.py:630-679: a particle inside a solid cell moves out along the
// axis with the nearest free cell (at most 7 cells), its inward velocity zeroed
__device__ __forceinline__ void push_out_of_solids(const int* __restrict__ solid, int nx, int ny, int nz, float dx,
                                                   float x[3], float v[3]) {
  const int i = min(max((int)(x[0] / dx), 0), nx - 1);
  const int j = min(max((int)(x[1] / dx), 0), ny - 1);
  const int k = min(max((int)(x[2] / dx), 0), nz - 1);
  if (solid[((long long)i * ny + j) * nz + k] == 0) return;
  float best = 1.0e9f;
  int bax = 0, bsg = 1;
  for (int d = 0; d < 6; ++d) {
    const int ax = d / 2, sg = (d % 2 == 0) ? -1 : 1;
    for (int t = 1; t < 8; ++t) {
      const int ii = i + (ax == 0 ? sg * t : 0), jj = j + (ax == 1 ? sg * t : 0), kk = k + (ax == 2 ? sg * t : 0);
      if (ii < 0 || jj < 0 || kk < 0 || ii >= nx || jj >= ny || kk >= nz) break;
      if (solid[((long long)ii * ny + jj) * nz + kk] == 0) {
        const float dist = (float)t;
        if (dist < best) {
          best = dist;
          bax = ax;
          bsg = sg;
        }
        break;
      }
    }
  }
  if (best <= 1.0e8f) {
    const float off = (best + 0.5f) * dx * (float)bsg;
    // x[bax] and v[bax] through compile-time indices: a runtime index would
    // keep x and v in local memory for the whole particle loop
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (c != bax) continue;
      x[c] = x[c] + off;
      if ((float)bsg * v[c] < 0.f) v[c] = 0.f;
    }
  }
}

__global__ void __launch_bounds__(256) k_g2p_advect(const __grid_constant__ G2PArgs a) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += (long long)gridDim.x * blockDim.x) {
    float4 P = a.pos[p];
    float4 V = a.vel[p];
    const int flags = __float_as_int(P.w);
    const int pstate = (flags >> PF_PSTATE_SHIFT) & 3;
    const bool liquid = (flags & PF_FLAG_LIQUID) != 0;
    float x[3] = {P.x, P.y, P.z};
    float v[3] = {V.x, V.y, V.z};
    if (a.do_g2p && pstate == 0) {
      const float alpha = liquid ? a.a_liq : a.a_air;
      Frame fr;
      make_frame(x, a.inv_dx, a.nx, a.ny, a.nz, fr);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float delta = sample_c<true>(a.u[c], a.us[c], c, fr, a.ny, a.nz);
        const float pic = sample_c<false>(a.u[c], nullptr, c, fr, a.ny, a.nz);
        v[c] = alpha * (v[c] + delta) + (1.f - alpha) * pic;
      }
    }
    if (a.do_advect) {
      if (pstate == 0) {
        const float* const* f = liquid ? a.ul : a.u;
        float k1[3], k2[3], k3[3], y[3];
        sample_vel(f, x, a.inv_dx, a.nx, a.ny, a.nz, k1);
        const float h1 = 0.5f * a.dt, h2 = 0.75f * a.dt;
#pragma unroll
        for (int c = 0; c < 3; ++c) y[c] = x[c] + h1 * k1[c];
        sample_vel(f, y, a.inv_dx, a.nx, a.ny, a.nz, k2);
#pragma unroll
        for (int c = 0; c < 3; ++c) y[c] = x[c] + h2 * k2[c];
        sample_vel(f, y, a.inv_dx, a.nx, a.ny, a.nz, k3);
        const float c1 = 2.0f / 9.0f, c2 = 3.0f / 9.0f, c3 = 4.0f / 9.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float xn = x[c] + a.dt * (c1 * k1[c] + c2 * k2[c] + c3 * k3[c]);
          x[c] = fminf(fmaxf(xn, a.lo[c]), a.hi[c]);
        }
      }
      if (pstate != 2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (x[c] <= a.lo[c]) {
            x[c] = a.lo[c];
            v[c] = fmaxf(v[c], 0.f);
          } else if (x[c] >= a.hi[c]) {
            x[c] = a.hi[c];
            v[c] = fminf(v[c], 0.f);
          }
        }
        if (a.solid) push_out_of_solids(a.solid, a.nx, a.ny, a.nz, a.dx, x, v);
      }
    }
    P.x = x[0]; P.y = x[1]; P.z = x[2];
    V.x = v[0]; V.y = v[1]; V.z = v[2];
    a.pos[p] = P;
    a.vel[p] = V;
  }
}

// ---------------------------------------------------------------- paired taps
// The same particle pass reading the face fields through quads: for every face
// f = (i, j, k) of a face grid, q[f] = (v[j][k], v[j][k+1], v[j+1][k],
// v[j+1][k+1]) of the same i-plane, with j+1 -> j and k+1 -> k on the last
// plane of the grid.  A trilinear sample is then two 16-byte loads (the lower
// and the upper i-plane) instead of eight gathers.  Interpolation runs as
// lerp chains (t (b - a) + a) over the quads; the reference's weighted sum of
// the eight taps rounds differently, within an ulp or two.  u, u* and the
// extrapolated field ul each get their quads.
struct FacePack {
  FaceSpace s;
  const float* u[3];
  const float* us[3];
  const float* ul[3];
  float4* qu[3];
  float4* qs[3];
  float4* ql[3];
};

struct G2PPackedArgs {
  long long n;
  int nx, ny, nz;
  float dx, inv_dx, dt, a_liq, a_air;
  float lo[3], hi[3];
  float4* pos;
  float4* vel;
  const float4* qu[3];
  const float4* qs[3];
  const float4* ql[3];
  const int* solid;
  int do_g2p, do_advect;
  float* max_speed;  // NULL, or max |v| of the FLIP particles after the pass
};

__global__ void __launch_bounds__(C3_NT) k_pack_faces(FacePack fp) {
  long long f;
  int i, j, k;
  const int ax = locate(fp.s, &f, &i, &j, &k);
  if (ax < 0 || ax > 2) return;
  const int n1 = fp.s.ny + (ax == 1), n2 = fp.s.nz + (ax == 2);
  const long long dk = (k < n2 - 1) ? 1 : 0, dj = (j < n1 - 1) ? n2 : 0;
  const float* u = fp.u[ax];
  fp.qu[ax][f] = make_float4(u[f], u[f + dk], u[f + dj], u[f + dj + dk]);
  if (const float* us = fp.us[ax]) fp.qs[ax][f] = make_float4(us[f], us[f + dk], us[f + dj], us[f + dj + dk]);
  if (const float* ul = fp.ul[ax]) fp.ql[ax][f] = make_float4(ul[f], ul[f + dk], ul[f + dj], ul[f + dj + dk]);
}

// Per position, the lower tap index and the upper weight of each axis d for
// node offset 0 (v = 0: the normal axis of face grid d, extent n_d + 1) and
// 0.5 (v = 1: extent n_d), as pfflip/kernels.py:52-79 computes them:
//   g = x/dx - o, i0 = floor(g), t = g - i0, taps clamp(i0) and clamp(i0 + 1).
// The offset-0.5 frame follows from the offset-0 one: with q = x/dx,
// i = floor(q) and s = q - i, floor(q - 0.5) is i (s >= 0.5) or i - 1 and
// t = s - 0.5 or s + 0.5, the binary32 values the reference computes wherever
// its two taps differ (q - 0.5 is exact for q >= 0.5; below, both taps clamp
// to index 0).  The index clamps are folded into the weight: both taps at 0
// is taps (0, 1) with t = 0, both at the last index is (last - 1, last) with
// t = 1, so the upper tap is always lo + 1; frames away from the walls skip
// the clamps.
struct LeanFrame {
  int lo[3][2];
  float t[3][2];
};

__device__ __forceinline__ void lean_frame(const float x[3], float inv_dx, const int n[3], LeanFrame& f) {
  bool edge = false;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float q = x[d] * inv_dx;
    const float fl = floorf(q);
    const int i = (int)fl;
    const float s = q - fl;
    const bool up = s >= 0.5f;
    f.lo[d][0] = i;
    f.t[d][0] = s;
    f.lo[d][1] = up ? i : i - 1;
    f.t[d][1] = s + (up ? -0.5f : 0.5f);
    edge = edge || i < 1 || i > n[d] - 2;
  }
  if (edge) {
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const int last = v == 0 ? n[d] : n[d] - 1;
        if (f.lo[d][v] < 0) {
          f.lo[d][v] = 0;
          f.t[d][v] = 0.f;
        } else if (f.lo[d][v] >= last) {
          f.lo[d][v] = last - 1;
          f.t[d][v] = 1.f;
        }
      }
  }
}

__device__ __forceinline__ float lerpf(float a, float b, float t) { return fmaf(t, b - a, a); }

// bilinear in (j, k) of one quad (v[j][k], v[j][k+1], v[j+1][k], v[j+1][k+1])
__device__ __forceinline__ float bilerp_q(float4 v, float tj, float tk) {
  return lerpf(lerpf(v.x, v.y, tk), lerpf(v.z, v.w, tk), tj);
}

// face grid C: node offsets of the three axes (0 on the normal axis), the
// quad index of the frame's lower (i, j, k) taps, and the upper-plane stride
template <int C> struct Comp {
  static constexpr int VI = C == 0 ? 0 : 1, VJ = C == 1 ? 0 : 1, VK = C == 2 ? 0 : 1;
};

template <int C>
__device__ __forceinline__ int quad_row(const LeanFrame& f, int n1, int n2) {
  return (f.lo[0][Comp<C>::VI] * n1 + f.lo[1][Comp<C>::VJ]) * n2 + f.lo[2][Comp<C>::VK];
}

// the two quads (lower and upper i-plane) of one component's field at the
// taps of a frame, and the quad row they were read from
struct QuadPair {
  float4 lo, hi;
  int row;
};

template <int C> __device__ __forceinline__ float lerp_pair(const QuadPair& q, const LeanFrame& f) {
  const float tj = f.t[1][Comp<C>::VJ], tk = f.t[2][Comp<C>::VK];
  return lerpf(bilerp_q(q.lo, tj, tk), bilerp_q(q.hi, tj, tk), f.t[0][Comp<C>::VI]);
}

// G2P sample of component C: delta = I(u - u*) tap by tap, pic = I(u); the u
// quads stay in qp
template <int C>
__device__ __forceinline__ void sample_g2p_lean(const float4* __restrict__ qu, const float4* __restrict__ qs,
                                                const LeanFrame& f, int n1, int n2, float& delta, float& pic,
                                                QuadPair& qp) {
  const int row = quad_row<C>(f, n1, n2);
  const int up = n1 * n2;
  const float4 u0 = __ldg(qu + row), u1 = __ldg(qu + row + up);
  const float4 s0 = __ldg(qs + row), s1 = __ldg(qs + row + up);
  const float tj = f.t[1][Comp<C>::VJ], tk = f.t[2][Comp<C>::VK], ti = f.t[0][Comp<C>::VI];
  pic = lerpf(bilerp_q(u0, tj, tk), bilerp_q(u1, tj, tk), ti);
  const float4 d0 = make_float4(u0.x - s0.x, u0.y - s0.y, u0.z - s0.z, u0.w - s0.w);
  const float4 d1 = make_float4(u1.x - s1.x, u1.y - s1.y, u1.z - s1.z, u1.w - s1.w);
  delta = lerpf(bilerp_q(d0, tj, tk), bilerp_q(d1, tj, tk), ti);
  qp.lo = u0;
  qp.hi = u1;
  qp.row = row;
}

// RK3 sample of component C at frame f through the quads of the previous
// sample of the same field: a stage moves a particle a fraction of a cell, so
// its taps mostly stay where they were and only the lanes whose taps moved
// load.  The quads are the same values either way, so the sample is too.
template <int C>
__device__ __forceinline__ float sample_reuse(const float4* __restrict__ q, QuadPair& qp, const LeanFrame& f,
                                              int n1, int n2) {
  const int row = quad_row<C>(f, n1, n2);
  if (row != qp.row) {
    qp.lo = __ldg(q + row);
    qp.hi = __ldg(q + row + n1 * n2);
    qp.row = row;
  }
  return lerp_pair<C>(qp, f);
}

// RK3 sample of the velocity: liquid particles read the extrapolated field,
// air the raw one
__device__ __forceinline__ void sample_vel_reuse(const float4* const* fld, QuadPair qp[3], int ny, int nz,
                                                 const LeanFrame& f, float out[3]) {
  out[0] = sample_reuse<0>(fld[0], qp[0], f, ny, nz);
  out[1] = sample_reuse<1>(fld[1], qp[1], f, ny + 1, nz);
  out[2] = sample_reuse<2>(fld[2], qp[2], f, ny, nz + 1);
}

__global__ void __launch_bounds__(256, 3) k_g2p_advect_packed(const __grid_constant__ G2PPackedArgs a) {
  float vmax = 0.f;  // CFL speed^2 of this thread's FLIP particles (pfflip/kernels.py:552-564)
  const int nn[3] = {a.nx, a.ny, a.nz};
  // each warp walks one contiguous chunk of the cell-sorted streams, 32
  // particles at a time: its successive samples fall in neighbouring cells,
  // whose quads are still in L1 (a grid-stride walk would jump to unrelated
  // cells at every step)
  long long c0, c1;
  warp_chunk(a.n, c0, c1);
  for (long long p = c0 + (threadIdx.x & 31); p < c1; p += 32) {
    float4 P = a.pos[p];
    float4 V = a.vel[p];
    const int flags = __float_as_int(P.w);
    const int pstate = (flags >> PF_PSTATE_SHIFT) & 3;
    const bool liquid = (flags & PF_FLAG_LIQUID) != 0;
    float x[3] = {P.x, P.y, P.z};
    float v[3] = {V.x, V.y, V.z};
    const bool flip = pstate == 0;
    LeanFrame fx;
    if (flip && (a.do_g2p || a.do_advect)) lean_frame(x, a.inv_dx, nn, fx);
    float pic[3];  // I(u) at x: an air particle's first RK3 stage samples the same field there
    QuadPair qp[3];  // per component, the quads of the last sample of the RK3 field
#pragma unroll
    for (int c = 0; c < 3; ++c) qp[c].row = -1;
    if (a.do_g2p && flip) {
      const float alpha = liquid ? a.a_liq : a.a_air;
      float delta[3];
      sample_g2p_lean<0>(a.qu[0], a.qs[0], fx, a.ny, a.nz, delta[0], pic[0], qp[0]);
      sample_g2p_lean<1>(a.qu[1], a.qs[1], fx, a.ny + 1, a.nz, delta[1], pic[1], qp[1]);
      sample_g2p_lean<2>(a.qu[2], a.qs[2], fx, a.ny, a.nz + 1, delta[2], pic[2], qp[2]);
#pragma unroll
      for (int c = 0; c < 3; ++c) v[c] = alpha * (v[c] + delta[c]) + (1.f - alpha) * pic[c];
    }
    if (a.do_advect) {
      if (flip) {
        float k1[3], k2[3], k3[3], y[3];
        const float4* const* fld = liquid ? a.ql : a.qu;
        if (a.do_g2p && !liquid) {
#pragma unroll
          for (int c = 0; c < 3; ++c) k1[c] = pic[c];  // qp holds the u quads at x
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c) qp[c].row = -1;  // qp held u (liquid: the RK3 field is ul)
          sample_vel_reuse(fld, qp, a.ny, a.nz, fx, k1);
        }
        const float h1 = 0.5f * a.dt, h2 = 0.75f * a.dt;
#pragma unroll
        for (int c = 0; c < 3; ++c) y[c] = x[c] + h1 * k1[c];
        LeanFrame fy;
        lean_frame(y, a.inv_dx, nn, fy);
        sample_vel_reuse(fld, qp, a.ny, a.nz, fy, k2);
#pragma unroll
        for (int c = 0; c < 3; ++c) y[c] = x[c] + h2 * k2[c];
        lean_frame(y, a.inv_dx, nn, fy);
        sample_vel_reuse(fld, qp, a.ny, a.nz, fy, k3);
        const float c1 = 2.0f / 9.0f, c2 = 3.0f / 9.0f, c3 = 4.0f / 9.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float xn = x[c] + a.dt * (c1 * k1[c] + c2 * k2[c] + c3 * k3[c]);
          x[c] = fminf(fmaxf(xn, a.lo[c]), a.hi[c]);
        }
      }
      if (pstate != 2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (x[c] <= a.lo[c]) {
            x[c] = a.lo[c];
            v[c] = fmaxf(v[c], 0.f);
          } else if (x[c] >= a.hi[c]) {
            x[c] = a.hi[c];
            v[c] = fminf(v[c], 0.f);
          }
        }
        if (a.solid) push_out_of_solids(a.solid, a.nx, a.ny, a.nz, a.dx, x, v);
      }
    }
    P.x = x[0]; P.y = x[1]; P.z = x[2];
    V.x = v[0]; V.y = v[1]; V.z = v[2];
    a.pos[p] = P;
    a.vel[p] = V;
    if (flip) vmax = fmaxf(vmax, v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    // the records of the particle two iterations on into L2, so that its chain
    // of dependent gathers starts from an L2 hit (a prefetch holds no
    // register; issued here, where few values are live)
    const long long q = p + 64;
    if (q < c1) {
      asm volatile("prefetch.global.L2 [%0];" ::"l"(a.pos + q));
      asm volatile("prefetch.global.L2 [%0];" ::"l"(a.vel + q));
    }
  }
  if (a.max_speed) {  // uniform: every thread of the grid takes this branch or none does
    __shared__ float sh[40];
    // sqrt is correctly rounded and monotone: the root of the max is the max of the roots
    vmax = sqrtf(block_max<256>(vmax, sh));
    if (threadIdx.x == 0) atomic_max_nonneg(a.max_speed, vmax);
  }
}

}  // namespace pf

using namespace pf;

extern "C" int pf_g2p_advect(const pf_grid* g, int64_t n, float* pos4, float* vel4, const float* vel_x,
                             const float* vel_y, const float* vel_z, const float* vstar_x, const float* vstar_y,
                             const float* vstar_z, const float* vliq_x, const float* vliq_y, const float* vliq_z,
                             const int32_t* solid, float alpha_liquid, float alpha_air, float dt, const float lo[3],
                             const float hi[3], int32_t do_g2p, int32_t do_advect, void* stream) {
  PF_REQUIRE(g && pos4 && vel4 && vel_x && vel_y && vel_z, "null argument");
  PF_REQUIRE(!do_g2p || (vstar_x && vstar_y && vstar_z), "u* fields required for G2P");
  PF_REQUIRE(!do_advect || (vliq_x && vliq_y && vliq_z && lo && hi), "extrapolated fields and bounds required");
  PF_REQUIRE(aligned16(pos4) && aligned16(vel4), "particle streams must be 16-byte aligned");
  if (n <= 0) return PF_OK;
  G2PArgs a;
  a.n = n;
  a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
  a.dx = g->dx;
  a.inv_dx = (float)(1.0 / (double)g->dx);  // exact for the power-of-two spacings of the benchmarks
  a.dt = dt;
  a.a_liq = alpha_liquid; a.a_air = alpha_air;
  for (int c = 0; c < 3; ++c) {
    a.lo[c] = lo ? lo[c] : 0.f;
    a.hi[c] = hi ? hi[c] : 0.f;
  }
  a.pos = reinterpret_cast<float4*>(pos4);
  a.vel = reinterpret_cast<float4*>(vel4);
  a.u[0] = vel_x; a.u[1] = vel_y; a.u[2] = vel_z;
  a.us[0] = vstar_x; a.us[1] = vstar_y; a.us[2] = vstar_z;
  a.ul[0] = vliq_x; a.ul[1] = vliq_y; a.ul[2] = vliq_z;
  a.solid = solid;
  a.do_g2p = do_g2p;
  a.do_advect = do_advect;
  k_g2p_advect<<<grid_for(n, 256, kNumSMs * 16), 256, 0, S(stream)>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}

namespace {

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// workspace layout: per axis the float4 (u, u*) pairs, then the float2 ul pairs
// workspace layout: per axis the quads of u, of u* and of the extrapolated field
size_t packed_bytes(const pf_grid* g, size_t offs[9]) {
  const FaceSpace sp = make_space(g->nx, g->ny, g->nz);
  size_t off = 0;
  for (int f = 0; f < 3; ++f)
    for (int c = 0; c < 3; ++c) {
      offs[3 * f + c] = off;
      off += align256((size_t)sp.nf[c] * sizeof(float4));
    }
  return off;
}

}  // namespace

extern "C" size_t pf_g2p_workspace_bytes(const pf_grid* g) {
  if (!g || g->nx <= 0 || g->ny <= 0 || g->nz <= 0) return 0;
  size_t offs[9];
  return packed_bytes(g, offs);
}

extern "C" int pf_g2p_advect_packed(const pf_grid* g, int64_t n, float* pos4, float* vel4, const float* vel_x,
                                    const float* vel_y, const float* vel_z, const float* vstar_x,
                                    const float* vstar_y, const float* vstar_z, const float* vliq_x,
                                    const float* vliq_y, const float* vliq_z, const int32_t* solid,
                                    float alpha_liquid, float alpha_air, float dt, const float lo[3],
                                    const float hi[3], int32_t do_g2p, int32_t do_advect, float* max_speed,
                                    void* workspace, size_t workspace_bytes, void* stream) {
  PF_REQUIRE(g && pos4 && vel4 && vel_x && vel_y && vel_z, "null argument");
  PF_REQUIRE(g->nx > 0 && g->ny > 0 && g->nz > 0, "bad grid");
  PF_REQUIRE(g->nx >= 2 && g->ny >= 2 && g->nz >= 2, "the quad pass needs at least 2 cells per axis");
  PF_REQUIRE(!do_g2p || (vstar_x && vstar_y && vstar_z), "u* fields required for G2P");
  PF_REQUIRE(!do_advect || (vliq_x && vliq_y && vliq_z && lo && hi), "extrapolated fields and bounds required");
  PF_REQUIRE(aligned16(pos4) && aligned16(vel4), "particle streams must be 16-byte aligned");
  size_t offs[9];
  PF_REQUIRE(workspace && workspace_bytes >= packed_bytes(g, offs), "workspace too small");
  PF_REQUIRE((reinterpret_cast<uintptr_t>(workspace) & 255) == 0, "workspace must be 256-byte aligned");
  PF_REQUIRE((long long)g->nx * g->ny * (g->nz + 1) < (1LL << 31) &&
                 (long long)(g->nx + 1) * g->ny * g->nz < (1LL << 31) &&
                 (long long)g->nx * (g->ny + 1) * g->nz < (1LL << 31),
             "face arrays must hold < 2^31 entries");
  cudaStream_t s = S(stream);
  if (max_speed) PF_CUDA_TRY(cudaMemsetAsync(max_speed, 0, sizeof(float), s));
  if (n <= 0) return PF_OK;
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  FacePack fp;
  fp.s = make_space(g->nx, g->ny, g->nz);
  const float* u[3] = {vel_x, vel_y, vel_z};
  const float* us[3] = {vstar_x, vstar_y, vstar_z};
  const float* ul[3] = {vliq_x, vliq_y, vliq_z};
  G2PPackedArgs a;
  for (int c = 0; c < 3; ++c) {
    fp.u[c] = u[c];
    fp.us[c] = do_g2p ? us[c] : nullptr;
    fp.ul[c] = do_advect ? ul[c] : nullptr;
    fp.qu[c] = reinterpret_cast<float4*>(ws + offs[c]);
    fp.qs[c] = do_g2p ? reinterpret_cast<float4*>(ws + offs[3 + c]) : nullptr;
    fp.ql[c] = do_advect ? reinterpret_cast<float4*>(ws + offs[6 + c]) : nullptr;
    a.qu[c] = fp.qu[c];
    a.qs[c] = fp.qs[c];
    a.ql[c] = fp.ql[c];
  }
  k_pack_faces<<<grid_faces(g->nx, g->ny, g->nz, false), C3_NT, 0, s>>>(fp);
  PF_LAUNCHED();
  a.n = n;
  a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
  a.dx = g->dx;
  a.inv_dx = (float)(1.0 / (double)g->dx);
  a.dt = dt;
  a.a_liq = alpha_liquid; a.a_air = alpha_air;
  for (int c = 0; c < 3; ++c) {
    a.lo[c] = lo ? lo[c] : 0.f;
    a.hi[c] = hi ? hi[c] : 0.f;
  }
  a.pos = reinterpret_cast<float4*>(pos4);
  a.vel = reinterpret_cast<float4*>(vel4);
  a.solid = solid;
  a.do_g2p = do_g2p;
  a.do_advect = do_advect;
  a.max_speed = max_speed;
  // 64 CTAs per SM: warp chunks of ~750 particles at 128^3 / 27 ppc, long
  // enough for the walk's L1 reuse, short enough that the chunks balance
  k_g2p_advect_packed<<<grid_for(n, 256, kNumSMs * 64), 256, 0, s>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}
