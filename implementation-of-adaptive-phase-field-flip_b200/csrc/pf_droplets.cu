// Escaped particles, Lagrangian droplets and the spray density field on
// sm_100a (reference pfflip/droplets.py, run by pfflip/sim.py:343-401).
//
// Droplets share the particle streams: a particle's state lives in bits 1-2 of
// its flags (0 FLIP, 1 droplet, 2 dead), so a conversion is a flag change.
// The droplet radius is a separate float per particle that follows the sort
// (pf_permute_f32).
//
// Random numbers.  The reference draws radii and spray emission from Warp's
// rand_init/randn/randf stream, which is not reproduced here.  This library
// uses a counter-based stream of its own: the 32-bit PCG-RXS-M-XS hash
// (O'Neill 2014; as a GPU hash, Jarzynski & Olano 2020) seeded per particle
// with hash(hash(seed) + p), uniforms from the top 24 bits, normals by
// Box-Muller.  Radii therefore follow the same log-normal law as the
// reference's, not the same values; everything else is deterministic.
#include "pf_faces.cuh"

namespace pf {

constexpr int kStateFlip = 0, kStateDroplet = 1, kStateDead = 2;

__device__ __forceinline__ uint32_t pcg_hash(uint32_t v) {
  const uint32_t s = v * 747796405u + 2891336453u;
  const uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}

struct DropRng {
  uint32_t s;
  __device__ __forceinline__ DropRng(uint32_t seed, uint32_t p) : s(pcg_hash(pcg_hash(seed) + p)) {}
  __device__ __forceinline__ float uniform() {  // in (0, 1)
    s = pcg_hash(s);
    return ((float)(s >> 8) + 0.5f) * (1.0f / 16777216.0f);
  }
  __device__ __forceinline__ float normal() {
    const float u1 = uniform(), u2 = uniform();
    return sqrtf(-2.0f * logf(u1)) * cosf(6.28318530717958647692f * u2);
  }
};

__device__ __forceinline__ int state_of(int flags) { return (flags >> PF_PSTATE_SHIFT) & 3; }
__device__ __forceinline__ int with_state(int flags, int st) {
  return (flags & ~(3 << PF_PSTATE_SHIFT)) | (st << PF_PSTATE_SHIFT);
}

// trilinear sample of a cell-centred field at x (pfflip/droplets.py:41-64)
__device__ __forceinline__ float sample_cell(const float* __restrict__ f, int nx, int ny, int nz, float dx,
                                             float x, float y, float z) {
  const float g0 = x / dx - 0.5f, g1 = y / dx - 0.5f, g2 = z / dx - 0.5f;
  const int i0 = (int)floorf(g0), j0 = (int)floorf(g1), k0 = (int)floorf(g2);
  const float tx = g0 - (float)i0, ty = g1 - (float)j0, tz = g2 - (float)k0;
  float acc = 0.f;
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    const float wa = a == 0 ? 1.f - tx : tx;
    const int ii = min(max(i0 + a, 0), nx - 1);
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const float wb = b == 0 ? 1.f - ty : ty;
      const int jj = min(max(j0 + b, 0), ny - 1);
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const float wc = c == 0 ? 1.f - tz : tz;
        const int kk = min(max(k0 + c, 0), nz - 1);
        acc += wa * wb * wc * f[((long long)ii * ny + jj) * nz + kk];
      }
    }
  }
  return acc;
}

// trilinear sample of face array `axis` at x (pfflip/droplets.py:282-306)
__device__ __forceinline__ float sample_face_u(const float* __restrict__ f, int nx, int ny, int nz, float dx,
                                               const float x[3], int axis) {
  const int n0 = nx + (axis == 0), n1 = ny + (axis == 1), n2 = nz + (axis == 2);
  const float ox = axis == 0 ? 0.f : 0.5f, oy = axis == 1 ? 0.f : 0.5f, oz = axis == 2 ? 0.f : 0.5f;
  const float g0 = x[0] / dx - ox, g1 = x[1] / dx - oy, g2 = x[2] / dx - oz;
  const int i0 = (int)floorf(g0), j0 = (int)floorf(g1), k0 = (int)floorf(g2);
  const float tx = g0 - (float)i0, ty = g1 - (float)j0, tz = g2 - (float)k0;
  float acc = 0.f;
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    const float wa = a == 0 ? 1.f - tx : tx;
    const int ii = min(max(i0 + a, 0), n0 - 1);
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const float wb = b == 0 ? 1.f - ty : ty;
      const int jj = min(max(j0 + b, 0), n1 - 1);
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const float wc = c == 0 ? 1.f - tz : tz;
        const int kk = min(max(k0 + c, 0), n2 - 1);
        acc += wa * wb * wc * __ldg(f + ((long long)ii * n1 + jj) * n2 + kk);
      }
    }
  }
  return acc;
}

struct ClassifyArgs {
  long long n;
  int nx, ny, nz;
  float dx, delta_phi, r_mu, r_sigma, r_min, r_max;
  uint32_t seed;
  float4* pos;
  const float4* vel;  // .w = the particle's original id, which keys its random stream
  float* drop_r;
  const float* phi;
  int* counters;
};

// pfflip/droplets.py:67-106 classify_escaped
__global__ void __launch_bounds__(256) k_droplet_classify(const __grid_constant__ ClassifyArgs a) {
  int emitted = 0, bubbles = 0, merged = 0;
  long long c0, c1;  // a contiguous chunk of the sorted streams per warp: field samples stay in L1
  warp_chunk(a.n, c0, c1);
  for (long long p = c0 + (threadIdx.x & 31); p < c1; p += 32) {
    float4 P = a.pos[p];
    const int flags = __float_as_int(P.w);
    const int st = state_of(flags);
    if (st == kStateDead) continue;
    const float f = sample_cell(a.phi, a.nx, a.ny, a.nz, a.dx, P.x, P.y, P.z);
    int nst = st;
    if (st == kStateFlip) {
      const bool liquid = (flags & PF_FLAG_LIQUID) != 0;
      if (liquid && f < 0.5f - a.delta_phi) {
        nst = kStateDroplet;
        DropRng rng(a.seed, (uint32_t)__float_as_int(a.vel[p].w));
        const float r = expf(a.r_mu + a.r_sigma * rng.normal());
        a.drop_r[p] = fminf(fmaxf(r, a.r_min), a.r_max);
        ++emitted;
      } else if (!liquid && f > 0.5f + a.delta_phi) {
        nst = kStateDead;
        ++bubbles;
      }
    } else if (f > 0.5f + a.delta_phi) {  // droplet back inside the liquid
      nst = kStateFlip;
      ++merged;
    }
    if (nst != st) {
      P.w = __int_as_float(with_state(flags, nst));
      a.pos[p] = P;
    }
  }
  emitted = warp_sum_int(emitted);
  bubbles = warp_sum_int(bubbles);
  merged = warp_sum_int(merged);
  if ((threadIdx.x & 31) == 0) {
    if (emitted) atomicAdd(a.counters + 0, emitted);
    if (bubbles) atomicAdd(a.counters + 1, bubbles);
    if (merged) atomicAdd(a.counters + 2, merged);
  }
}

// pfflip/droplets.py:153-194 velocity_gradient_magnitude
__global__ void __launch_bounds__(C3_NT) k_velocity_gradient(int nx, int ny, int nz, const float* __restrict__ u,
                                                             const float* __restrict__ v, const float* __restrict__ w,
                                                             float* __restrict__ out, float dx) {
  const Cell3 cc = cell_here();
  if (cc.j >= ny || cc.k >= nz) return;
  const int i = cc.i, j = cc.j, k = cc.k;
  auto U = [&](int a, int b, int c) { return u[((long long)a * ny + b) * nz + c]; };
  auto V = [&](int a, int b, int c) { return v[((long long)a * (ny + 1) + b) * nz + c]; };
  auto W = [&](int a, int b, int c) { return w[((long long)a * ny + b) * (nz + 1) + c]; };
  const float dudx = (U(i + 1, j, k) - U(i, j, k)) / dx;
  const float dvdy = (V(i, j + 1, k) - V(i, j, k)) / dx;
  const float dwdz = (W(i, j, k + 1) - W(i, j, k)) / dx;
  float acc = dudx * dudx + dvdy * dvdy + dwdz * dwdz;
  const int jm = max(j - 1, 0), jp = min(j + 1, ny - 1), km = max(k - 1, 0), kp = min(k + 1, nz - 1);
  const int im = max(i - 1, 0), ip = min(i + 1, nx - 1);
  const float dudy = (0.5f * (U(i, jp, k) + U(i + 1, jp, k)) - 0.5f * (U(i, jm, k) + U(i + 1, jm, k))) / (2.0f * dx);
  const float dudz = (0.5f * (U(i, j, kp) + U(i + 1, j, kp)) - 0.5f * (U(i, j, km) + U(i + 1, j, km))) / (2.0f * dx);
  const float dvdx = (0.5f * (V(ip, j, k) + V(ip, j + 1, k)) - 0.5f * (V(im, j, k) + V(im, j + 1, k))) / (2.0f * dx);
  const float dwdx = (0.5f * (W(ip, j, k) + W(ip, j, k + 1)) - 0.5f * (W(im, j, k) + W(im, j, k + 1))) / (2.0f * dx);
  acc += dudy * dudy + dudz * dudz + dvdx * dvdx + dwdx * dwdx;
  out[((long long)i * ny + j) * nz + k] = sqrtf(acc);
}

struct SprayArgs {
  long long n;
  int nx, ny, nz;
  float dx, threshold, rate, r_mu, r_sigma, r_min, r_max;
  uint32_t seed;
  float4* pos;
  const float4* vel;
  float* drop_r;
  const float* phi;
  const float* shear;
  int* counters;
};

// pfflip/droplets.py:112-150 emit_spray_in_shear
__global__ void __launch_bounds__(256) k_spray_emit(const __grid_constant__ SprayArgs a) {
  int spray = 0;
  long long c0, c1;  // a contiguous chunk of the sorted streams per warp: field samples stay in L1
  warp_chunk(a.n, c0, c1);
  for (long long p = c0 + (threadIdx.x & 31); p < c1; p += 32) {
    float4 P = a.pos[p];
    const int flags = __float_as_int(P.w);
    if (state_of(flags) != kStateFlip || (flags & PF_FLAG_LIQUID) == 0) continue;
    const float f = sample_cell(a.phi, a.nx, a.ny, a.nz, a.dx, P.x, P.y, P.z);
    if (f > 0.9f || f < 0.1f) continue;  // only the interfacial band breaks up
    if (sample_cell(a.shear, a.nx, a.ny, a.nz, a.dx, P.x, P.y, P.z) < a.threshold) continue;
    DropRng rng(a.seed + 104729u, (uint32_t)__float_as_int(a.vel[p].w));
    if (rng.uniform() > a.rate) continue;
    P.w = __int_as_float(with_state(flags, kStateDroplet));
    a.pos[p] = P;
    a.drop_r[p] = fminf(fmaxf(expf(a.r_mu + a.r_sigma * rng.normal()), a.r_min), a.r_max);
    ++spray;
  }
  spray = warp_sum_int(spray);
  if ((threadIdx.x & 31) == 0 && spray) atomicAdd(a.counters + 3, spray);
}

struct AdvanceArgs {
  long long n;
  int nx, ny, nz;
  float dx, dt, g[3], rho_g, rho_l, cd, evap_k, r_min, lo[3], hi[3];
  int max_substeps;
  float4* pos;
  float4* vel;
  float* drop_r;
  const float* u[3];
};

// pfflip/droplets.py:197-279: gravity + sphere drag a = 3 rho_g Cd |v_rel| v_rel
// / (8 rho_l r), per-droplet sub-steps from its own CFL, evaporation
// dr/dt = -k/r by RK2; a droplet leaving the domain or shrinking below r_min
// dies
__global__ void __launch_bounds__(256) k_droplet_advance(AdvanceArgs a) {
  long long c0, c1;  // a contiguous chunk of the sorted streams per warp: field samples stay in L1
  warp_chunk(a.n, c0, c1);
  for (long long p = c0 + (threadIdx.x & 31); p < c1; p += 32) {
    float4 P = a.pos[p];
    const int flags = __float_as_int(P.w);
    if (state_of(flags) != kStateDroplet) continue;
    const float4 V = a.vel[p];
    float x[3] = {P.x, P.y, P.z}, v[3] = {V.x, V.y, V.z};
    float r = a.drop_r[p];
    const float speed = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + 1e-8f;
    const int nsub = min(max((int)(speed * a.dt / (0.5f * a.dx)) + 1, 1), a.max_substeps);
    const float h = a.dt / (float)nsub;
    bool dead = false;
    for (int s = 0; s < nsub && !dead; ++s) {
      float ua[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) ua[c] = sample_face_u(a.u[c], a.nx, a.ny, a.nz, a.dx, x, c);
      const float vr[3] = {ua[0] - v[0], ua[1] - v[1], ua[2] - v[2]};
      const float sr = sqrtf(vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]);
      const bool drag = sr > 0.f && r > 0.f;
      const float coef = drag ? (3.0f * a.rho_g * a.cd * sr / (8.0f * a.rho_l * r)) : 0.f;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float acc = a.g[c] + (drag ? coef * vr[c] : 0.f);
        v[c] = v[c] + h * acc;
        x[c] = x[c] + h * v[c];
      }
      if (a.evap_k > 0.f && r > 0.f) {
        const float k1 = -a.evap_k / r;
        const float rm = fmaxf(r + 0.5f * h * k1, 1e-9f);
        r = r + h * (-a.evap_k / rm);
        if (r <= a.r_min) dead = true;
      }
    }
    if (!dead)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (x[c] <= a.lo[c] || x[c] >= a.hi[c]) dead = true;
    if (dead) {  // the reference leaves position, velocity and radius as they were
      P.w = __int_as_float(with_state(flags, kStateDead));
      a.pos[p] = P;
      continue;
    }
    a.drop_r[p] = r;
    a.vel[p] = make_float4(v[0], v[1], v[2], V.w);
    P.x = x[0]; P.y = x[1]; P.z = x[2];
    a.pos[p] = P;
  }
}

// pfflip/droplets.py:309-353 rasterize_spray: droplet volume splatted
// trilinearly into a float16 density grid of spacing dx_spray
__global__ void __launch_bounds__(256) k_spray_rasterize(long long n, const float4* __restrict__ pos,
                                                         const float* __restrict__ drop_r, __half* density, int sx,
                                                         int sy, int sz, float dxs) {
  long long c0, c1;  // a contiguous chunk per warp: its atomics land on neighbouring cells
  warp_chunk(n, c0, c1);
  for (long long p = c0 + (threadIdx.x & 31); p < c1; p += 32) {
    const float4 P = pos[p];
    if (state_of(__float_as_int(P.w)) != kStateDroplet) continue;
    const float r = drop_r[p];
    const float vol = (4.0f / 3.0f) * 3.14159265f * r * r * r;
    const float g0 = P.x / dxs - 0.5f, g1 = P.y / dxs - 0.5f, g2 = P.z / dxs - 0.5f;
    const int i0 = (int)floorf(g0), j0 = (int)floorf(g1), k0 = (int)floorf(g2);
    const float tx = g0 - (float)i0, ty = g1 - (float)j0, tz = g2 - (float)k0;
    const float cell_vol = dxs * dxs * dxs;
    for (int a = 0; a < 2; ++a) {
      const float wa = a == 0 ? 1.f - tx : tx;
      const int ii = i0 + a;
      if (ii < 0 || ii >= sx) continue;
      for (int b = 0; b < 2; ++b) {
        const float wb = b == 0 ? 1.f - ty : ty;
        const int jj = j0 + b;
        if (jj < 0 || jj >= sy) continue;
        for (int c = 0; c < 2; ++c) {
          const float wc = c == 0 ? 1.f - tz : tz;
          const int kk = k0 + c;
          if (kk < 0 || kk >= sz) continue;
          atomicAdd(density + ((long long)ii * sy + jj) * sz + kk, __float2half(wa * wb * wc * vol / cell_vol));
        }
      }
    }
  }
}

__global__ void k_permute_f32(long long n, const int* __restrict__ perm, const float* __restrict__ in,
                              float* __restrict__ out) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    out[t] = in[perm[t]];
}

}  // namespace pf

using namespace pf;

extern "C" {

int pf_droplet_classify(const pf_grid* g, int64_t n, float* pos4, const float* vel4, float* drop_r,
                        const float* phi_cell, float delta_phi, float r_mu, float r_sigma, float r_min, float r_max, uint32_t seed,
                        int32_t* counters, void* stream) {
  PF_REQUIRE(g && pos4 && vel4 && drop_r && phi_cell && counters, "null argument");
  PF_REQUIRE(aligned16(pos4) && aligned16(vel4), "particle streams must be 16-byte aligned");
  if (n <= 0) return PF_OK;
  ClassifyArgs a;
  a.vel = reinterpret_cast<const float4*>(vel4);
  a.n = n;
  a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
  a.dx = g->dx;
  a.delta_phi = delta_phi;
  a.r_mu = r_mu; a.r_sigma = r_sigma; a.r_min = r_min; a.r_max = r_max;
  a.seed = seed;
  a.pos = reinterpret_cast<float4*>(pos4);
  a.drop_r = drop_r;
  a.phi = phi_cell;
  a.counters = counters;
  k_droplet_classify<<<grid_for(n, 256, kNumSMs * 16), 256, 0, S(stream)>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_velocity_gradient(const pf_grid* g, const float* vel_x, const float* vel_y, const float* vel_z, float* out,
                         void* stream) {
  PF_REQUIRE(g && vel_x && vel_y && vel_z && out, "null argument");
  k_velocity_gradient<<<grid_cells(g->nx, g->ny, g->nz), C3_NT, 0, S(stream)>>>(g->nx, g->ny, g->nz, vel_x, vel_y,
                                                                               vel_z, out, g->dx);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_spray_emit(const pf_grid* g, int64_t n, float* pos4, const float* vel4, float* drop_r, const float* phi_cell,
                  const float* shear,
                  float threshold, float rate, float r_mu, float r_sigma, float r_min, float r_max, uint32_t seed,
                  int32_t* counters, void* stream) {
  PF_REQUIRE(g && pos4 && vel4 && drop_r && phi_cell && shear && counters, "null argument");
  PF_REQUIRE(aligned16(pos4) && aligned16(vel4), "particle streams must be 16-byte aligned");
  if (n <= 0) return PF_OK;
  SprayArgs a;
  a.vel = reinterpret_cast<const float4*>(vel4);
  a.n = n;
  a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
  a.dx = g->dx;
  a.threshold = threshold;
  a.rate = rate;
  a.r_mu = r_mu; a.r_sigma = r_sigma; a.r_min = r_min; a.r_max = r_max;
  a.seed = seed;
  a.pos = reinterpret_cast<float4*>(pos4);
  a.drop_r = drop_r;
  a.phi = phi_cell;
  a.shear = shear;
  a.counters = counters;
  k_spray_emit<<<grid_for(n, 256, kNumSMs * 16), 256, 0, S(stream)>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_droplet_advance(const pf_grid* g, int64_t n, float* pos4, float* vel4, float* drop_r, const float* vel_x,
                       const float* vel_y, const float* vel_z, float dt, const float gravity[3], float rho_g,
                       float rho_l, float drag_cd, float evap_k, float r_min, const float lo[3], const float hi[3],
                       int32_t max_substeps, void* stream) {
  PF_REQUIRE(g && pos4 && vel4 && drop_r && vel_x && vel_y && vel_z && gravity && lo && hi, "null argument");
  PF_REQUIRE(aligned16(pos4) && aligned16(vel4), "particle streams must be 16-byte aligned");
  PF_REQUIRE(max_substeps >= 1, "max_substeps must be >= 1");
  if (n <= 0) return PF_OK;
  AdvanceArgs a;
  a.n = n;
  a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
  a.dx = g->dx;
  a.dt = dt;
  for (int c = 0; c < 3; ++c) {
    a.g[c] = gravity[c];
    a.lo[c] = lo[c];
    a.hi[c] = hi[c];
  }
  a.rho_g = rho_g; a.rho_l = rho_l; a.cd = drag_cd; a.evap_k = evap_k; a.r_min = r_min;
  a.max_substeps = max_substeps;
  a.pos = reinterpret_cast<float4*>(pos4);
  a.vel = reinterpret_cast<float4*>(vel4);
  a.drop_r = drop_r;
  a.u[0] = vel_x; a.u[1] = vel_y; a.u[2] = vel_z;
  k_droplet_advance<<<grid_for(n, 256, kNumSMs * 16), 256, 0, S(stream)>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_spray_rasterize(int64_t n, const float* pos4, const float* drop_r, void* density_f16, int32_t sx, int32_t sy,
                       int32_t sz, float dx_spray, void* stream) {
  PF_REQUIRE(pos4 && drop_r && density_f16 && sx > 0 && sy > 0 && sz > 0 && dx_spray > 0.f, "bad argument");
  PF_REQUIRE(aligned16(pos4), "particle streams must be 16-byte aligned");
  cudaStream_t s = S(stream);
  PF_CUDA_TRY(cudaMemsetAsync(density_f16, 0, sizeof(__half) * (size_t)sx * sy * sz, s));
  if (n <= 0) return PF_OK;
  k_spray_rasterize<<<grid_for(n, 256, kNumSMs * 16), 256, 0, s>>>(
      n, reinterpret_cast<const float4*>(pos4), drop_r, static_cast<__half*>(density_f16), sx, sy, sz, dx_spray);
  PF_LAUNCHED();
  return PF_OK;
}

int pf_permute_f32(int64_t n, const int32_t* perm, const float* in, float* out, void* stream) {
  PF_REQUIRE(n >= 0 && perm && in && out && in != out, "bad argument");
  if (n == 0) return PF_OK;
  k_permute_f32<<<grid_for(n, 256, kNumSMs * 16), 256, 0, S(stream)>>>(n, perm, in, out);
  PF_LAUNCHED();
  return PF_OK;
}

}  // extern "C"
