// P2G on sm_100a: eq. (3)-(6) mass/momentum splatting to the three MAC face
// grids and the cell grid (reference pfflip/kernels.py:100-209, launched four
// times by pfflip/sim.py:205-228 with one global atomic per weight).
//
// Particles are sorted by cell (pf_sort_particles).  One CTA owns a tile of
// TI x TJ x TK cells and keeps all 8 accumulators (mass and momentum of the 3
// face grids, cell mass, cell weight sum) of the tile plus a one-node halo in
// shared memory.  A warp owns one row of TK = 32 cells along k at a time; the
// row's particles (a contiguous range after the sort) are split evenly over
// the lanes, so adjacent lanes work on adjacent cells and their shared-memory
// atomics rarely meet.  After the tile's particles are done, each accumulator
// node is flushed once with a global reduction (red.global.add.f32); nodes
// that a rounding edge case puts outside the tile box go to global memory
// directly.  The weight window and weight of every (particle, node) pair
// follow the reference exactly: window floor(c - R) + 1 .. floor(c + R)
// clamped to the grid, w = max(1 - d^2/r^2, 0)^3 (d^2/r^2 as d^2 * (1/r^2)).
#include "pf_common.cuh"

namespace pf {

constexpr int PG_TI = 4, PG_TJ = 8, PG_TK = 32;
constexpr int PG_NT = 256;
constexpr int PG_BI = PG_TI + 2, PG_BJ = PG_TJ + 2, PG_BK = PG_TK + 2;
constexpr int PG_BOX = PG_BI * PG_BJ * PG_BK;  // nodes per accumulator box
constexpr int PG_NACC = 8;
constexpr size_t PG_SMEM = sizeof(float) * PG_NACC * PG_BOX;

struct P2GArgs {
  int nx, ny, nz;
  float dx, inv_r2, R;
  float rho_l, rho_g;
  const float4* pos;
  const float4* vel;
  const int* cell_start;
  float* out[PG_NACC];  // mass x,y,z, mom x,y,z, cell_mass, cell_wsum
};

__device__ __forceinline__ float splat_w(float d2, float inv_r2) {
  float t = fmaxf(1.f - d2 * inv_r2, 0.f);
  return t * t * t;
}

__global__ void __launch_bounds__(PG_NT) k_p2g(P2GArgs a) {
  extern __shared__ __align__(16) float acc[];  // [PG_NACC][PG_BOX]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int k0 = blockIdx.x * PG_TK, j0 = blockIdx.y * PG_TJ, i0 = blockIdx.z * PG_TI;
  for (int e = tid; e < PG_NACC * PG_BOX; e += PG_NT) acc[e] = 0.f;
  __syncthreads();

  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const float dx = a.dx, R = a.R, inv_r2 = a.inv_r2;
  const int k1 = min(k0 + PG_TK, nz);

  for (int row = warp; row < PG_TI * PG_TJ; row += PG_NT / 32) {
    const int i = i0 + row / PG_TJ, j = j0 + row % PG_TJ;
    if (i >= nx || j >= ny || k0 >= nz) continue;
    const int key0 = (i * ny + j) * nz + k0;
    const int rs = a.cell_start[key0], re = a.cell_start[key0 + (k1 - k0)];
    const int len = re - rs;
    const int chunk = (len + 31) >> 5;
    const int ps = rs + lane * chunk, pe = min(re, ps + chunk);
    for (int t = ps; t < pe; ++t) {
      const float4 P = __ldg(a.pos + t);
      const int flags = __float_as_int(P.w);
      if ((flags >> PF_PSTATE_SHIFT) & 3) continue;  // droplets / dead particles do not splat
      const float4 V = __ldg(a.vel + t);
      const float m = (flags & PF_FLAG_LIQUID) ? a.rho_l : a.rho_g;
      const float q[3] = {P.x / dx, P.y / dx, P.z / dx};
      const float xp[3] = {P.x, P.y, P.z};
      const float up[3] = {V.x, V.y, V.z};
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        // node offsets o_d and grid extents of grid g (3 = cell centres)
        float o[3];
        int n[3], blo[3];
        const int tile0[3] = {i0, j0, k0};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const bool normal = (g == d);
          o[d] = normal ? 0.f : 0.5f;
          n[d] = (d == 0 ? nx : d == 1 ? ny : nz) + (normal ? 1 : 0);
          blo[d] = tile0[d] - (normal ? 0 : 1);
        }
        int lo[3], hi[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const float c = q[d] - o[d];
          lo[d] = max((int)floorf(c - R) + 1, 0);
          hi[d] = min((int)floorf(c + R), n[d] - 1);
        }
        const float v1 = m;
        const float v2 = (g < 3) ? up[g] : 0.f;
        float* A1 = acc + (g < 3 ? g : 6) * PG_BOX;
        float* A2 = acc + (g < 3 ? 3 + g : 7) * PG_BOX;
        float* G1 = a.out[g < 3 ? g : 6];
        float* G2 = a.out[g < 3 ? 3 + g : 7];
        for (int ii = lo[0]; ii <= hi[0]; ++ii) {
          const float fx = ((float)ii + o[0]) * dx - xp[0];
          for (int jj = lo[1]; jj <= hi[1]; ++jj) {
            const float fy = ((float)jj + o[1]) * dx - xp[1];
            const float fxy = fx * fx + fy * fy;
            for (int kk = lo[2]; kk <= hi[2]; ++kk) {
              const float fz = ((float)kk + o[2]) * dx - xp[2];
              const float w = splat_w(fxy + fz * fz, inv_r2);
              if (w > 0.f) {
                const float wm = w * v1;
                const float w2 = (g < 3) ? wm * v2 : w;
                const int li = ii - blo[0], lj = jj - blo[1], lk = kk - blo[2];
                if ((unsigned)li < (unsigned)PG_BI && (unsigned)lj < (unsigned)PG_BJ &&
                    (unsigned)lk < (unsigned)PG_BK) {
                  const int e = (li * PG_BJ + lj) * PG_BK + lk;
                  atomicAdd(A1 + e, wm);
                  atomicAdd(A2 + e, w2);
                } else {
                  const long long ge = ((long long)ii * n[1] + jj) * n[2] + kk;
                  atomicAdd(G1 + ge, wm);
                  atomicAdd(G2 + ge, w2);
                }
              }
            }
          }
        }
      }
    }
  }
  __syncthreads();
  // flush: each node once
  for (int e = tid; e < PG_NACC * PG_BOX; e += PG_NT) {
    const float v = acc[e];
    if (v == 0.f) continue;
    const int arr = e / PG_BOX, b = e % PG_BOX;
    const int g = arr < 6 ? arr % 3 : 3;
    const int li = b / (PG_BJ * PG_BK), lj = (b / PG_BK) % PG_BJ, lk = b % PG_BK;
    const int gi = i0 + li - (g == 0 ? 0 : 1);
    const int gj = j0 + lj - (g == 1 ? 0 : 1);
    const int gk = k0 + lk - (g == 2 ? 0 : 1);
    const int n0 = nx + (g == 0), n1 = ny + (g == 1), n2 = nz + (g == 2);
    if (gi < 0 || gj < 0 || gk < 0 || gi >= n0 || gj >= n1 || gk >= n2) continue;
    atomicAdd(a.out[arr] + ((long long)gi * n1 + gj) * n2 + gk, v);
  }
}

}  // namespace pf

using namespace pf;

extern "C" int pf_p2g(const pf_grid* g, int64_t n, const float* pos4, const float* vel4, const int32_t* cell_start,
                      float rho_l, float rho_g, float r_p, float* mass_x, float* mass_y, float* mass_z, float* mom_x,
                      float* mom_y, float* mom_z, float* cell_mass, float* cell_wsum, void* stream) {
  PF_REQUIRE(g && pos4 && vel4 && cell_start && mass_x && mass_y && mass_z && mom_x && mom_y && mom_z && cell_mass &&
                 cell_wsum,
             "null argument");
  PF_REQUIRE(g->nx > 0 && g->ny > 0 && g->nz > 0 && g->dx > 0.f && r_p > 0.f, "bad grid");
  PF_REQUIRE(aligned16(pos4) && aligned16(vel4), "particle streams must be 16-byte aligned");
  static bool attr_set = false;
  if (!attr_set) {
    PF_CUDA_TRY(cudaFuncSetAttribute(k_p2g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PG_SMEM));
    attr_set = true;
  }
  cudaStream_t s = S(stream);
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const size_t fx = (size_t)(nx + 1) * ny * nz, fy = (size_t)nx * (ny + 1) * nz, fz = (size_t)nx * ny * (nz + 1),
               nc = (size_t)nx * ny * nz;
  float* outs[PG_NACC] = {mass_x, mass_y, mass_z, mom_x, mom_y, mom_z, cell_mass, cell_wsum};
  const size_t sizes[PG_NACC] = {fx, fy, fz, fx, fy, fz, nc, nc};
  for (int q = 0; q < PG_NACC; ++q) PF_CUDA_TRY(cudaMemsetAsync(outs[q], 0, sizes[q] * sizeof(float), s));
  if (n <= 0) return PF_OK;
  P2GArgs a;
  a.nx = nx; a.ny = ny; a.nz = nz;
  a.dx = g->dx;
  a.R = r_p / g->dx;
  a.inv_r2 = 1.f / (r_p * r_p);
  a.rho_l = rho_l; a.rho_g = rho_g;
  a.pos = reinterpret_cast<const float4*>(pos4);
  a.vel = reinterpret_cast<const float4*>(vel4);
  a.cell_start = cell_start;
  for (int q = 0; q < PG_NACC; ++q) a.out[q] = outs[q];
  dim3 grid((nz + PG_TK - 1) / PG_TK, (ny + PG_TJ - 1) / PG_TJ, (nx + PG_TI - 1) / PG_TI);
  k_p2g<<<grid, PG_NT, PG_SMEM, s>>>(a);
  PF_LAUNCHED();
  return PF_OK;
}
