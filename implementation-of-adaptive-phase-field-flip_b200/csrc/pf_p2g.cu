// P2G on sm_100a: eq. (3)-(6) mass/momentum splatting to the three MAC face
// grids and the cell grid (reference pfflip/kernels.py:100-209, launched four
// times by pfflip/sim.py:205-228 with one global atomic per weight).
//
// Particles are sorted by cell (pf_sort_particles).  One CTA owns a tile of
// TI x TJ x 32 cells and the tile's 8 accumulator boxes (tile + one node
// halo) in shared memory.  A warp owns one row of 32 cells along k and each
// lane one cell: for each grid the lane sums its particles' weights into a
// register box covering every node its cell's particles can reach (3x3x3 for
// the cell grid, 2 along the normal axis of a face grid).  The lanes of a
// row then combine the k-neighbour parts of their boxes with warp shuffles
// and add one value per node to shared memory: ~60 shared atomics per cell
// instead of 64 per particle, and no two lanes of a warp ever add to the same
// node.  Each tile node is flushed to global memory once (red.global.add).
//
// Weights: w = max(1 - d^2/r^2, 0)^3 with d^2 = (fx^2 + fy^2) + fz^2 and
// fx = (n + o)*dx - x in the reference's order (d^2/r^2 as d^2*(1/r^2)).  The
// register box includes nodes outside the reference's window
// floor(c - R) + 1 .. floor(c + R); those lie at least r away, so their
// weight is exactly 0, and nodes outside the grid are never flushed.
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
  float dx, inv_r2;
  float rho_l, rho_g;
  const float4* pos;
  const float4* vel;
  const int* cell_start;
  float* out[PG_NACC];  // mass x,y,z, mom x,y,z, cell_mass, cell_wsum
};

// Register box of grid G (0,1,2 = face axis, 3 = cell centres) for one cell.
template <int G> struct Box {
  static constexpr int NX = (G == 0) ? 2 : 3, NY = (G == 1) ? 2 : 3, NZ = (G == 2) ? 2 : 3;
  static constexpr int LX = (G == 0) ? 0 : -1, LY = (G == 1) ? 0 : -1, LZ = (G == 2) ? 0 : -1;
  static constexpr float OX = (G == 0) ? 0.f : 0.5f, OY = (G == 1) ? 0.f : 0.5f, OZ = (G == 2) ? 0.f : 0.5f;
  float m[NX][NY][NZ];   // sum of w * m_p
  float q[NX][NY][NZ];   // sum of w * m_p * u_G (faces) or of w (cells)

  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int a = 0; a < NX; ++a)
#pragma unroll
      for (int b = 0; b < NY; ++b)
#pragma unroll
        for (int c = 0; c < NZ; ++c) m[a][b][c] = q[a][b][c] = 0.f;
  }

  // add one particle (x, mass, velocity component) of cell (ci, cj, ck)
  __device__ __forceinline__ void add(int ci, int cj, int ck, const float x[3], float mp, float up, float dx,
                                      float inv_r2) {
    float DX[NX], DY[NY], DZ[NZ];
#pragma unroll
    for (int a = 0; a < NX; ++a) {
      const float f = ((float)(ci + LX + a) + OX) * dx - x[0];
      DX[a] = f * f;
    }
#pragma unroll
    for (int b = 0; b < NY; ++b) {
      const float f = ((float)(cj + LY + b) + OY) * dx - x[1];
      DY[b] = f * f;
    }
#pragma unroll
    for (int c = 0; c < NZ; ++c) {
      const float f = ((float)(ck + LZ + c) + OZ) * dx - x[2];
      DZ[c] = f * f;
    }
#pragma unroll
    for (int a = 0; a < NX; ++a)
#pragma unroll
      for (int b = 0; b < NY; ++b) {
        const float dxy = DX[a] + DY[b];
#pragma unroll
        for (int c = 0; c < NZ; ++c) {
          const float t = fmaxf(1.f - (dxy + DZ[c]) * inv_r2, 0.f);
          const float w = t * t * t;
          const float wm = w * mp;
          m[a][b][c] += wm;
          q[a][b][c] += (G < 3) ? wm * up : w;
        }
      }
  }

  // combine along k across the lanes of the row and add to the shared boxes.
  // Lane l owns cell k0 + l; box k index of node k is k - k0 - LZ.
  __device__ __forceinline__ void flush(float* sm1, float* sm2, int li, int lj, int lane) {
#pragma unroll
    for (int a = 0; a < NX; ++a)
#pragma unroll
      for (int b = 0; b < NY; ++b) {
        const int row = ((li + a) * PG_BJ + (lj + b)) * PG_BK;
        if (NZ == 3) {
          // node k0+l (box index l+1) = own centre + lane l-1's upper + lane l+1's lower
          const float up1 = __shfl_up_sync(0xffffffffu, m[a][b][2], 1);
          const float up2 = __shfl_up_sync(0xffffffffu, q[a][b][2], 1);
          const float dn1 = __shfl_down_sync(0xffffffffu, m[a][b][0], 1);
          const float dn2 = __shfl_down_sync(0xffffffffu, q[a][b][0], 1);
          float v1 = m[a][b][1], v2 = q[a][b][1];
          if (lane > 0) { v1 += up1; v2 += up2; }
          if (lane < 31) { v1 += dn1; v2 += dn2; }
          if (v1 != 0.f) atomicAdd(sm1 + row + lane + 1, v1);
          if (v2 != 0.f) atomicAdd(sm2 + row + lane + 1, v2);
          if (lane == 0) {
            if (m[a][b][0] != 0.f) atomicAdd(sm1 + row, m[a][b][0]);
            if (q[a][b][0] != 0.f) atomicAdd(sm2 + row, q[a][b][0]);
          }
          if (lane == 31) {
            if (m[a][b][2] != 0.f) atomicAdd(sm1 + row + 33, m[a][b][2]);
            if (q[a][b][2] != 0.f) atomicAdd(sm2 + row + 33, q[a][b][2]);
          }
        } else {
          // z-faces: node k0+l (box index l) = own lower + lane l-1's upper
          const float up1 = __shfl_up_sync(0xffffffffu, m[a][b][NZ - 1], 1);
          const float up2 = __shfl_up_sync(0xffffffffu, q[a][b][NZ - 1], 1);
          float v1 = m[a][b][0], v2 = q[a][b][0];
          if (lane > 0) { v1 += up1; v2 += up2; }
          if (v1 != 0.f) atomicAdd(sm1 + row + lane, v1);
          if (v2 != 0.f) atomicAdd(sm2 + row + lane, v2);
          if (lane == 31) {
            if (m[a][b][NZ - 1] != 0.f) atomicAdd(sm1 + row + 32, m[a][b][NZ - 1]);
            if (q[a][b][NZ - 1] != 0.f) atomicAdd(sm2 + row + 32, q[a][b][NZ - 1]);
          }
        }
      }
  }
};

// one grid over the particles of cell (i, j, k) (range [s, e)), then the row flush
template <int G>
__device__ __forceinline__ void p2g_grid(const P2GArgs& a, float* acc, int i, int j, int k, int s, int e, int li,
                                         int lj, int lane) {
  Box<G> box;
  box.zero();
  // one particle of prefetch: the loads of t+1 are in flight while t is splatted
  float4 Pn = make_float4(0.f, 0.f, 0.f, 0.f), Vn = Pn;
  if (s < e) {
    Pn = __ldg(a.pos + s);
    if (G < 3) Vn = __ldg(a.vel + s);
  }
  for (int t = s; t < e; ++t) {
    const float4 P = Pn, V = Vn;
    if (t + 1 < e) {
      Pn = __ldg(a.pos + t + 1);
      if (G < 3) Vn = __ldg(a.vel + t + 1);
    }
    const int flags = __float_as_int(P.w);
    if ((flags >> PF_PSTATE_SHIFT) & 3) continue;  // droplets / dead particles do not splat
    const float mp = (flags & PF_FLAG_LIQUID) ? a.rho_l : a.rho_g;
    const float up = G == 0 ? V.x : G == 1 ? V.y : V.z;
    const float x[3] = {P.x, P.y, P.z};
    box.add(i, j, k, x, mp, up, a.dx, a.inv_r2);
  }
  const int a1 = (G < 3) ? G : 6, a2 = (G < 3) ? 3 + G : 7;
  box.flush(acc + a1 * PG_BOX, acc + a2 * PG_BOX, li, lj, lane);
}

__global__ void __launch_bounds__(PG_NT) k_p2g(P2GArgs a) {
  extern __shared__ __align__(16) float acc[];  // [PG_NACC][PG_BOX]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int k0 = blockIdx.x * PG_TK, j0 = blockIdx.y * PG_TJ, i0 = blockIdx.z * PG_TI;
  for (int e = tid; e < PG_NACC * PG_BOX; e += PG_NT) acc[e] = 0.f;
  __syncthreads();

  const int nx = a.nx, ny = a.ny, nz = a.nz;
  for (int row = warp; row < PG_TI * PG_TJ; row += PG_NT / 32) {
    const int li = row / PG_TJ, lj = row % PG_TJ;
    const int i = i0 + li, j = j0 + lj, k = k0 + lane;
    if (i >= nx || j >= ny) continue;  // warp-uniform
    int s = 0, e = 0;
    if (k < nz) {
      const int key = (i * ny + j) * nz + k;
      s = a.cell_start[key];
      e = a.cell_start[key + 1];
    }
    p2g_grid<3>(a, acc, i, j, k, s, e, li, lj, lane);
    p2g_grid<0>(a, acc, i, j, k, s, e, li, lj, lane);
    p2g_grid<1>(a, acc, i, j, k, s, e, li, lj, lane);
    p2g_grid<2>(a, acc, i, j, k, s, e, li, lj, lane);
  }
  __syncthreads();
  // flush: each tile node once
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
  PF_REQUIRE(g->nx > 0 && g->ny > 0 && g->nz > 0 && g->dx > 0.f, "bad grid");
  // the register boxes cover nodes within one cell of the particle's cell: the
  // support radius must not exceed one cell (the reference uses r_p = dx)
  PF_REQUIRE(r_p > 0.f && r_p <= g->dx, "r_p must be in (0, dx]");
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
