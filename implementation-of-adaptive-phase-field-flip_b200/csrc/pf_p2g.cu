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
// Weights: w = max(1 - d^2/r^2, 0)^3, evaluated in the cell's own scaled
// frame: per axis xl = x - i*dx (one rounding, the product exact inside the
// fma), X = xl/r, and for a node at (i + L + o)*dx the scaled offset
// f = (L + o)*(dx/r) - X; then s = (fx^2 - 1) + fy^2 + fz^2 = d^2/r^2 - 1 and
// w = -min(s, 0)^3, the sign folded into the particle's mass.  This is the
// reference's weight to rounding (its d^2 sums in world units; the scaled
// offsets here carry no more error than its fx = (n + o)*dx - x).  The
// register box includes nodes outside the reference's window
// floor(c - R) + 1 .. floor(c + R); those lie at least r away, so their
// weight is exactly 0, and nodes outside the grid are never flushed.  The
// weight arithmetic runs on packed f32x2 pairs.
#include "pf_common.cuh"
#include "pf_f32x2.cuh"

namespace pf {

constexpr int PG_TI = 2, PG_TJ = 8, PG_TK = 32;
constexpr int PG_NT = 256;
constexpr int PG_BI = PG_TI + 2, PG_BJ = PG_TJ + 2, PG_BK = PG_TK + 2;
constexpr int PG_BOX = PG_BI * PG_BJ * PG_BK;  // nodes per accumulator box
constexpr int PG_NACC = 8;
constexpr size_t PG_SMEM = sizeof(float) * PG_NACC * PG_BOX;

struct P2GArgs {
  int nx, ny, nz;
  float dx, inv_r, s_node;  // s_node = dx / r
  float rho_l, rho_g;
  const float4* pos;
  const float4* vel;
  const int* cell_start;
  float* out[PG_NACC];  // mass x,y,z, mom x,y,z, cell_mass, cell_wsum
};

// Register box of grid G (0,1,2 = face axis, 3 = cell centres) for one cell.
// The accumulators are packed pairs (f32x2) along one axis PA: the face
// grids pair their two nodes along the normal axis, the cell grid pairs z
// nodes 0 and 1 and keeps z node 2 in scalars.  Every node still sums its
// particles in particle order with the scalar operations
// d^2 = (dx^2 + dy^2) + dz^2, t = max(fma(-d^2, 1/r^2, 1), 0), w = (t t) t,
// wm = w m_p, m += wm, q += wm u (fma) or q += w.
template <int G> struct Box {
  static constexpr int NX = (G == 0) ? 2 : 3, NY = (G == 1) ? 2 : 3, NZ = (G == 2) ? 2 : 3;
  static constexpr int LX = (G == 0) ? 0 : -1, LY = (G == 1) ? 0 : -1, LZ = (G == 2) ? 0 : -1;
  static constexpr float OX = (G == 0) ? 0.f : 0.5f, OY = (G == 1) ? 0.f : 0.5f, OZ = (G == 2) ? 0.f : 0.5f;
  static constexpr int PA = G < 3 ? G : 2;  // paired axis
  static constexpr int QX = PA == 0 ? 1 : NX, QY = PA == 1 ? 1 : NY, QZ = PA == 2 ? 1 : NZ;
  static constexpr int SX = G == 3 ? 3 : 1;  // cell grid: scalar z node 2 per (a, b)
  f2 m2[QX][QY][QZ];  // sum of w * m_p
  f2 q2[QX][QY][QZ];  // sum of w * m_p * u_G (faces) or of w (cells)
  float m1[SX][SX], q1[SX][SX];

  __device__ __forceinline__ void zero() {
    const f2 z = f2_bcast(0.f);
#pragma unroll
    for (int a = 0; a < QX; ++a)
#pragma unroll
      for (int b = 0; b < QY; ++b)
#pragma unroll
        for (int c = 0; c < QZ; ++c) m2[a][b][c] = q2[a][b][c] = z;
#pragma unroll
    for (int a = 0; a < SX; ++a)
#pragma unroll
      for (int b = 0; b < SX; ++b) m1[a][b] = q1[a][b] = 0.f;
  }

  // the accumulated values of node (a, b, c)
  __device__ __forceinline__ float M(int a, int b, int c) const {
    if (G == 3 && c == 2) return m1[a][b];
    const f2 v = m2[PA == 0 ? 0 : a][PA == 1 ? 0 : b][PA == 2 ? 0 : c];
    return (PA == 0 ? a : PA == 1 ? b : c) == 0 ? f2_x(v) : f2_y(v);
  }
  __device__ __forceinline__ float Q(int a, int b, int c) const {
    if (G == 3 && c == 2) return q1[a][b];
    const f2 v = q2[PA == 0 ? 0 : a][PA == 1 ? 0 : b][PA == 2 ? 0 : c];
    return (PA == 0 ? a : PA == 1 ? b : c) == 0 ? f2_x(v) : f2_y(v);
  }

  // one node pair: s = d^2/r^2 - 1 per half; u = min(s, 0), w = -u^3; the
  // accumulators take m += w m_p and q += w m_p u_G (faces) or q += w (cells)
  // as fma(u^3, -m_p, m) and fma(u^3, -m_p u_G, q) / fma(u^3, -1, q)
  __device__ __forceinline__ static void node2(f2 s, f2 nmp2, f2 nq2, f2& m, f2& q) {
    float a, b;
    f2_split(s, a, b);
    const f2 u = f2_make(fminf(a, 0.f), fminf(b, 0.f));
    const f2 u3 = f2_mul(f2_mul(u, u), u);
    m = f2_fma(u3, nmp2, m);
    q = f2_fma(u3, nq2, q);
  }

  // scaled squared offsets along one axis to the nodes L + o (o = 0 .. N-1) of
  // the cell, minus one when M1: a pair (o = 0, 1) for the paired axis,
  // broadcast pairs per node otherwise.  X = (x - i dx)/r; off = node offset
  // within its cell (0 or 0.5); sn = dx/r.
  template <int N, int L, bool PAIRED, bool M1>
  __device__ __forceinline__ static void dist2(float off, float X, float sn, f2* out) {
    const f2 nx = f2_bcast(-X), one = f2_bcast(M1 ? -1.f : 0.f);
    if (PAIRED) {
      const f2 f = f2_fma(f2_make((float)L + off, (float)(L + 1) + off), f2_bcast(sn), nx);
      out[0] = f2_fma(f, f, one);
    } else {
#pragma unroll
      for (int o = 0; o < N; ++o) {
        const f2 f = f2_fma(f2_bcast((float)(L + o) + off), f2_bcast(sn), nx);
        out[o] = f2_fma(f, f, one);
      }
    }
  }

  // add one particle (scaled cell-local position X, mass, velocity component)
  __device__ __forceinline__ void add(const float X[3], float mp, float up, float sn) {
    const f2 nmp2 = f2_bcast(-mp), nq2 = f2_bcast(G < 3 ? -mp * up : -1.f);
    f2 DX[PA == 0 ? 1 : NX], DY[PA == 1 ? 1 : NY], DZ[PA == 2 ? 1 : NZ];
    dist2<NX, LX, PA == 0, true>(OX, X[0], sn, DX);
    dist2<NY, LY, PA == 1, false>(OY, X[1], sn, DY);
    dist2<NZ, LZ, PA == 2, false>(OZ, X[2], sn, DZ);
    float dz2 = 0.f;  // cell grid: z node 2
    if (G == 3) {
      const float f = fmaf((float)(LZ + 2) + OZ, sn, -X[2]);
      dz2 = f * f;
    }
    if (PA == 0) {
#pragma unroll
      for (int b = 0; b < NY; ++b) {
        const f2 dxy = f2_add(DX[0], DY[b]);
#pragma unroll
        for (int c = 0; c < NZ; ++c) node2(f2_add(dxy, DZ[c]), nmp2, nq2, m2[0][b][c], q2[0][b][c]);
      }
    } else if (PA == 1) {
#pragma unroll
      for (int a = 0; a < NX; ++a) {
        const f2 dxy = f2_add(DX[a], DY[0]);
#pragma unroll
        for (int c = 0; c < NZ; ++c) node2(f2_add(dxy, DZ[c]), nmp2, nq2, m2[a][0][c], q2[a][0][c]);
      }
    } else {
#pragma unroll
      for (int a = 0; a < NX; ++a)
#pragma unroll
        for (int b = 0; b < NY; ++b) {
          const f2 dxy = f2_add(DX[a], DY[b]);
          node2(f2_add(dxy, DZ[0]), nmp2, nq2, m2[a][b][0], q2[a][b][0]);
          if (G == 3) {
            const float u = fminf(f2_x(dxy) + dz2, 0.f);
            const float u3 = u * u * u;
            m1[a < SX ? a : 0][b < SX ? b : 0] = fmaf(u3, -mp, m1[a < SX ? a : 0][b < SX ? b : 0]);
            q1[a < SX ? a : 0][b < SX ? b : 0] -= u3;
          }
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
          const float up1 = __shfl_up_sync(0xffffffffu, M(a, b, 2), 1);
          const float up2 = __shfl_up_sync(0xffffffffu, Q(a, b, 2), 1);
          const float dn1 = __shfl_down_sync(0xffffffffu, M(a, b, 0), 1);
          const float dn2 = __shfl_down_sync(0xffffffffu, Q(a, b, 0), 1);
          float v1 = M(a, b, 1), v2 = Q(a, b, 1);
          if (lane > 0) { v1 += up1; v2 += up2; }
          if (lane < 31) { v1 += dn1; v2 += dn2; }
          if (v1 != 0.f) atomicAdd(sm1 + row + lane + 1, v1);
          if (v2 != 0.f) atomicAdd(sm2 + row + lane + 1, v2);
          if (lane == 0) {
            if (M(a, b, 0) != 0.f) atomicAdd(sm1 + row, M(a, b, 0));
            if (Q(a, b, 0) != 0.f) atomicAdd(sm2 + row, Q(a, b, 0));
          }
          if (lane == 31) {
            if (M(a, b, 2) != 0.f) atomicAdd(sm1 + row + 33, M(a, b, 2));
            if (Q(a, b, 2) != 0.f) atomicAdd(sm2 + row + 33, Q(a, b, 2));
          }
        } else {
          // z-faces: node k0+l (box index l) = own lower + lane l-1's upper
          const float up1 = __shfl_up_sync(0xffffffffu, M(a, b, NZ - 1), 1);
          const float up2 = __shfl_up_sync(0xffffffffu, Q(a, b, NZ - 1), 1);
          float v1 = M(a, b, 0), v2 = Q(a, b, 0);
          if (lane > 0) { v1 += up1; v2 += up2; }
          if (v1 != 0.f) atomicAdd(sm1 + row + lane, v1);
          if (v2 != 0.f) atomicAdd(sm2 + row + lane, v2);
          if (lane == 31) {
            if (M(a, b, NZ - 1) != 0.f) atomicAdd(sm1 + row + 32, M(a, b, NZ - 1));
            if (Q(a, b, NZ - 1) != 0.f) atomicAdd(sm2 + row + 32, Q(a, b, NZ - 1));
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
  const float ci = (float)i, cj = (float)j, ck = (float)k;
  // two particles of prefetch: the loads of t+2 are in flight while t is
  // splatted (a warp holds too few peers on its SM to hide an L2 round trip
  // behind one particle's arithmetic)
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 Pa = z4, Va = z4, Pb = z4, Vb = z4;
  if (s < e) {
    Pa = __ldg(a.pos + s);
    if (G < 3) Va = __ldg(a.vel + s);
  }
  if (s + 1 < e) {
    Pb = __ldg(a.pos + s + 1);
    if (G < 3) Vb = __ldg(a.vel + s + 1);
  }
  for (int t = s; t < e; ++t) {
    const float4 P = Pa, V = Va;
    Pa = Pb;
    Va = Vb;
    if (t + 2 < e) {
      Pb = __ldg(a.pos + t + 2);
      if (G < 3) Vb = __ldg(a.vel + t + 2);
    }
    const int flags = __float_as_int(P.w);
    if ((flags >> PF_PSTATE_SHIFT) & 3) continue;  // droplets / dead particles do not splat
    const float mp = (flags & PF_FLAG_LIQUID) ? a.rho_l : a.rho_g;
    const float up = G == 0 ? V.x : G == 1 ? V.y : V.z;
    const float X[3] = {fmaf(ci, -a.dx, P.x) * a.inv_r, fmaf(cj, -a.dx, P.y) * a.inv_r,
                        fmaf(ck, -a.dx, P.z) * a.inv_r};
    box.add(X, mp, up, a.s_node);
  }
  const int a1 = (G < 3) ? G : 6, a2 = (G < 3) ? 3 + G : 7;
  box.flush(acc + a1 * PG_BOX, acc + a2 * PG_BOX, li, lj, lane);
}

__global__ void __launch_bounds__(PG_NT, 2) k_p2g(const __grid_constant__ P2GArgs a) {
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
    // the smallest shared-memory carveout that holds two CTAs' accumulators,
    // so that the rest of the SM's unified memory serves as L1 for the passes'
    // re-reads (a hint: the driver rounds up to a carveout it supports)
    PF_CUDA_TRY(cudaFuncSetAttribute(k_p2g, cudaFuncAttributePreferredSharedMemoryCarveout, 40));
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
  a.inv_r = 1.f / r_p;
  a.s_node = g->dx / r_p;
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
