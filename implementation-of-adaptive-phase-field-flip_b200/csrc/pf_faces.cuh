// Face-array index space shared by the grid and adjoint kernels: the three
// MAC face arrays (x-faces (nx+1, ny, nz), y-faces (nx, ny+1, nz), z-faces
// (nx, ny, nz+1)) and, optionally, the cell array, covered by one launch; the
// eq. (7) phase field and the wall/obstacle face tests.
#pragma once
#include "pf_common.cuh"

namespace pf {

// eq. (7), pfflip/kernels.py:234-241
__device__ __forceinline__ float phase_field(float rho, float rho_min, float alpha_phi, float rho_0l) {
  if (rho < rho_min) return 0.f;
  return fminf(sqrtf(fmaxf(rho - rho_min, 0.f) / (alpha_phi * rho_0l)), 1.f);
}

struct FaceSpace {  // the three face arrays and the cells as one index space
  int nx, ny, nz;
  long long nf[3], nc;
  __device__ __forceinline__ long long total() const { return nf[0] + nf[1] + nf[2] + nc; }
};

__host__ __device__ inline FaceSpace make_space(int nx, int ny, int nz) {
  FaceSpace s;
  s.nx = nx; s.ny = ny; s.nz = nz;
  s.nf[0] = (long long)(nx + 1) * ny * nz;
  s.nf[1] = (long long)nx * (ny + 1) * nz;
  s.nf[2] = (long long)nx * ny * (nz + 1);
  s.nc = (long long)nx * ny * nz;
  return s;
}

// One launch covers the three face arrays (and, with cells, the cell array):
// blockIdx.z runs over the i-planes of x-faces (nx+1), y-faces (nx), z-faces
// (nx) and cells (nx); blockIdx.y/x and the thread give j (8 rows) and k (32).
// Returns the array (0..2 faces, 3 cells) and the element's flat index, or -1
// outside the array.
__host__ inline dim3 grid_faces(int nx, int ny, int nz, bool with_cells) {
  return dim3((unsigned)((nz + 1 + C3_TK - 1) / C3_TK), (unsigned)((ny + 1 + C3_TJ - 1) / C3_TJ),
              (unsigned)(3 * nx + 1 + (with_cells ? nx : 0)));
}
// The same space with pz consecutive planes per block: blockIdx.z covers the
// planes pz*blockIdx.z .. +pz-1, so a thread can issue the loads of all its
// planes before it uses any of them.
__host__ inline dim3 grid_faces_multi(int nx, int ny, int nz, bool with_cells, int pz) {
  const int planes = 3 * nx + 1 + (with_cells ? nx : 0);
  return dim3((unsigned)((nz + 1 + C3_TK - 1) / C3_TK), (unsigned)((ny + 1 + C3_TJ - 1) / C3_TJ),
              (unsigned)((planes + pz - 1) / pz));
}
// element of plane z (of `planes` in all) for this thread, as locate
__device__ __forceinline__ int locate_plane(const FaceSpace& s, int z, int planes, long long* f, int* i, int* j,
                                            int* k) {
  if (z >= planes) return -1;
  int a;
  if (z < s.nx + 1) a = 0;
  else if ((z -= s.nx + 1) < s.nx) a = 1;
  else if ((z -= s.nx) < s.nx) a = 2;
  else { z -= s.nx; a = 3; }
  const int n1 = s.ny + (a == 1), n2 = s.nz + (a == 2);
  const int jj = (int)(blockIdx.y * C3_TJ + (threadIdx.x >> 5)), kk = (int)(blockIdx.x * C3_TK + (threadIdx.x & 31));
  if (jj >= n1 || kk >= n2) return -1;
  *i = z;
  *j = jj;
  *k = kk;
  *f = ((long long)z * n1 + jj) * n2 + kk;
  return a;
}

__device__ __forceinline__ int locate(const FaceSpace& s, long long* f, int* i, int* j, int* k) {
  int z = (int)blockIdx.z, a;
  if (z < s.nx + 1) a = 0;
  else if ((z -= s.nx + 1) < s.nx) a = 1;
  else if ((z -= s.nx) < s.nx) a = 2;
  else { z -= s.nx; a = 3; }
  const int n1 = s.ny + (a == 1), n2 = s.nz + (a == 2);
  const int jj = (int)(blockIdx.y * C3_TJ + (threadIdx.x >> 5)), kk = (int)(blockIdx.x * C3_TK + (threadIdx.x & 31));
  if (jj >= n1 || kk >= n2) return -1;
  *i = z;
  *j = jj;
  *k = kk;
  *f = ((long long)z * n1 + jj) * n2 + kk;
  return a;
}

__device__ __forceinline__ bool boundary_face(int a, int i, int j, int k, int nx, int ny, int nz) {
  const int n = a == 0 ? i : a == 1 ? j : k;
  const int last = a == 0 ? nx : a == 1 ? ny : nz;
  return n == 0 || n == last;
}

__device__ __forceinline__ bool solid_face(const int* solid, int a, int i, int j, int k, int nx, int ny, int nz) {
  if (!solid) return false;
  const int im = i - (a == 0), jm = j - (a == 1), km = k - (a == 2);
  bool b = false;
  if (i < nx && j < ny && k < nz) b = b || solid[((long long)i * ny + j) * nz + k] != 0;
  if (im >= 0 && jm >= 0 && km >= 0) b = b || solid[((long long)im * ny + jm) * nz + km] != 0;
  return b;
}

}  // namespace pf
