// Stable counting sort of particles by cell (no reference counterpart: the
// reference keeps particles in seeding order, pfflip/scenes.py:23-29).
//
//   1. keys + ranks: key = linear index of the cell floor(x/dx) (IEEE binary32
//      division, clamped); a warp-aggregated atomicAdd on the cell's count
//      returns each particle's arrival rank within its cell
//   2. exclusive scan of the counts -> cell_start (3-phase block scan)
//   3. scatter: perm[cell_start[key] + rank] = p (no atomics)
//   4. per-cell order fix: the ranks of one cell follow arrival order; one
//      warp per cell ranks the original indices so each cell's segment is
//      ascending, which is exactly a stable sort; sorted keys are written here
//   5. gather of the two float4 particle streams through perm, by the same
//      warp right after each cell's fix (one kernel for 4 and 5)
//
// Bytes per particle: 16 (pos) + 8 (key, rank) in pass 1, 8 + 4 in pass 3,
// 12 in pass 4, 4 + 32 + 32 in pass 5, plus 8 per cell for the scan.
#include <cuda.h>

#include <mutex>

#include "pf_common.cuh"

namespace pf {

// pass 1: key and arrival rank within the cell (ranks of one cell are
// 0..count-1 in some order), counts into `counts`.  Each warp walks one
// contiguous chunk of the stream: on a stream already near cell order the
// ranks of a cell then mostly arrive in index order, even where the cell
// spans two batches of 32, so the order fix has less to do.
__global__ void k_keys_rank(long long n, const float4* __restrict__ pos, float dx, int nx, int ny, int nz,
                            int2* __restrict__ key_rank, int* __restrict__ counts) {
  long long c0, c1;
  warp_chunk(n, c0, c1);
  for (long long base = c0; base < c1; base += 32) {  // warp-uniform bound: every lane takes the ballot
    const long long p = base + (threadIdx.x & 31);
    const bool in = p < c1;
    const unsigned active = __ballot_sync(0xffffffffu, in);
    if (!in) continue;
    const float4 q = __ldg(pos + p);
    const int key = cell_key(q.x, q.y, q.z, dx, nx, ny, nz);
    key_rank[p] = make_int2(key, agg_inc(counts, key, active));
  }
}

// ---------------------------------------------------------------- scan
constexpr int SCAN_NT = 1024, SCAN_PER = 4, SCAN_TILE = SCAN_NT * SCAN_PER;

__device__ __forceinline__ int block_excl_scan(int v, int* sh /*32*/, int* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    sh[lane] = s;
  }
  __syncthreads();
  const int before = (w > 0 ? sh[w - 1] : 0);
  *total = sh[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before + x - v;
}

// in place exclusive scan of a[0..n) per tile; tile totals to sums[]
__global__ void __launch_bounds__(SCAN_NT) k_scan_tiles(long long n, int* __restrict__ a, int* __restrict__ sums) {
  __shared__ int sh[32];
  const long long t0 = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_PER;
  int v[SCAN_PER], s = 0;
#pragma unroll
  for (int q = 0; q < SCAN_PER; ++q) {
    v[q] = (t0 + q < n) ? a[t0 + q] : 0;
    s += v[q];
  }
  int tot;
  int ex = block_excl_scan(s, sh, &tot);
#pragma unroll
  for (int q = 0; q < SCAN_PER; ++q) {
    if (t0 + q < n) a[t0 + q] = ex;
    ex += v[q];
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// exclusive scan of the tile sums by one CTA (any count)
__global__ void __launch_bounds__(SCAN_NT) k_scan_sums(int m, int* __restrict__ sums) {
  __shared__ int sh[32];
  int carry = 0;
  for (int base = 0; base < m; base += SCAN_NT) {
    const int i = base + threadIdx.x;
    const int v = (i < m) ? sums[i] : 0;
    int tot;
    const int ex = block_excl_scan(v, sh, &tot);
    if (i < m) sums[i] = carry + ex;
    carry += tot;
  }
}

__global__ void k_scan_add(long long n, int* __restrict__ a, const int* __restrict__ sums) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    a[e] += sums[e / SCAN_TILE];
}

// ---------------------------------------------------------------- scatter + order fix
// pass 3: perm[start[key] + rank] = p; the slots of one cell are then in
// arrival order, which k_fix_gather turns into index order
__global__ void k_scatter_rank(long long n, const int2* __restrict__ key_rank, const int* __restrict__ start,
                               int* __restrict__ perm) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int2 kr = key_rank[p];
    perm[start[kr.x] + kr.y] = (int)p;
  }
}

// one warp per cell: rank the segment's original indices (distinct) so the
// segment becomes ascending; also writes the sorted keys
// One warp per batch of 32 consecutive cells: lane i loads the bounds of cell
// c0 + i (one coalesced pair of loads for the batch), then the warp walks the
// batch, writing the sorted keys of each cell and ranking its segment, with the
// next cell's segment loaded while the current one is checked.
// number of the n ascending values of a below v
__device__ __forceinline__ int count_below(const int* a, int n, int v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// A long segment (more than 32 particles in one cell, in arrival order) made
// ascending by the warp: 32-element chunks are ranked in registers, then runs
// are merged pairwise (each element's output slot is its index in its own run
// plus its count in the other run; the values are distinct), ping-ponging with
// the segment's own keys_out slots, which receive the cell key only afterwards.
// O(len log^2 len / 32) steps per lane: bounded however many particles share
// the cell.  a and b are not restrict: lanes read what others wrote before the
// __syncwarp.
__device__ void sort_long_segment(int* a, int* b, int len, int lane) {
  for (int c0 = 0; c0 < len; c0 += 32) {
    const int m = min(32, len - c0);
    const int v = lane < m ? a[c0 + lane] : INT_MAX;
    int rank = 0;
    for (int q = 0; q < m; ++q) rank += (__shfl_sync(0xffffffffu, v, q) < v);
    __syncwarp();
    if (lane < m) a[c0 + rank] = v;
    __syncwarp();
  }
  int* src = a;
  int* dst = b;
  for (long long w2 = 32; w2 < len; w2 *= 2) {
    const int w = (int)w2;
    for (long long r = 0; r < len; r += 2 * w2) {
      const int r0 = (int)r;
      const int na = min(w, len - r0), nb = max(0, min(w, len - r0 - w));
      const int* A = src + r0;
      const int* B = A + na;
      for (int t = lane; t < na + nb; t += 32) {
        const bool in_a = t < na;
        const int v = in_a ? A[t] : B[t - na];
        const int pos = in_a ? t + count_below(B, nb, v) : (t - na) + count_below(A, na, v);
        dst[r0 + pos] = v;
      }
    }
    __syncwarp();
    int* tmp = src;
    src = dst;
    dst = tmp;
  }
  if (src != a)
    for (int t = lane; t < len; t += 32) a[t] = src[t];
  __syncwarp();
}

// Passes 4 and 5 in one.  A cell's segment of perm holds its particles in
// arrival order; the warp puts it in index order (which is exactly the stable
// sort), writes the cell's sorted keys, and copies the segment's particles --
// both float4 streams -- to their sorted slots, so perm is read once and the
// writes of a segment are contiguous.  Segments of up to 32 particles are
// ranked in registers (most arrive in order already); longer ones take the
// warp merge sort above.
__device__ __forceinline__ void fix_gather_segment(int s, int len, int v, int c, int lane, int* __restrict__ perm,
                                                   int* __restrict__ keys_out, const float4* __restrict__ pin,
                                                   const float4* __restrict__ vin, float4* __restrict__ pout,
                                                   float4* __restrict__ vout) {
  if (len > 32) {
    sort_long_segment(perm + s, keys_out + s, len, lane);
    for (int t = lane; t < len; t += 32) {
      keys_out[s + t] = c;
      const int p = perm[s + t];
      pout[s + t] = __ldg(pin + p);
      vout[s + t] = __ldg(vin + p);
    }
    return;
  }
  if (len == 0) return;
  // already ascending?  (the common case: arrivals were in order)
  const int nxt = __shfl_down_sync(0xffffffffu, v, 1);
  const bool ok = (lane >= len - 1) || (v < nxt);
  int slot = lane;
  if (!__all_sync(0xffffffffu, ok)) {
    int rank = 0;
    for (int q = 0; q < len; ++q) rank += (__shfl_sync(0xffffffffu, v, q) < v);
    slot = rank;
    if (lane < len) perm[s + rank] = v;
  }
  if (lane < len) {
    keys_out[s + lane] = c;
    pout[s + slot] = __ldg(pin + v);
    vout[s + slot] = __ldg(vin + v);
  }
}

// One warp per batch of 32 consecutive cells: lane i loads the bounds of cell
// c0 + i (one coalesced pair of loads for the batch), then the warp walks the
// batch, the next cell's segment loaded while the current one is ordered and
// copied.
__global__ void k_fix_gather(int ncells, const int* __restrict__ start, int* __restrict__ perm,
                             int* __restrict__ keys_out, const float4* __restrict__ pin,
                             const float4* __restrict__ vin, float4* __restrict__ pout, float4* __restrict__ vout) {
  const int lane = threadIdx.x & 31;
  const int nbatch = (ncells + 31) >> 5;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int bt = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; bt < nbatch; bt += warps) {
    const int c0 = bt << 5, nb = min(32, ncells - c0);
    const int my_s = lane < nb ? start[c0 + lane] : 0;
    const int my_e = lane < nb ? start[c0 + lane + 1] : 0;
    int s = __shfl_sync(0xffffffffu, my_s, 0), len = __shfl_sync(0xffffffffu, my_e, 0) - s;
    int v = (lane < len && len <= 32) ? perm[s + lane] : INT_MAX;
    for (int q = 0; q < nb; ++q) {
      int s2 = 0, len2 = 0, v2 = INT_MAX;
      if (q + 1 < nb) {  // the next cell's segment, in flight while this one is handled
        s2 = __shfl_sync(0xffffffffu, my_s, q + 1);
        len2 = __shfl_sync(0xffffffffu, my_e, q + 1) - s2;
        v2 = (lane < len2 && len2 <= 32) ? perm[s2 + lane] : INT_MAX;
      }
      fix_gather_segment(s, len, v, c0 + q, lane, perm, keys_out, pin, vin, pout, vout);
      s = s2;
      len = len2;
      v = v2;
    }
  }
}

}  // namespace pf

using namespace pf;

extern "C" {

size_t pf_sort_workspace_bytes(const pf_grid* g, int64_t n) {
  if (!g) return 0;
  const long long nc = (long long)g->nx * g->ny * g->nz;
  const long long tiles = (nc + 1 + SCAN_TILE - 1) / SCAN_TILE;
  return (size_t)(8 * n + 4 * (tiles + 1) + 256);
}

}  // extern "C"

namespace {
// passes 2-5, after (key, rank) per particle and the counts in cell_start
int sort_from_keys(const pf_grid* g, int64_t n, const int2* key_rank, int* sums, const float* pos4_in,
                   const float* vel4_in, float* pos4_out, float* vel4_out, int32_t* keys_out, int32_t* perm_out,
                   int32_t* cell_start, cudaStream_t s) {
  const long long nc = (long long)g->nx * g->ny * g->nz;
  const long long tiles = (nc + 1 + SCAN_TILE - 1) / SCAN_TILE;
  k_scan_tiles<<<(int)tiles, SCAN_NT, 0, s>>>(nc + 1, cell_start, sums);
  PF_LAUNCHED();
  k_scan_sums<<<1, SCAN_NT, 0, s>>>((int)tiles, sums);
  PF_LAUNCHED();
  k_scan_add<<<grid_for(nc + 1, 256, kNumSMs * 16), 256, 0, s>>>(nc + 1, cell_start, sums);
  PF_LAUNCHED();
  if (n == 0) return PF_OK;
  k_scatter_rank<<<grid_for(n, 256, kNumSMs * 16), 256, 0, s>>>(n, key_rank, cell_start, perm_out);
  PF_LAUNCHED();
  k_fix_gather<<<grid_for(nc, 256, 1 << 20), 256, 0, s>>>(
      (int)nc, cell_start, perm_out, keys_out, reinterpret_cast<const float4*>(pos4_in),
      reinterpret_cast<const float4*>(vel4_in), reinterpret_cast<float4*>(pos4_out),
      reinterpret_cast<float4*>(vel4_out));
  PF_LAUNCHED();
  return PF_OK;
}

// pass 1: clear the counts, then (key, rank) per particle
int keys_and_ranks(const pf_grid* g, int64_t n, const float* pos4_in, int2* key_rank, int32_t* cell_start,
                   cudaStream_t s) {
  const long long nc = (long long)g->nx * g->ny * g->nz;
  PF_CUDA_TRY(cudaMemsetAsync(cell_start, 0, sizeof(int) * (nc + 1), s));
  if (n > 0) {
    k_keys_rank<<<grid_for(n, 256, kNumSMs * 16), 256, 0, s>>>(n, reinterpret_cast<const float4*>(pos4_in), g->dx,
                                                               g->nx, g->ny, g->nz, key_rank, cell_start);
    PF_LAUNCHED();
  }
  return PF_OK;
}

// true when the byte ranges [a, a + na) and [b, b + nb) share a byte
bool ranges_overlap(const void* a, long long na, const void* b, long long nb) {
  if (na <= 0 || nb <= 0) return false;
  const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return x < y + (uintptr_t)nb && y < x + (uintptr_t)na;
}

// the argument checks every entry point shares
int check_sort_args(const pf_grid* g, int64_t n, const float* pos4_in, const float* vel4_in, const float* pos4_out,
                    const float* vel4_out, const int32_t* keys_out, const int32_t* perm_out,
                    const int32_t* cell_start) {
  PF_REQUIRE(g && n >= 0 && pos4_in && vel4_in && pos4_out && vel4_out && keys_out && perm_out && cell_start,
             "null argument");
  PF_REQUIRE(g->nx > 0 && g->ny > 0 && g->nz > 0 && g->dx > 0.f, "bad grid");
  PF_REQUIRE((long long)g->nx * g->ny * g->nz < (1LL << 31) && n < (1LL << 31), "too large for int32 indices");
  PF_REQUIRE(aligned16(pos4_in) && aligned16(vel4_in) && aligned16(pos4_out) && aligned16(vel4_out),
             "particle streams must be 16-byte aligned");
  PF_REQUIRE(pos4_in != pos4_out && vel4_in != vel4_out, "sort output must not alias its input");
  // every output must be disjoint from every other buffer of the call (the
  // static variant also keeps its scratch in pos4_out for the whole call)
  const long long nc = (long long)g->nx * g->ny * g->nz;
  const struct {
    const void* p;
    long long bytes;
    const char* name;
    bool out;
  } buf[7] = {{pos4_in, 16 * n, "pos4_in", false},   {vel4_in, 16 * n, "vel4_in", false},
              {pos4_out, 16 * n, "pos4_out", true},  {vel4_out, 16 * n, "vel4_out", true},
              {keys_out, 4 * n, "keys_out", true},   {perm_out, 4 * n, "perm_out", true},
              {cell_start, 4 * (nc + 1), "cell_start", true}};
  for (int a = 0; a < 7; ++a)
    for (int b = a + 1; b < 7; ++b) {
      if (!buf[a].out && !buf[b].out) continue;  // two inputs may share memory
      PF_REQUIRE(!ranges_overlap(buf[a].p, buf[a].bytes, buf[b].p, buf[b].bytes), "%s overlaps %s", buf[a].name,
                 buf[b].name);
    }
  return PF_OK;
}
}  // namespace

extern "C" {

// workspace layout: (key, rank) per particle (8n bytes), then the scan's
// per-tile sums
int pf_sort_particles(const pf_grid* g, int64_t n, const float* pos4_in, const float* vel4_in, float* pos4_out,
                      float* vel4_out, int32_t* keys_out, int32_t* perm_out, int32_t* cell_start, void* workspace,
                      size_t workspace_bytes, void* stream) {
  int rc = check_sort_args(g, n, pos4_in, vel4_in, pos4_out, vel4_out, keys_out, perm_out, cell_start);
  if (rc != PF_OK) return rc;
  PF_REQUIRE(workspace && workspace_bytes >= pf_sort_workspace_bytes(g, n) && aligned16(workspace),
             "workspace too small or not 16-byte aligned");
  {
    const long long nc = (long long)g->nx * g->ny * g->nz, wb = (long long)workspace_bytes;
    PF_REQUIRE(!ranges_overlap(workspace, wb, pos4_in, 16 * n) && !ranges_overlap(workspace, wb, vel4_in, 16 * n) &&
                   !ranges_overlap(workspace, wb, pos4_out, 16 * n) &&
                   !ranges_overlap(workspace, wb, vel4_out, 16 * n) &&
                   !ranges_overlap(workspace, wb, keys_out, 4 * n) && !ranges_overlap(workspace, wb, perm_out, 4 * n) &&
                   !ranges_overlap(workspace, wb, cell_start, 4 * (nc + 1)),
               "workspace overlaps a particle stream or an output");
  }
  cudaStream_t s = S(stream);
  int2* key_rank = reinterpret_cast<int2*>(workspace);
  rc = keys_and_ranks(g, n, pos4_in, key_rank, cell_start, s);
  if (rc != PF_OK) return rc;
  return sort_from_keys(g, n, key_rank, reinterpret_cast<int*>(key_rank + n), pos4_in, vel4_in, pos4_out, vel4_out,
                        keys_out, perm_out, cell_start, s);
}

}  // extern "C"

// ---------------------------------------------------------------- sort without a workspace
// pf_sort_particles_static: the same stable sort for hosts that cannot hand
// the library a device workspace.  Some hosts fix all device memory when they
// start (one pool, sized once, with no allocator reachable from the step) or
// embed the step in code that must not allocate at all; such callers own the
// particle streams and the outputs, and nothing else.
//
// Scratch: the keys and arrival ranks of pass 1 sit in pos4_out (8 of its 16
// bytes per particle) until the gather overwrites it; the slot of a particle
// is cell_start[key] + rank, so no per-cell cursor copy is needed.  The only
// scratch left is the scan's per-tile sums, held in a file-scope device array
// sized for grids of up to kStaticMaxCells cells.  Nothing in that array has
// to start at zero: k_scan_tiles writes every entry the later passes read.
// The counts accumulate in cell_start, which each call clears on its stream.
// All calls on one device share the array, so calls whose executions overlap
// (two streams, two host threads) race on it.
namespace pf {

constexpr long long kStaticMaxCells = PF_SORT_STATIC_MAX_CELLS;
constexpr int kStaticTiles = (int)((kStaticMaxCells + 1 + SCAN_TILE - 1) / SCAN_TILE);
constexpr int kMaxDevices = 64;

static __device__ __align__(256) int g_static_tile_sums[(kStaticTiles + 63) / 64 * 64];

// Device address of g_static_tile_sums, looked up once per device and
// context.  The address belongs to the context the module was loaded into:
// after cudaDeviceReset (or with another context current on the same device)
// the cached pointer would be stale, so the cache is keyed on the context's
// process-unique id (cuCtxGetId, reached through the runtime's driver entry
// point, so the library does not link the driver) and looked up again when
// the current context changes.
struct StaticSums {
  unsigned long long ctx_id;  // 0: not looked up yet
  int* addr;
};
static StaticSums g_static_sums[kMaxDevices];
static std::mutex g_static_sums_mutex;

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// id of the context current on this thread, 0 when none is current yet
static int current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = cudaDriverEntryPointSymbolNotFound;
    PF_CUDA_TRY(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1));
    PF_CUDA_TRY(cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2));
    if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
      set_error(PF_ERR_CUDA, "driver entry points cuCtxGetCurrent/cuCtxGetId unavailable");
      return PF_ERR_CUDA;
    }
    get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
    get_id = reinterpret_cast<CtxGetIdFn>(f2);
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS) {
    set_error(PF_ERR_CUDA, "cuCtxGetCurrent failed");
    return PF_ERR_CUDA;
  }
  *id = 0;
  if (ctx && get_id(ctx, id) != CUDA_SUCCESS) {
    set_error(PF_ERR_CUDA, "cuCtxGetId failed");
    return PF_ERR_CUDA;
  }
  return PF_OK;
}

static int static_tile_sums(int** out) {
  int dev = 0;
  PF_CUDA_TRY(cudaGetDevice(&dev));
  PF_REQUIRE(dev >= 0 && dev < kMaxDevices, "device ordinal %d beyond %d", dev, kMaxDevices);
  std::lock_guard<std::mutex> lock(g_static_sums_mutex);
  unsigned long long id = 0;
  int rc = current_context_id(&id);
  if (rc != PF_OK) return rc;
  StaticSums& c = g_static_sums[dev];
  if (id == 0 || c.ctx_id != id) {
    // set-up for this device and context: the symbol lookup also creates the
    // device's primary context when none is current yet
    void* sym = nullptr;
    PF_CUDA_TRY(cudaGetSymbolAddress(&sym, g_static_tile_sums));
    rc = current_context_id(&id);
    if (rc != PF_OK) return rc;
    c.addr = static_cast<int*>(sym);
    c.ctx_id = id;
  }
  *out = c.addr;
  return PF_OK;
}

}  // namespace pf

extern "C" int pf_sort_particles_static(const pf_grid* g, int64_t n, const float* pos4_in, const float* vel4_in,
                                        float* pos4_out, float* vel4_out, int32_t* keys_out, int32_t* perm_out,
                                        int32_t* cell_start, void* stream) {
  int rc = check_sort_args(g, n, pos4_in, vel4_in, pos4_out, vel4_out, keys_out, perm_out, cell_start);
  if (rc != PF_OK) return rc;
  const long long nc = (long long)g->nx * g->ny * g->nz;
  PF_REQUIRE(nc <= kStaticMaxCells,
             "grid of %lld cells exceeds the %lld cells (512^3) the static scratch covers; use pf_sort_particles "
             "with a workspace",
             nc, kStaticMaxCells);
  int* sums = nullptr;
  rc = static_tile_sums(&sums);
  if (rc != PF_OK) return rc;
  cudaStream_t s = S(stream);
  int2* key_rank = reinterpret_cast<int2*>(pos4_out);
  rc = keys_and_ranks(g, n, pos4_in, key_rank, cell_start, s);
  if (rc != PF_OK) return rc;
  return sort_from_keys(g, n, key_rank, sums, pos4_in, vel4_in, pos4_out, vel4_out, keys_out, perm_out, cell_start,
                        s);
}
