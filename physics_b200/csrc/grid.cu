// Spatial hash of the SPH step on the device: integer cell keys, a counting
// sort by cell, a stable within-cell order by insertion index, and the gather
// that moves every per-particle array into the new order.
//
// Reference behaviour reproduced (crates/phy-fluid/src/sph/grid.rs):
//   * key_of: floor(x * (1/cell)) per axis, f64 -> i64, None -> 0 (25-33);
//   * build: a cell's particles in ascending insertion index (35-40).
// The sort is deterministic even though the histogram uses atomics: ranks
// inside a cell are recomputed from the insertion indices, so the final order
// is the total order (cell, insertion index) whatever the atomic order was.
//
// All kernels here are integer/byte work bound by HBM bandwidth; launches use
// 256-thread blocks and grid-stride loops sized to a multiple of the SM count.
#include <cuda_runtime.h>

#include <algorithm>

#include "sph_buffers.h"

namespace phy {

namespace {

constexpr int kThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kThreads * kScanItems;  // 4096 cells per scan block

int grid_for(int n, int threads = kThreads) {
  int b = (n + threads - 1) / threads;
  return b < 1 ? 1 : b;
}

// Spreads the low 10 bits of v three bits apart (Morton interleave).
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// Position inside its cell quantised to 1024 steps per axis (non-finite or
// out-of-range values clamp).
__device__ __forceinline__ uint32_t quantise_local(double x, long long k, double h0, double inv) {
  const double t = (x - (double)k * h0) * inv * 1024.0;
  if (!(t > 0.0)) return 0u;
  return t >= 1023.0 ? 1023u : (uint32_t)t;
}

// Cell of every particle plus its arrival rank inside its bucket: the cell
// (bucket_shift 0), or the tile of 2^bucket_shift consecutive cells (the
// overflow cell's bucket follows the last tile's).  Lanes of a warp that
// share a bucket (the common case: the previous order is already sorted by
// cell) are aggregated into one atomic.
__global__ void __launch_bounds__(kThreads) k_cell_hist(StepConsts c, int bucket_shift,
                                                        const double* __restrict__ px,
                                                        const double* __restrict__ py,
                                                        const double* __restrict__ pz,
                                                        uint32_t* __restrict__ cell_of,
                                                        uint32_t* __restrict__ rank,
                                                        uint32_t* __restrict__ count,
                                                        uint32_t* __restrict__ flags,
                                                        const uint16_t* __restrict__ scene,
                                                        const uint32_t* __restrict__ id,
                                                        unsigned long long* __restrict__ okey) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool active = i < c.n;
  uint32_t cell = 0;
  if (active) {
    long long kx = key_axis(px[i], c.inv_cell);
    long long ky = key_axis(py[i], c.inv_cell);
    long long kz = key_axis(pz[i], c.inv_cell);
    bool inside;
    if (c.tile) {
      // Tiled linearisation: the particle's scene box.
      const SceneBox& bx = c.boxes[scene ? scene[i] : 0];
      const long long a = kx - bx.b0[0], b = ky - bx.b0[1], d = kz - bx.b0[2];
      inside = a >= 1 && b >= 1 && d >= 1 && a < bx.nc[0] - 1 && b < bx.nc[1] - 1 && d < bx.nc[2] - 1;
      if (inside) cell = (uint32_t)box_tiled_index(c, bx, (int)a, (int)b, (int)d);
    } else {
      inside = cell_interior(c, kx, ky, kz);
      if (inside) cell = (uint32_t)cell_linear(c, kx, ky, kz);
    }
    if (!inside) {
      cell = (uint32_t)c.ncells;  // overflow cell: never visited as a neighbour
      atomicOr(flags, kFlagOutOfBox);
    }
    cell_of[i] = cell;
    if (okey) {
      // Tiled form: particles of a cell in Morton order of their position in
      // the cell, so that a warp's queries are spatial neighbours (the
      // insertion index breaks ties, keeping the order deterministic).
      const uint32_t m = (spread3(quantise_local(px[i], kx, c.h0, c.inv_cell)) << 2) |
                         (spread3(quantise_local(py[i], ky, c.h0, c.inv_cell)) << 1) |
                         spread3(quantise_local(pz[i], kz, c.h0, c.inv_cell));
      okey[i] = ((unsigned long long)m << 32) | id[i];
    }
  }
  unsigned mask = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  const uint32_t bucket = cell >> bucket_shift;
  unsigned peers = __match_any_sync(mask, bucket);
  int lane = threadIdx.x & 31;
  int leader = __ffs(peers) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(&count[bucket], (uint32_t)__popc(peers));
  base = __shfl_sync(peers, base, leader);
  rank[i] = base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
}

// Sum of each 4096-cell tile.
__global__ void __launch_bounds__(kThreads) k_scan_reduce(const uint32_t* __restrict__ v,
                                                          uint32_t* __restrict__ block_sums) {
  const uint4* t = reinterpret_cast<const uint4*>(v + (size_t)blockIdx.x * kScanTile) + threadIdx.x * 4;
  uint32_t s = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint4 a = t[q];
    s += a.x + a.y + a.z + a.w;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ uint32_t ws[kThreads / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t tot = 0;
    for (int w = 0; w < kThreads / 32; ++w) tot += ws[w];
    block_sums[blockIdx.x] = tot;
  }
}

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t& total) {
  __shared__ uint32_t ws[32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  int nw = blockDim.x >> 5;
  if (warp == 0) {
    uint32_t w = lane < nw ? ws[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) ws[lane] = w;
  }
  __syncthreads();
  uint32_t warp_off = warp > 0 ? ws[warp - 1] : 0;
  total = ws[nw - 1];
  __syncthreads();
  return warp_off + x - v;
}

// Exclusive scan of the tile sums, one block of 1024 threads, in chunks.
__global__ void __launch_bounds__(1024) k_scan_top(uint32_t* __restrict__ block_sums, int nb) {
  uint32_t carry = 0;
  for (int base = 0; base < nb; base += blockDim.x) {
    int k = base + threadIdx.x;
    uint32_t v = k < nb ? block_sums[k] : 0;
    uint32_t total;
    uint32_t ex = block_exclusive_scan(v, total);
    if (k < nb) block_sums[k] = carry + ex;
    carry += total;
  }
}

// In-place exclusive scan of each tile plus its tile offset.
__global__ void __launch_bounds__(kThreads) k_scan_apply(uint32_t* __restrict__ v,
                                                         const uint32_t* __restrict__ block_sums) {
  uint4* t = reinterpret_cast<uint4*>(v + (size_t)blockIdx.x * kScanTile) + threadIdx.x * 4;
  uint32_t a[kScanItems];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint4 u = t[q];
    a[4 * q] = u.x;
    a[4 * q + 1] = u.y;
    a[4 * q + 2] = u.z;
    a[4 * q + 3] = u.w;
  }
  uint32_t s = 0;
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    uint32_t x = a[q];
    a[q] = s;
    s += x;
  }
  uint32_t total;
  uint32_t off = block_exclusive_scan(s, total) + block_sums[blockIdx.x];
#pragma unroll
  for (int q = 0; q < 4; ++q)
    t[q] = make_uint4(a[4 * q] + off, a[4 * q + 1] + off, a[4 * q + 2] + off, a[4 * q + 3] + off);
}

// Every particle to its bucket's range (start = the scanned bucket counts),
// in arrival order inside the bucket.
__global__ void __launch_bounds__(kThreads) k_scatter(int n, int bucket_shift, const uint32_t* __restrict__ cell_of,
                                                      const uint32_t* __restrict__ rank,
                                                      const uint32_t* __restrict__ start,
                                                      uint32_t* __restrict__ tmp) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  tmp[start[cell_of[i] >> bucket_shift] + rank[i]] = (uint32_t)i;
}

// Cells up to kOrderSmall particles are ordered by k_order (each particle
// counts the smaller keys of its cell); cells up to kOrderLarge by a bitonic
// sort in shared memory (k_order_large); larger cells fall back to counting.
constexpr uint32_t kOrderSmall = 64;
constexpr uint32_t kOrderLarge = 4096;
constexpr int kOrderThreads = 512;

// Final slot of every particle: its rank by insertion index (or by in-cell
// order key) among the particles of its cell.  The overflow cell keeps
// arrival order (its particles never interact).  Cells of kOrderSmall <
// count <= kOrderLarge particles are left to k_order_large: the thread of
// their first slot appends them to `large` (a list in any order; each cell's
// result does not depend on it).
__global__ void __launch_bounds__(kThreads) k_order(int n, int ncells, const uint32_t* __restrict__ cell_of,
                                                    const uint32_t* __restrict__ cell_start,
                                                    const uint32_t* __restrict__ tmp,
                                                    const uint32_t* __restrict__ id,
                                                    const unsigned long long* __restrict__ okey,
                                                    uint32_t* __restrict__ perm,
                                                    uint32_t* __restrict__ large,
                                                    uint32_t* __restrict__ large_count) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t i = tmp[s];
  uint32_t cell = cell_of[i];
  if ((int)cell == ncells) {
    perm[s] = i;
    return;
  }
  uint32_t cs = cell_start[cell], ce = cell_start[cell + 1];
  if (ce - cs > kOrderSmall && ce - cs <= kOrderLarge) {
    if ((uint32_t)s == cs) large[atomicAdd(large_count, 1u)] = cell;
    return;
  }
  uint32_t r = 0;
  if (okey) {
    const unsigned long long mine = okey[i];
    for (uint32_t k = cs; k < ce; ++k) r += okey[tmp[k]] < mine ? 1u : 0u;
  } else {
    const uint32_t mine = id[i];
    for (uint32_t k = cs; k < ce; ++k) r += id[tmp[k]] < mine ? 1u : 0u;
  }
  perm[cs + r] = i;
}

// Order key of particle i: the in-cell order key (tiled form) or the
// insertion index.
__device__ __forceinline__ unsigned long long order_key(const unsigned long long* okey, const uint32_t* id,
                                                        uint32_t i) {
  return okey ? okey[i] : (unsigned long long)id[i];
}

// The cells k_order left: one CTA per cell (persistent grid over the
// device-side list) stages the cell's (key, particle) pairs in shared memory
// (keys are unique: they end in the insertion index).  A cell of at most
// kRankCount particles ranks each pair by counting the smaller keys (no
// barrier between steps); a larger one is sorted with a bitonic network
// padded to a power of two.  Either way each particle goes to its final slot.
constexpr uint32_t kRankCount = 256;
__global__ void __launch_bounds__(kOrderThreads) k_order_large(const uint32_t* __restrict__ cell_start,
                                                              const uint32_t* __restrict__ tmp,
                                                              const uint32_t* __restrict__ id,
                                                              const unsigned long long* __restrict__ okey,
                                                              const uint32_t* __restrict__ large,
                                                              const uint32_t* __restrict__ large_count,
                                                              uint32_t* __restrict__ perm) {
  __shared__ unsigned long long s_key[kOrderLarge];
  __shared__ uint32_t s_val[kOrderLarge];
  const uint32_t nl = *large_count;
  for (uint32_t w = blockIdx.x; w < nl; w += gridDim.x) {
    const uint32_t cell = large[w];
    const uint32_t cs = cell_start[cell], cnt = cell_start[cell + 1] - cs;
    uint32_t m = 1;
    while (m < cnt) m <<= 1;
    __syncthreads();  // the previous cell's pairs are written out
    for (uint32_t k = threadIdx.x; k < m; k += kOrderThreads) {
      if (k < cnt) {
        const uint32_t i = tmp[cs + k];
        s_key[k] = order_key(okey, id, i);
        s_val[k] = i;
      } else {
        s_key[k] = ~0ull;  // padding sorts last
        s_val[k] = 0;
      }
    }
    __syncthreads();
    if (cnt <= kRankCount) {
      for (uint32_t k = threadIdx.x; k < cnt; k += kOrderThreads) {
        const unsigned long long mine = s_key[k];
        uint32_t r = 0;
        for (uint32_t q = 0; q < cnt; ++q) r += s_key[q] < mine ? 1u : 0u;
        perm[cs + r] = s_val[k];
      }
      continue;  // uniform; the next cell's staging waits at the loop's first barrier
    }
    for (uint32_t size = 2; size <= m; size <<= 1) {
      for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
        for (uint32_t k = threadIdx.x; k < m / 2; k += kOrderThreads) {
          // Element pair (lo, lo + stride) of compare step k.
          const uint32_t lo = 2 * k - (k & (stride - 1));
          const uint32_t hi = lo + stride;
          const bool up = (lo & size) == 0;
          const unsigned long long a = s_key[lo], b = s_key[hi];
          if ((a > b) == up) {
            s_key[lo] = b;
            s_key[hi] = a;
            const uint32_t t = s_val[lo];
            s_val[lo] = s_val[hi];
            s_val[hi] = t;
          }
        }
        __syncthreads();
      }
    }
    for (uint32_t k = threadIdx.x; k < cnt; k += kOrderThreads) perm[cs + k] = s_val[k];
  }
}

// ---- Tiled sort: counts per tile, cells per occupied tile ------------------
//
// The tiled linearisation numbers a tile's cells consecutively, so the sort
// counts particles per tile (a histogram a 64th of the cell box, or an 8th
// with 2x2x2 tiles), scans the tile counts and the occupied-tile flags, and
// orders each occupied tile's particles in one CTA with shared counters.
// Only occupied tiles get cell starts: a reader of a cell in an empty tile
// finds the tile empty in the scanned tile counts (its start equals the next
// tile's start).

// Per scan tile of the tile counts (kScanTile entries, kScanItems per
// thread): the sum of the counts and the number of occupied tiles (index
// below ntiles, count above zero).
__global__ void __launch_bounds__(kThreads) k_tile_reduce(uint32_t ntiles, const uint32_t* __restrict__ cnt,
                                                          uint2* __restrict__ sums) {
  const uint32_t e0 = blockIdx.x * (uint32_t)kScanTile + threadIdx.x * (uint32_t)kScanItems;
  const uint4* t = reinterpret_cast<const uint4*>(cnt + e0);
  uint32_t s = 0, o = 0;
#pragma unroll
  for (int q = 0; q < kScanItems / 4; ++q) {
    const uint4 a = t[q];
    const uint32_t e = e0 + 4u * (uint32_t)q;
    s += a.x + a.y + a.z + a.w;
    o += (a.x != 0u && e < ntiles) + (a.y != 0u && e + 1 < ntiles) + (a.z != 0u && e + 2 < ntiles) +
         (a.w != 0u && e + 3 < ntiles);
  }
  for (int d = 16; d > 0; d >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, d);
    o += __shfl_xor_sync(0xffffffffu, o, d);
  }
  __shared__ uint2 ws[kThreads / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = make_uint2(s, o);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint2 tot = make_uint2(0u, 0u);
    for (int w = 0; w < kThreads / 32; ++w) {
      tot.x += ws[w].x;
      tot.y += ws[w].y;
    }
    sums[blockIdx.x] = tot;
  }
}

// Exclusive scans of the tile counts (in place: the tile starts) and of the
// occupied flags, which place every occupied tile in the tile list (tile_of,
// ascending tile index); each block first adds up the sums of the scan tiles
// before its own.  The thread holding entry ntiles (the overflow bucket)
// writes the overflow cell's range, the number of occupied tiles and the end
// of the last tile.
__global__ void __launch_bounds__(kThreads) k_tile_scan(int n, int ncells, uint32_t ntiles, uint32_t* __restrict__ cnt,
                                                        const uint2* __restrict__ sums,
                                                        uint32_t* __restrict__ cell_start,
                                                        uint32_t* __restrict__ tile_of,
                                                        uint32_t* __restrict__ tile_slot,
                                                        uint32_t* __restrict__ num_tiles) {
  uint32_t ps = 0, po = 0, total = 0;
  for (uint32_t k = threadIdx.x; k < blockIdx.x; k += blockDim.x) {
    const uint2 v = sums[k];
    ps += v.x;
    po += v.y;
  }
  (void)block_exclusive_scan(ps, total);
  const uint32_t carry_s = total;
  (void)block_exclusive_scan(po, total);
  const uint32_t carry_o = total;
  const uint32_t e0 = blockIdx.x * (uint32_t)kScanTile + threadIdx.x * (uint32_t)kScanItems;
  uint4* t = reinterpret_cast<uint4*>(cnt + e0);
  uint32_t a[kScanItems];
#pragma unroll
  for (int q = 0; q < kScanItems / 4; ++q) {
    const uint4 u = t[q];
    a[4 * q] = u.x;
    a[4 * q + 1] = u.y;
    a[4 * q + 2] = u.z;
    a[4 * q + 3] = u.w;
  }
  uint32_t s = 0, o = 0, occ = 0;
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    const uint32_t x = a[q];
    const bool f = x != 0u && e0 + (uint32_t)q < ntiles;
    occ |= (uint32_t)f << q;
    o += f;
    a[q] = s;
    s += x;
  }
  const uint32_t off_s = block_exclusive_scan(s, total) + carry_s;
  const uint32_t off_o = block_exclusive_scan(o, total) + carry_o;
#pragma unroll
  for (int q = 0; q < kScanItems / 4; ++q)
    t[q] = make_uint4(a[4 * q] + off_s, a[4 * q + 1] + off_s, a[4 * q + 2] + off_s, a[4 * q + 3] + off_s);
  uint32_t li = off_o;
  for (uint32_t bits = occ; bits != 0u; bits &= bits - 1u) tile_of[li++] = e0 + (uint32_t)(__ffs(bits) - 1);
  if (ntiles >= e0 && ntiles < e0 + (uint32_t)kScanItems) {
    const uint32_t q = ntiles - e0;
    uint32_t of = off_s;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j)
      if ((uint32_t)j == q) of = a[j] + off_s;
    const uint32_t count = off_o + (uint32_t)__popc(occ);  // no flags at or past ntiles
    cell_start[ncells] = of;
    cell_start[ncells + 1] = (uint32_t)n;
    *num_tiles = count;
    tile_slot[count] = of;  // the end of the last tile
  }
}

// One CTA per occupied tile (persistent over the tile list).  The tile's
// particles (`tmp`, grouped by tile) are counted per cell in shared memory;
// the cells' starts are written, with the start of the next tile's first
// cell (the end of this tile's last), and the tile's list entry with the flag
// that routes a tile whose occupied cells average more than dense_mean
// particles to the dense-cell passes.  Then every particle goes to its final
// slot in `perm`: its rank among its cell's particles by in-cell order key
// (the keys are unique).  A tile of at most kTileOrder particles whose cells
// hold at most kOrderSmall each counts the smaller keys in shared memory;
// other tiles scatter their particles by cell into `out` and count in global
// memory, except in cells of kOrderSmall < count <= kOrderLarge particles,
// which go to `large` for k_order_large (the thread of the cell's first slot
// appends it).  Particles of the overflow cell keep their slots.
constexpr int kTileCache = 4;                         // particles per thread held in registers
constexpr int kTileOrder = kTileCache * kThreads;     // 1024
template <int kCells>
__global__ void __launch_bounds__(kThreads) k_tile_cells(int n, int ncells, const uint32_t* __restrict__ tstart,
                                                         const uint32_t* __restrict__ tile_of,
                                                         const uint32_t* __restrict__ num_tiles,
                                                         const uint32_t* __restrict__ tmp,
                                                         const uint32_t* __restrict__ cell_of,
                                                         const unsigned long long* __restrict__ okey,
                                                         uint32_t* __restrict__ rank, uint32_t* __restrict__ perm,
                                                         uint32_t* __restrict__ out, uint32_t* __restrict__ cell_start,
                                                         uint32_t* __restrict__ tile_slot,
                                                         uint8_t* __restrict__ tile_crowd, int dense_mean,
                                                         uint32_t* __restrict__ large,
                                                         uint32_t* __restrict__ large_count) {
  static_assert(kCells == 8 || kCells == 64, "tile of 2x2x2 or 4x4x4 cells");
  __shared__ uint32_t s_cnt[kCells];
  __shared__ uint32_t s_off[kCells + 1];
  __shared__ unsigned long long s_key[kTileOrder];
  __shared__ int s_small;  // every cell of the tile holds at most kOrderSmall particles
  const uint32_t count = *num_tiles;
  const int lane = threadIdx.x & 31;
  for (uint32_t k = blockIdx.x; k < count; k += gridDim.x) {
    const uint32_t t = tile_of[k];
    const uint32_t ts = tstart[t], te = tstart[t + 1];
    const uint32_t cell0 = t * (uint32_t)kCells;
    const bool cached = te - ts <= (uint32_t)kTileOrder;  // uniform
    for (int l = threadIdx.x; l < kCells; l += blockDim.x) s_cnt[l] = 0;
    __syncthreads();
    uint32_t ci[kTileCache], cl[kTileCache], cr[kTileCache];
    if (cached) {
#pragma unroll
      for (int j = 0; j < kTileCache; ++j) {
        const uint32_t e = ts + threadIdx.x + (uint32_t)(j * kThreads);
        ci[j] = cl[j] = cr[j] = 0;
        if (e < te) {
          ci[j] = tmp[e];
          cl[j] = cell_of[ci[j]] - cell0;
          cr[j] = atomicAdd(&s_cnt[cl[j]], 1u);
        }
      }
    } else {
      // A crowded tile: kTileCache particles per thread per round, their
      // loads issued before their counters are taken.
      for (uint32_t e0 = ts + threadIdx.x; e0 < te; e0 += (uint32_t)(kTileCache * kThreads)) {
        uint32_t ii[kTileCache], ll[kTileCache];
#pragma unroll
        for (int j = 0; j < kTileCache; ++j) {
          const uint32_t e = e0 + (uint32_t)(j * kThreads);
          ii[j] = e < te ? tmp[e] : 0u;
        }
#pragma unroll
        for (int j = 0; j < kTileCache; ++j) ll[j] = e0 + (uint32_t)(j * kThreads) < te ? cell_of[ii[j]] - cell0 : 0u;
#pragma unroll
        for (int j = 0; j < kTileCache; ++j)
          if (e0 + (uint32_t)(j * kThreads) < te) rank[ii[j]] = atomicAdd(&s_cnt[ll[j]], 1u);
      }
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      // Lane l holds cells l and l + 32: two warp scans.
      const uint32_t a0 = lane < kCells ? s_cnt[lane] : 0u;
      const uint32_t a1 = kCells > 32 ? s_cnt[(lane + 32) & (kCells - 1)] : 0u;
      uint32_t x0 = a0, x1 = a1;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y0 = __shfl_up_sync(0xffffffffu, x0, o), y1 = __shfl_up_sync(0xffffffffu, x1, o);
        if (lane >= o) {
          x0 += y0;
          x1 += y1;
        }
      }
      const uint32_t total0 = __shfl_sync(0xffffffffu, x0, 31);
      const uint32_t occ = __popc(__ballot_sync(0xffffffffu, a0 > 0u)) + __popc(__ballot_sync(0xffffffffu, a1 > 0u));
      const bool big = __any_sync(0xffffffffu, a0 > kOrderSmall || a1 > kOrderSmall);
      if (lane < kCells) {
        s_off[lane] = x0 - a0;
        cell_start[cell0 + lane] = ts + x0 - a0;
      }
      if (kCells > 32) {
        s_off[lane + 32] = total0 + x1 - a1;
        cell_start[cell0 + lane + 32] = ts + total0 + x1 - a1;
      }
      if (lane == 0) {
        s_off[kCells] = te - ts;
        cell_start[cell0 + kCells] = te;  // the next tile's first cell starts here too
        tile_slot[k] = ts;
        tile_crowd[k] = te - ts > (uint32_t)dense_mean * occ ? 1 : 0;
        s_small = big ? 0 : 1;
      }
    }
    __syncthreads();
    if (cached && s_small) {
#pragma unroll
      for (int j = 0; j < kTileCache; ++j)
        if (ts + threadIdx.x + (uint32_t)(j * kThreads) < te) s_key[s_off[cl[j]] + cr[j]] = okey[ci[j]];
      __syncthreads();
#pragma unroll
      for (int j = 0; j < kTileCache; ++j)
        if (ts + threadIdx.x + (uint32_t)(j * kThreads) < te) {
          const uint32_t c0 = s_off[cl[j]], c1 = s_off[cl[j] + 1];
          const unsigned long long mine = s_key[c0 + cr[j]];
          uint32_t r = 0;
          for (uint32_t q = c0; q < c1; ++q) r += s_key[q] < mine ? 1u : 0u;
          perm[ts + c0 + r] = ci[j];
        }
    } else {
      if (cached) {
#pragma unroll
        for (int j = 0; j < kTileCache; ++j)
          if (ts + threadIdx.x + (uint32_t)(j * kThreads) < te) out[ts + s_off[cl[j]] + cr[j]] = ci[j];
      } else {
        for (uint32_t e0 = ts + threadIdx.x; e0 < te; e0 += (uint32_t)(kTileCache * kThreads)) {
          uint32_t ii[kTileCache], ll[kTileCache], rr[kTileCache];
#pragma unroll
          for (int j = 0; j < kTileCache; ++j) {
            const uint32_t e = e0 + (uint32_t)(j * kThreads);
            ii[j] = e < te ? tmp[e] : 0u;
          }
#pragma unroll
          for (int j = 0; j < kTileCache; ++j) {
            const bool v = e0 + (uint32_t)(j * kThreads) < te;
            ll[j] = v ? cell_of[ii[j]] - cell0 : 0u;
            rr[j] = v ? rank[ii[j]] : 0u;
          }
#pragma unroll
          for (int j = 0; j < kTileCache; ++j)
            if (e0 + (uint32_t)(j * kThreads) < te) out[ts + s_off[ll[j]] + rr[j]] = ii[j];
        }
      }
      __syncthreads();  // the by-cell order is complete
      for (uint32_t e = ts + threadIdx.x; e < te; e += blockDim.x) {
        const uint32_t i = out[e];
        const uint32_t l = cell_of[i] - cell0;
        const uint32_t c0 = ts + s_off[l], c1 = ts + s_off[l + 1];
        if (c1 - c0 > kOrderSmall && c1 - c0 <= kOrderLarge) {
          if (e == c0) large[atomicAdd(large_count, 1u)] = cell0 + l;
          continue;
        }
        const unsigned long long mine = okey[i];
        uint32_t r = 0;
        for (uint32_t q = c0; q < c1; ++q) r += okey[out[q]] < mine ? 1u : 0u;
        perm[c0 + r] = i;
      }
    }
    __syncthreads();  // the counters and keys are free for the next tile
  }
  const uint32_t of = cell_start[ncells];
  for (uint32_t e = of + blockIdx.x * blockDim.x + threadIdx.x; e < (uint32_t)n; e += gridDim.x * blockDim.x) {
    out[e] = tmp[e];
    perm[e] = tmp[e];
  }
}

struct GatherArgs {
  const double* src_pv[6];
  double* dst_pv[6];
  ParticleConsts src, dst;
  int has_ba;
  const uint32_t* cell_of;
  uint32_t* sorted_cell;  // nullable: cell of every sorted slot
  // Tiled compensated form (nullable): the f32 operands of every sorted slot
  // (cell-local position and mass; velocity), and the persistent passes' work
  // queues, reset here.
  float4* cpos;
  float4* cvel;
  uint32_t* queue;
  double inv_cell, h0;
};

__global__ void __launch_bounds__(kThreads) k_gather(int n, const uint32_t* __restrict__ perm, GatherArgs g) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t i = perm[s];
#pragma unroll
  for (int k = 0; k < 6; ++k) g.dst_pv[k][s] = g.src_pv[k][i];
  g.dst.mass[s] = g.src.mass[i];
  g.dst.mat[s] = g.src.mat[i];
  g.dst.id[s] = g.src.id[i];
  if (g.has_ba) {
#pragma unroll
    for (int k = 0; k < 3; ++k) g.dst.ba[k][s] = g.src.ba[k][i];
  }
  if (g.src.scene) g.dst.scene[s] = g.src.scene[i];
  if (g.sorted_cell) g.sorted_cell[s] = g.cell_of[i];
  if (g.cpos) {
    // Cell-local f32 coordinates (the cell is that of the f64 cell key).
    const double x = g.dst_pv[0][s], y = g.dst_pv[1][s], z = g.dst_pv[2][s];
    const long long kx = key_axis(x, g.inv_cell), ky = key_axis(y, g.inv_cell), kz = key_axis(z, g.inv_cell);
    g.cpos[s] = make_float4((float)(x - (double)kx * g.h0), (float)(y - (double)ky * g.h0),
                            (float)(z - (double)kz * g.h0), (float)g.dst.mass[s]);
    g.cvel[s] = make_float4((float)g.dst_pv[3][s], (float)g.dst_pv[4][s], (float)g.dst_pv[5][s], 0.0f);
    if (s == 0 && g.queue) {
      g.queue[0] = 0;  // density and force tile queues
      g.queue[1] = 0;
      g.queue[2] = 0;  // dense-cell task count
      g.queue[3] = 0;  // dense-cell tasks taken by the density and force passes
      g.queue[4] = 0;
    }
  }
}

__global__ void k_unsort_f64(int n, const uint32_t* __restrict__ id, const double* __restrict__ src,
                             double* __restrict__ dst) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) dst[id[s]] = src[s];
}
__global__ void k_unsort_u32(int n, const uint32_t* __restrict__ id, const uint32_t* __restrict__ src,
                             double* __restrict__ dst) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) dst[id[s]] = (double)src[s];
}
__global__ void k_iota(uint32_t* dst, int n) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) dst[s] = (uint32_t)s;
}
__global__ void k_fill(double* dst, double v, int n) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) dst[s] = v;
}
__global__ void k_interleave3(const double* x, const double* y, const double* z, double* d, int n) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) {
    d[3 * (size_t)s] = x[s];
    d[3 * (size_t)s + 1] = y[s];
    d[3 * (size_t)s + 2] = z[s];
  }
}
__global__ void k_deinterleave3(const double* d, double* x, double* y, double* z, int n) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) {
    x[s] = d[3 * (size_t)s];
    y[s] = d[3 * (size_t)s + 1];
    z[s] = d[3 * (size_t)s + 2];
  }
}
__global__ void k_u32_from_f64(const double* src, uint32_t* dst, int n) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) dst[s] = (uint32_t)src[s];
}

}  // namespace

// Persistent grid of k_order_large: its resident CTAs on every SM.
static int order_large_blocks() {
  static const int blocks = [] {
    int dev = 0, sms = 1, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_order_large, kOrderThreads, 0);
    return std::max(sms, 1) * std::max(per, 1);
  }();
  return blocks;
}

// Persistent grid of k_tile_cells: its resident CTAs on every SM.
static int tile_cells_blocks() {
  static const int blocks = [] {
    int dev = 0, sms = 1, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_tile_cells<64>, kThreads, 0);
    return std::max(sms, 1) * std::max(per, 1);
  }();
  return blocks;
}

// Entries scanned per step: the buckets (cells, or tiles) plus the overflow
// bucket, rounded up to whole scan tiles (the padding stays zero, so the
// prefix at index buckets+1 is n).
static int scan_length(int buckets) { return ((buckets + 2 + kScanTile - 1) / kScanTile) * kScanTile; }

size_t scan_block_sums_needed(int ncells) { return (size_t)scan_length(ncells) / kScanTile; }
size_t tile_scan_length(int ncells) { return (size_t)scan_length(ncells / 8); }
size_t tile_scan_sums_needed(int ncells) { return 2 * tile_scan_length(ncells) / kScanTile; }

// Cells of the current positions (pv1): cell_start over the box and perm[s]
// = the particle (index into the current arrays) at sorted slot s, ordered
// by (cell, okey) when okey is given, else by (cell, insertion index).
// In-place exclusive scan of len (a whole number of scan tiles) entries.
static void scan_in_place(uint32_t* v, int len, uint32_t* block_sums, cudaStream_t s) {
  const int nb = len / kScanTile;
  k_scan_reduce<<<nb, kThreads, 0, s>>>(v, block_sums);
  k_scan_top<<<1, 1024, 0, s>>>(block_sums, nb);
  k_scan_apply<<<nb, kThreads, 0, s>>>(v, block_sums);
}

static void build_cells(const StepConsts& c, DevBuffers& b, cudaStream_t s, int bs, unsigned long long* okey,
                        uint32_t* flags) {
  const int n = c.n;
  const ParticleConsts& src = b.pc[b.cur];
  cudaMemsetAsync(b.order_count, 0, sizeof(uint32_t), s);
  if (c.tile) {
    // Tiled: counts per tile, their scan with the occupied-tile list, then
    // cells and in-cell order per occupied tile (the tile-count array is
    // tile_head; the by-cell list of the tiles ordered in global memory goes
    // to sorted_cell, which the gather rewrites).
    const int shift = 3 * c.tile_log2;
    const int ntiles = c.ncells >> shift;
    const int tlen = scan_length(ntiles);
    uint2* sums = reinterpret_cast<uint2*>(b.block_sums);  // 2 x tlen / kScanTile entries
    cudaMemsetAsync(b.tile_head, 0, (size_t)tlen * sizeof(uint32_t), s);
    k_cell_hist<<<grid_for(n, bs), bs, 0, s>>>(c, shift, b.pv1[0], b.pv1[1], b.pv1[2], b.cell_of, b.rank,
                                                 b.tile_head, flags, src.scene, src.id, okey);
    k_tile_reduce<<<tlen / kScanTile, kThreads, 0, s>>>((uint32_t)ntiles, b.tile_head, sums);
    k_tile_scan<<<tlen / kScanTile, kThreads, 0, s>>>(n, c.ncells, (uint32_t)ntiles, b.tile_head, sums,
                                                      b.cell_start, b.tile_of, b.tile_slot, b.num_tiles);
    k_scatter<<<grid_for(n, bs), bs, 0, s>>>(n, shift, b.cell_of, b.rank, b.tile_head, b.tmp);
    auto cells = c.tile == 4 ? k_tile_cells<64> : k_tile_cells<8>;
    cells<<<tile_cells_blocks(), kThreads, 0, s>>>(n, c.ncells, b.tile_head, b.tile_of, b.num_tiles, b.tmp, b.cell_of,
                                                  okey, b.rank, b.perm, b.sorted_cell, b.cell_start, b.tile_slot,
                                                  b.tile_crowd, c.dense_mean, b.large_cells, b.order_count);
    k_order_large<<<order_large_blocks(), kOrderThreads, 0, s>>>(b.cell_start, b.sorted_cell, src.id, okey,
                                                                 b.large_cells, b.order_count, b.perm);
    return;
  }
  const int len = scan_length(c.ncells);
  cudaMemsetAsync(b.cell_start, 0, (size_t)len * sizeof(uint32_t), s);
  k_cell_hist<<<grid_for(n, bs), bs, 0, s>>>(c, 0, b.pv1[0], b.pv1[1], b.pv1[2], b.cell_of, b.rank, b.cell_start,
                                               flags, src.scene, src.id, okey);
  scan_in_place(b.cell_start, len, b.block_sums, s);
  k_scatter<<<grid_for(n, bs), bs, 0, s>>>(n, 0, b.cell_of, b.rank, b.cell_start, b.tmp);
  // `rank` is free after the scatter: it holds the list of large cells.
  k_order<<<grid_for(n, bs), bs, 0, s>>>(n, c.ncells, b.cell_of, b.cell_start, b.tmp, src.id, okey, b.perm, b.rank,
                                         b.order_count);
  k_order_large<<<order_large_blocks(), kOrderThreads, 0, s>>>(b.cell_start, b.tmp, src.id, okey, b.rank,
                                                               b.order_count, b.perm);
}

void launch_cell_index(const StepConsts& c, DevBuffers& b, uint32_t* flags, cudaStream_t s) {
  build_cells(c, b, s, kThreads, nullptr, flags);
}

void launch_sort(const StepConsts& c, DevBuffers& b, cudaStream_t s, int block) {
  // Per-particle kernels take any warp multiple up to kThreads.
  const int bs = block >= 32 && block <= kThreads ? block / 32 * 32 : kThreads;
  const int n = c.n;
  build_cells(c, b, s, bs, c.tile ? b.okey : nullptr, b.flags);
  const ParticleConsts& src = b.pc[b.cur];
  const ParticleConsts& dst = b.pc[b.cur ^ 1];
  GatherArgs g;
  for (int k = 0; k < 6; ++k) {
    g.src_pv[k] = b.pv1[k];
    g.dst_pv[k] = b.pv0[k];
  }
  g.src = src;
  g.dst = dst;
  g.has_ba = b.has_ba ? 1 : 0;
  g.cell_of = b.cell_of;
  g.sorted_cell = c.tile ? b.sorted_cell : nullptr;
  g.cpos = c.tile ? b.cpos : nullptr;
  g.cvel = c.tile ? b.cvel : nullptr;
  g.queue = c.tile ? b.queue : nullptr;
  g.inv_cell = c.inv_cell;
  g.h0 = c.h0;
  k_gather<<<grid_for(n, bs), bs, 0, s>>>(n, b.perm, g);
  b.cur ^= 1;
}

void launch_unsort_f64(const DevBuffers& b, int n, const double* src_sorted, double* dst_orig,
                       cudaStream_t s) {
  k_unsort_f64<<<grid_for(n), kThreads, 0, s>>>(n, b.pc[b.cur].id, src_sorted, dst_orig);
}
void launch_unsort_u32(const DevBuffers& b, int n, const uint32_t* src_sorted, double* dst_orig,
                       cudaStream_t s) {
  k_unsort_u32<<<grid_for(n), kThreads, 0, s>>>(n, b.pc[b.cur].id, src_sorted, dst_orig);
}
void launch_iota(uint32_t* dst, int n, cudaStream_t s) { k_iota<<<grid_for(n), kThreads, 0, s>>>(dst, n); }
void launch_fill_f64(double* dst, double v, int n, cudaStream_t s) {
  k_fill<<<grid_for(n), kThreads, 0, s>>>(dst, v, n);
}
void launch_interleave3(const double* x, const double* y, const double* z, double* dst, int n,
                        cudaStream_t s) {
  k_interleave3<<<grid_for(n), kThreads, 0, s>>>(x, y, z, dst, n);
}
void launch_deinterleave3(const double* src, double* x, double* y, double* z, int n, cudaStream_t s) {
  k_deinterleave3<<<grid_for(n), kThreads, 0, s>>>(src, x, y, z, n);
}
void launch_u32_from_f64(const double* src, uint32_t* dst, int n, cudaStream_t s) {
  k_u32_from_f64<<<grid_for(n), kThreads, 0, s>>>(src, dst, n);
}

}  // namespace phy
