// FP32-compensated SPH passes over staged cell tiles.
//
// The sort orders cells in TB x TB x TB tiles (tiled_index; TB = 4 by
// default, or 2), so the particles of a tile are one contiguous slot range.
// A persistent grid walks the list of occupied tiles; for each tile a CTA
// stages the particles of the tile's (TB+2)^3-cell halo into shared memory
// once (about 3.4 stagings per particle per pass at TB = 4, 8 at TB = 2,
// instead of ~219 per-candidate gathers through L1/L2) and every query
// particle of the tile reads its 27 neighbour cells from there.
//
// Arithmetic is the compensated form of step_comp.cu: f32 pair math on
// tile-relative coordinates (cell offset + cell-local f32 coordinate, so the
// absolute rounding error is about (B+1) h0 2^-24 whatever the scene's
// extent), Kahan-compensated density and force sums, f64 integration.
//
// The density pass records each particle's in-range neighbours as 16-bit
// shared-memory slot indices; the force pass re-stages the same halo in the
// same order and walks the list without re-filtering candidates, so its
// lanes stay converged.  A tile whose halo exceeds the staging capacity is
// processed in x-slabs of 2 or 1 cell layers; a particle whose list exceeds
// kMaxNeighbors is rescanned from the staged cells.  Tiles where no slab
// fits, or flagged crowded by the tile-list kernel (more than kDenseMean
// particles per occupied cell), go to the dense-cell kernels at the end of
// this file.
#include <cuda_runtime.h>

#include <algorithm>

#include "sph_buffers.h"

namespace phy {

namespace {

// Tile shape: TB cells per tile edge (4 or 2, the cells-per-tile knob), its
// log2, the halo edge and the halo's cell count.
template <int TB>
struct Tile {
  static_assert(TB == 2 || TB == 4, "tile edge 2 or 4");
  static constexpr int B = TB;
  static constexpr int L = TB == 4 ? 2 : 1;
  static constexpr int H = TB + 2;
  static constexpr int NH = H * H * H;
};
constexpr int kNHMax = Tile<4>::NH;             // halo table entries reserved in shared memory
constexpr int kTT = 256;                        // threads per CTA
constexpr int kHaloCap = 2000;                  // staged slots per tile (3 force CTAs fit an SM)
static_assert(kNHMax <= kTT, "one halo cell per thread");
static_assert(kHaloCap <= 65536, "16-bit slots");

__device__ __forceinline__ void kahan_add(float& s, float& c, float x) {
  float y = x - c;
  float t = s + y;
  c = (t - s) - y;
  s = t;
}

struct TiledArgs {
  const double* __restrict__ px;
  const double* __restrict__ py;
  const double* __restrict__ pz;
  const double* __restrict__ vx;
  const double* __restrict__ vy;
  const double* __restrict__ vz;
  const double* __restrict__ mass;
  const uint32_t* __restrict__ mat;
  // Cell starts of the occupied tiles' cells (and of the cell after each
  // occupied tile); a tile's particles start at tile_start[tile] and a tile
  // is empty when tile_start[tile + 1] equals it.
  const uint32_t* __restrict__ cell_start;
  const uint32_t* __restrict__ tile_start;
  const uint32_t* __restrict__ sorted_cell;
  const uint32_t* __restrict__ tile_slot;
  const uint8_t* __restrict__ tile_crowd;  // 1: route the tile to the dense-cell passes
  const uint32_t* __restrict__ num_tiles;
  float4* cpos;  // cell-local x, y, z and mass
  float4* cvel;  // vx, vy, vz and p/rho^2
  float* cmr;    // mass/rho
  double* bax;
  double* bay;
  double* baz;
  double* rho;
  double* p;
  double* acc[3];
  double* xsph[3];
  double* mu;
  double* out_pv[6];
  uint16_t* nbr16;
  uint32_t* nbr_count;
  const uint16_t* __restrict__ scene;  // null: one scene
  uint32_t* queue;                      // null: static tile stride
  // Tasks of the dense-cell kernels (tiles too dense to stage): first slot of
  // up to 32 consecutive particles of one cell, and the device task count.
  uint32_t* dense_q0;
  uint32_t* dense_count;
  uint32_t* dense_taken;  // [0]: tasks taken by the density pass, [1]: by the force pass
  // The density pass's in-range masks for the force pass (null: none kept).
  uint32_t* task_mbase;
  uint32_t* task_mcount;
  uint32_t* mask_hdr;
  uint32_t* mask_bits;
  unsigned long long* mask_ctl;
  unsigned long long mask_cap;
  int stride;
  uint32_t* flags;
  unsigned long long* counters;
};

// Packed f32x2 arithmetic (sm_100): two lanes of a 64-bit register pair per
// instruction.
struct f2 {
  unsigned long long v;
};
__device__ __forceinline__ f2 f2_pack(float a, float b) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void f2_unpack(f2 r, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r.v));
}
__device__ __forceinline__ f2 f2_sub(f2 a, f2 b) {
  f2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 f2_add(f2 a, f2 b) {
  f2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b) {
  f2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c) {
  f2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}

// nbr_count value of a particle whose tile was not staged (force rescans).
constexpr uint32_t kNoList = 0xffffffffu;

// Block-wide exclusive scan (kTT threads, one value each).
__device__ __forceinline__ uint32_t block_scan(uint32_t v, uint32_t* ws, uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kTT / 32 ? ws[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kTT / 32) ws[lane] = w;
  }
  __syncthreads();
  total = ws[kTT / 32 - 1];
  const uint32_t off = warp > 0 ? ws[warp - 1] : 0u;
  __syncthreads();
  return off + x - v;
}

struct TileGeom {
  int tx, ty, tz;  // tile coordinates inside the scene box
  int sc;          // scene
  uint32_t first, last;
};

template <int TB>
__device__ __forceinline__ TileGeom tile_geom(const StepConsts& c, const TiledArgs& a, uint32_t k) {
  using T = Tile<TB>;
  TileGeom g;
  g.first = a.tile_slot[k];
  g.last = a.tile_slot[k + 1];
  g.sc = a.scene ? (int)a.scene[g.first] : 0;
  const SceneBox& bx = c.boxes[g.sc];
  const int t = (int)((a.sorted_cell[g.first] - (uint32_t)bx.cell_base) >> (3 * T::L));
  g.tz = t % bx.nt[2];
  g.ty = (t / bx.nt[2]) % bx.nt[1];
  g.tx = t / (bx.nt[2] * bx.nt[1]);
  return g;
}

// Next tile of a persistent CTA: the static stride, or the next entry of the
// pass's work queue (one atomic per tile, broadcast through shared memory).
__device__ __forceinline__ uint32_t next_tile(uint32_t* queue, int pass, uint32_t strided, uint32_t* s_next) {
  if (!queue) return strided;
  __syncthreads();  // every thread has read the previous entry
  if (threadIdx.x == 0) *s_next = atomicAdd(queue + pass, 1u);
  __syncthreads();
  return *s_next;
}

// Slot range [s, e) of cell `lin` of the tiled box: empty when the cell's
// tile holds no particles (an empty tile's cell starts are not written).
template <int TB>
__device__ __forceinline__ void cell_range(const TiledArgs& a, uint32_t lin, uint32_t& s, uint32_t& e) {
  const uint32_t t = lin >> (3 * Tile<TB>::L);
  if (a.tile_start[t + 1] == a.tile_start[t]) {
    s = e = 0;
    return;
  }
  s = a.cell_start[lin];
  e = a.cell_start[lin + 1];
}

// Slot ranges of the tile's halo cells: s_src[h] / s_end[h] = global slot
// range, s_off[h] = first staged slot; every cell's staged range is padded to
// an even length (one far-away dummy particle), so all runs are pair-aligned.
// s_off[T::NH] = total staged slots.
template <int TB>
__device__ __forceinline__ uint32_t halo_table(const StepConsts& c, const TiledArgs& a, const TileGeom& g,
                                               uint32_t* s_src, uint32_t* s_end, uint32_t* s_off, uint32_t* ws) {
  using T = Tile<TB>;
  const int h = threadIdx.x;
  uint32_t cnt = 0, src = 0;
  if (h < T::NH) {
    const SceneBox& bx = c.boxes[g.sc];
    const int ax = g.tx * T::B - 1 + h / (T::H * T::H);
    const int ay = g.ty * T::B - 1 + (h / T::H) % T::H;
    const int az = g.tz * T::B - 1 + h % T::H;
    if (ax >= 0 && ay >= 0 && az >= 0 && ax < bx.nc[0] && ay < bx.nc[1] && az < bx.nc[2]) {
      uint32_t end;
      cell_range<TB>(a, (uint32_t)box_tiled_index(c, bx, ax, ay, az), src, end);
      cnt = end - src;
    }
  }
  uint32_t total;
  const uint32_t off = block_scan((cnt + 1u) & ~1u, ws, total);
  if (h < T::NH) {
    s_src[h] = src;
    s_end[h] = src + cnt;
    s_off[h] = off;
  }
  if (h == 0) s_off[T::NH] = total;
  __syncthreads();
  return total;
}

// Tile-relative f32 position of a particle staged from halo cell h.
template <int TB>
__device__ __forceinline__ float4 tile_rel(const StepConsts& c, float4 q, int h) {
  using T = Tile<TB>;
  const float ox = (float)(h / (T::H * T::H) - 1) * c.h0f;
  const float oy = (float)((h / T::H) % T::H - 1) * c.h0f;
  const float oz = (float)(h % T::H - 1) * c.h0f;
  return make_float4(ox + q.x, oy + q.y, oz + q.z, q.w);
}

// Halo cell of a particle of the tile itself.
template <int TB>
__device__ __forceinline__ int own_halo_cell(uint32_t cell) {
  using T = Tile<TB>;
  const int u = (int)(cell & ((1u << (3 * T::L)) - 1u));
  const int ux = u >> (2 * T::L), uy = (u >> T::L) & (T::B - 1), uz = u & (T::B - 1);
  return ((ux + 1) * T::H + (uy + 1)) * T::H + (uz + 1);
}

// Warp-cooperative staging: warp w copies halo z-runs w, w+8, ... (6 cells
// with fixed hx, hy; their staged slots are contiguous), lanes taking
// consecutive slots so global reads coalesce.  `emit(slot, h, src)` stores
// one particle read from global slot `src` of halo cell h.
template <int TB, class Emit, class Dummy>
__device__ __forceinline__ void stage_halo(const uint32_t* s_src, const uint32_t* s_end, const uint32_t* s_off,
                                           int run_lo, int run_hi, uint32_t base, Emit emit, Dummy dummy) {
  using T = Tile<TB>;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int run = run_lo + warp; run < run_hi; run += kTT / 32) {
    const int h0 = run * T::H;
    const uint32_t b0 = s_off[h0], b6 = s_off[h0 + T::H];
#pragma unroll 4
    for (uint32_t k = b0 + lane; k < b6; k += 32) {
      int hz = 0;
#pragma unroll
      for (int z = 1; z < T::H; ++z) hz += k >= s_off[h0 + z] ? 1 : 0;
      const int h = h0 + hz;
      const uint32_t src = s_src[h] + (k - s_off[h]);
      if (src < s_end[h])
        emit(k - base, h, src);
      else
        dummy(k - base);
    }
  }
}

// Slab decomposition of a tile whose whole halo does not fit the staging
// buffer: the core is processed in x-slabs of `slab` cell layers, each with
// the (slab+2) x H x H-cell halo (a contiguous halo-index range).  Returns
// the thickest slab (TB, 2 or 1) whose halos all fit, or 0 (none fits).
template <int TB>
__device__ __forceinline__ int pick_slab(const uint32_t* s_off, uint32_t cap) {
  using T = Tile<TB>;
  constexpr int L = T::H * T::H;  // halo cells per x-layer
  if (s_off[T::NH] <= cap) return T::B;
  if (T::B == 4 && s_off[4 * L] - s_off[0] <= cap && s_off[6 * L] - s_off[2 * L] <= cap) return 2;
  for (int x0 = 0; x0 < T::B; ++x0)
    if (s_off[(x0 + 3) * L] - s_off[x0 * L] > cap) return 0;
  return 1;
}

__device__ __forceinline__ void write_density(const StepConsts& c, const TiledArgs& a, int qi, double rho) {
  const double over = rho - c.rest;
  const double pr = over > 0.0 ? c.stiff * over : 0.0;
  const double inv = 1.0 / rho;
  a.rho[qi] = rho;
  a.p[qi] = pr;
  a.cvel[qi].w = (float)(pr * inv * inv);
  a.cmr[qi] = (float)(a.mass[qi] * inv);
}

// Staged density operands: slots 2p and 2p+1 share two float4s,
// (x0, x1, y0, y1) and (z0, z1, m0, m1), so a pair of candidates loads into
// 64-bit register pairs ready for f32x2 arithmetic.
__device__ __forceinline__ void put_pair_slot(float* sp, uint32_t k, float4 v) {
  float* base = sp + (k >> 1) * 8 + (k & 1);
  base[0] = v.x;
  base[2] = v.y;
  base[4] = v.z;
  base[6] = v.w;
}

constexpr float kFar = 1.0e18f;  // dummy particle coordinate (never in range)

// Filters staged candidates [cb, ce) (an even count, at most 32) against a
// query at (PX, PY, PZ): returns the in-range mask (bit k = candidate cb + k)
// and adds -m_j (h0^2 - r^2)^3 of the in-range candidates to NPART.  With the
// cutoff equal to the kernel radius (kExact) d = r^2 - h0^2 gives both: its
// sign bit is the in-range bit (d is never -0: r^2 >= +0 and h0^2 > 0), and
// min(d, 0)^3 = -(h0^2 - r^2)^3 rounds exactly as the positive form.  The
// bits are shifted in from the right, so the chunk's first candidate ends in
// the highest bit and one bit reversal restores candidate order.
template <bool kExact>
__device__ __forceinline__ uint32_t filter_chunk(const float4* s_pp4, uint32_t cb, uint32_t ce, f2 PX, f2 PY,
                                                 f2 PZ, f2 HC2, f2 H0SQ, f2& NPART) {
  uint32_t mask = 0;
#pragma unroll 2
  for (uint32_t j = cb; j < ce; j += 2) {
    const float4 A = s_pp4[j];      // x0 x1 y0 y1
    const float4 B = s_pp4[j + 1];  // z0 z1 m0 m1
    const f2 DX = f2_sub(f2_pack(A.x, A.y), PX);
    const f2 DY = f2_sub(f2_pack(A.z, A.w), PY);
    const f2 DZ = f2_sub(f2_pack(B.x, B.y), PZ);
    const f2 R2 = f2_fma(DZ, DZ, f2_fma(DY, DY, f2_mul(DX, DX)));
    float d0, d1, n0, n1;
    f2_unpack(f2_sub(R2, HC2), d0, d1);
    mask = __funnelshift_l(__float_as_uint(d0), mask, 1);
    mask = __funnelshift_l(__float_as_uint(d1), mask, 1);
    if (kExact) {
      n0 = fminf(d0, 0.f);
      n1 = fminf(d1, 0.f);
    } else {
      float e0, e1;
      f2_unpack(f2_sub(R2, H0SQ), e0, e1);
      n0 = d0 < 0.f ? e0 : 0.f;
      n1 = d1 < 0.f ? e1 : 0.f;
    }
    const f2 N = f2_pack(n0, n1);
    NPART = f2_fma(f2_mul(N, N), f2_mul(N, f2_pack(B.z, B.w)), NPART);
  }
  return __brev(mask) >> (32u - (ce - cb));
}

// Appends 16-bit neighbour slots to a particle's row-major list (row of
// kMaxNeighbors entries) through a 64-bit register accumulator (hi:lo) that
// shifts each new slot in from the top, so four pushes leave the oldest slot
// in the low 16 bits; flushed with 8-byte stores.  Entries past
// kMaxNeighbors are dropped (the count still grows and the force pass then
// rescans).
struct ListWriter {
  uint16_t* row;
  uint32_t lo = 0, hi = 0;
  uint32_t n = 0;
  __device__ __forceinline__ void push(uint32_t slot) {
    lo = __funnelshift_r(lo, hi, 16);    // low word of (hi:lo) >> 16
    hi = __byte_perm(hi, slot, 0x5432);  // (hi >> 16) | (slot << 16)
    ++n;
    if ((n & 3) == 0 && n <= (uint32_t)kMaxNeighbors)
      *reinterpret_cast<uint2*>(row + n - 4) = make_uint2(lo, hi);
  }
  __device__ __forceinline__ void finish() {
    const uint32_t r = n & 3;  // pending slots, in the top r * 16 bits
    if (r && n < (uint32_t)kMaxNeighbors) {
      const unsigned long long v = (((unsigned long long)hi << 32) | lo) >> (16 * (4 - r));
      *reinterpret_cast<unsigned long long*>(row + (n & ~3u)) = v;
    }
  }
};

// Appends the dense-cell work of tile g to the task list (one atomic per
// tile): every occupied cell of the tile contributes ceil(count / 32) tasks,
// each the first sorted slot of up to 32 consecutive particles of that cell
// (the cell is sorted_cell[slot]).  Uniform across the CTA; `s_pre` is
// shared scratch of T::B^3 + 1 entries (the caller lends the halo table's
// s_src, which the next tile rebuilds).
template <int TB>
__device__ __forceinline__ void queue_dense_tasks(const TiledArgs& a, const TileGeom& g, uint32_t* ws,
                                                  uint32_t* s_pre, uint32_t* s_base) {
  using T = Tile<TB>;
  constexpr int kCells = T::B * T::B * T::B;
  const uint32_t first_cell = (a.sorted_cell[g.first] >> (3 * T::L)) << (3 * T::L);
  const int t = threadIdx.x;
  const uint32_t cell = first_cell + (uint32_t)t;
  uint32_t q0 = 0, cnt = 0;
  if (t < kCells) {
    q0 = a.cell_start[cell];
    cnt = a.cell_start[cell + 1] - q0;
  }
  uint32_t total;
  const uint32_t off = block_scan((cnt + 31u) >> 5, ws, total);
  if (t < kCells) s_pre[t] = off;
  if (t == 0) {
    s_pre[kCells] = total;
    *s_base = atomicAdd(a.dense_count, total);
  }
  __syncthreads();
  const uint32_t base = *s_base;
  for (uint32_t k = (uint32_t)t; k < total; k += kTT) {
    int lo = 0, hi = kCells - 1;  // last cell with s_pre <= k
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (s_pre[mid] <= k) lo = mid; else hi = mid - 1;
    }
    a.dense_q0[base + k] = a.cell_start[first_cell + (uint32_t)lo] + 32u * (k - s_pre[lo]);
  }
  __syncthreads();
}

// kExact: the cutoff min(h, h0) equals the kernel radius h0 (the usual case).
// Six CTAs per SM is the shared-memory limit (35 KB each); the register cap
// that matches it (40) costs no spill.
template <int TB, bool kCount, bool kExact>
__global__ void __launch_bounds__(kTT, 6) k_density_tiled(StepConsts c, TiledArgs a) {
  using T = Tile<TB>;
  extern __shared__ __align__(16) unsigned char smem[];
  float* s_pp = reinterpret_cast<float*>(smem);  // kHaloCap slots, pair-interleaved
  uint32_t* s_src = reinterpret_cast<uint32_t*>(smem + kHaloCap * sizeof(float4));
  uint32_t* s_end = s_src + T::NH;
  uint32_t* s_off = s_end + T::NH;
  uint32_t* ws = s_off + T::NH + 1;
  const float hc2 = fminf(c.h2f, c.h0sqf);
  const f2 HC2 = f2_pack(hc2, hc2), H0SQ = f2_pack(c.h0sqf, c.h0sqf);
  __shared__ uint32_t s_next;
  const uint32_t ntiles = *a.num_tiles;
  unsigned cand = 0, pairs = 0;
  for (uint32_t k = next_tile(a.queue, 0, blockIdx.x, &s_next); k < ntiles;
       k = next_tile(a.queue, 0, k + gridDim.x, &s_next)) {
    const TileGeom g = tile_geom<TB>(c, a, k);
    halo_table<TB>(c, a, g, s_src, s_end, s_off, ws);
    const int slab = a.tile_crowd[k] ? 0 : pick_slab<TB>(s_off, (uint32_t)min(c.halo_cap, kHaloCap));
    if (slab == 0) {
      queue_dense_tasks<TB>(a, g, ws, s_src, &s_next);
      continue;  // uniform across the CTA
    }
    for (int x0 = 0; x0 < T::B; x0 += slab) {
    const uint32_t base = s_off[x0 * T::H * T::H];
    stage_halo<TB>(
        s_src, s_end, s_off, x0 * T::H, (x0 + slab + 2) * T::H, base,
        [&](uint32_t slot, int h, uint32_t src) { put_pair_slot(s_pp, slot, tile_rel<TB>(c, a.cpos[src], h)); },
        [&](uint32_t slot) { put_pair_slot(s_pp, slot, make_float4(kFar, kFar, kFar, 0.f)); });
    __syncthreads();
    const float4* s_pp4 = reinterpret_cast<const float4*>(s_pp);
    const uint32_t qfirst = s_src[((x0 + 1) * T::H + 1) * T::H + 1];
    const uint32_t qlast = s_end[((x0 + slab) * T::H + T::B) * T::H + T::B];
    for (uint32_t qi = qfirst + threadIdx.x; qi < qlast; qi += kTT) {
      const int hq = own_halo_cell<TB>(a.sorted_cell[qi]);
      const uint32_t si = s_off[hq] - base + (qi - s_src[hq]);
      const float* own = s_pp + (si >> 1) * 8 + (si & 1);
      const f2 PX = f2_pack(own[0], own[0]), PY = f2_pack(own[2], own[2]), PZ = f2_pack(own[4], own[4]);
      float s = 0.f, comp = 0.f;
      ListWriter lw;
      lw.row = a.nbr16 + (size_t)qi * kMaxNeighbors;
#pragma unroll
      for (int di = -1; di <= 1; ++di) {
#pragma unroll
        for (int dj = -1; dj <= 1; ++dj) {
          const int h0 = hq + di * T::H * T::H + dj * T::H - 1;  // cells h0 .. h0+2 (dk = -1, 0, 1)
          const uint32_t s0 = s_off[h0] - base, e0 = s_off[h0 + 3] - base;  // both even
          if (kCount)
            cand += (s_end[h0] - s_src[h0]) + (s_end[h0 + 1] - s_src[h0 + 1]) + (s_end[h0 + 2] - s_src[h0 + 2]);
          f2 NPART = f2_pack(0.f, 0.f);
          for (uint32_t cb = s0; cb < e0; cb += 32) {
            const uint32_t ce = min(cb + 32u, e0);
            uint32_t mask = filter_chunk<kExact>(s_pp4, cb, ce, PX, PY, PZ, HC2, H0SQ, NPART);
            if (kCount) pairs += __popc(mask);
            while (mask) {
              const uint32_t b = __ffs(mask) - 1;
              mask &= mask - 1;
              lw.push(cb + b);
            }
          }
          float p0, p1;
          f2_unpack(NPART, p0, p1);
          kahan_add(s, comp, c.poly6_cf * -(p0 + p1));
        }
      }
      lw.finish();
      a.nbr_count[qi] = lw.n;
      write_density(c, a, (int)qi, (double)s - (double)comp);
    }
    __syncthreads();
    }  // slabs
  }
  // Particles of the overflow cell (outside the grid box): no neighbours.
  const uint32_t end = a.tile_slot[ntiles];
  for (uint32_t qi = end + blockIdx.x * kTT + threadIdx.x; qi < (uint32_t)c.n; qi += gridDim.x * kTT) {
    write_density(c, a, (int)qi, 0.0);
    a.nbr_count[qi] = 0;
  }
  if (kCount) {
    const unsigned wc = __reduce_add_sync(0xffffffffu, cand);
    const unsigned wp = __reduce_add_sync(0xffffffffu, pairs);
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&a.counters[0], (unsigned long long)wc);
      atomicAdd(&a.counters[1], (unsigned long long)wp);
    }
  }
}

struct CompAcc {
  float fpx = 0.f, fpy = 0.f, fpz = 0.f, cpx = 0.f, cpy = 0.f, cpz = 0.f;
  float fvx = 0.f, fvy = 0.f, fvz = 0.f, cvx = 0.f, cvy = 0.f, cvz = 0.f;
  float xsx = 0.f, xsy = 0.f, xsz = 0.f, shear = 0.f, csh = 0.f;
};

// mu_eff, acc, integrate and bounds in f64 (world.rs:319-397).
// The f64 operands of a particle's integration epilogue, loaded before its
// pair loop so their latency overlaps the pair work.
struct OwnState {
  double rho, p3[3], v3[3];
  uint32_t mat;
};

__device__ __forceinline__ OwnState load_own(const TiledArgs& a, int i) {
  OwnState o;
  o.rho = a.rho[i];
  o.mat = a.mat[i];
  o.p3[0] = a.px[i];
  o.p3[1] = a.py[i];
  o.p3[2] = a.pz[i];
  o.v3[0] = a.vx[i];
  o.v3[1] = a.vy[i];
  o.v3[2] = a.vz[i];
  return o;
}

__device__ __forceinline__ void finish_particle(const StepConsts& c, const TiledArgs& a, int i, const CompAcc& q,
                                                const SceneBox& bx, const OwnState& own) {
  const double rho_i = own.rho;
  const uint32_t m = own.mat;
  const int midx = (int)m < c.n_visc_k ? (int)m : 0;
  double kc, nn;
  material_coeffs(c, midx, kc, nn);
  const double ex = nn - 1.0;
  const double sh = (double)q.shear - (double)q.csh;
  const double sreg = sh > c.shear_min ? sh : c.shear_min;
  const double mu = kc * (ex == 0.0 ? 1.0 : pow(sreg, ex));
  double ax = 0.0, ay = 0.0, az = 0.0;
  if (rho_i > 0.0) {
    const double inv = 1.0 / rho_i;
    ax = (((double)q.fpx - (double)q.cpx) + ((double)q.fvx - (double)q.cvx) * mu) * inv;
    ay = (((double)q.fpy - (double)q.cpy) + ((double)q.fvy - (double)q.cvy) * mu) * inv;
    az = (((double)q.fpz - (double)q.cpz) + ((double)q.fvz - (double)q.cvz) * mu) * inv;
  }
  a.acc[0][i] = ax;
  a.acc[1][i] = ay;
  a.acc[2][i] = az;
  a.xsph[0][i] = q.xsx;
  a.xsph[1][i] = q.xsy;
  a.xsph[2][i] = q.xsz;
  a.mu[i] = mu;
  double b3[3] = {0.0, 0.0, 0.0};
  if (a.bax) {
    b3[0] = a.bax[i];
    b3[1] = a.bay[i];
    b3[2] = a.baz[i];
    a.bax[i] = 0.0;
    a.bay[i] = 0.0;
    a.baz[i] = 0.0;
  }
  double p3[3] = {own.p3[0], own.p3[1], own.p3[2]};
  double v3[3] = {own.v3[0], own.v3[1], own.v3[2]};
  const double acc3[3] = {ax, ay, az};
  const double xs3[3] = {(double)q.xsx, (double)q.xsy, (double)q.xsz};
  bool finite = true;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double v = v3[k] + ((acc3[k] + c.g[k]) + b3[k]) * c.dt;
    v = v + xs3[k] * c.xsph_eps;
    double x = p3[k] + v * c.dt;
    if (x < bx.lo[k]) {
      x = bx.lo[k];
      v = -v * c.damp;
    } else if (x > bx.hi[k]) {
      x = bx.hi[k];
      v = -v * c.damp;
    }
    finite = finite && isfinite(x) && isfinite(v);
    a.out_pv[k][i] = x;
    a.out_pv[3 + k][i] = v;
  }
  if (!finite) atomicOr(a.flags, kFlagNonFinite);
}

// The same with the particle's f64 state loaded at the point of use.
__device__ __forceinline__ void finish_particle(const StepConsts& c, const TiledArgs& a, int i, const CompAcc& q,
                                                const SceneBox& bx) {
  finish_particle(c, a, i, q, bx, load_own(a, i));
}

// Batch partial sums of the pressure and raw viscous forces (and of the
// shear sum, when it is live); folded into the Kahan-compensated totals every
// eight pairs, scaled by the query's common factors (sp = m_i * spiky
// coefficient, sv = m_i * laplacian coefficient).
struct ForcePart {
  float fx = 0.f, fy = 0.f, fz = 0.f, vx = 0.f, vy = 0.f, vz = 0.f, sh = 0.f;
};

template <bool kShear>
__device__ __forceinline__ void fold(CompAcc& q, ForcePart& b, float sp, float sv) {
  kahan_add(q.fpx, q.cpx, sp * b.fx);
  kahan_add(q.fpy, q.cpy, sp * b.fy);
  kahan_add(q.fpz, q.cpz, sp * b.fz);
  kahan_add(q.fvx, q.cvx, sv * b.vx);
  kahan_add(q.fvy, q.cvy, sv * b.vy);
  kahan_add(q.fvz, q.cvz, sv * b.vz);
  if (kShear) kahan_add(q.shear, q.csh, b.sh);
  b = ForcePart();
}

// One listed neighbour (r < min(h, h0) by construction; r == 0, i.e. i
// itself or a coincident particle, contributes nothing, as the reference
// skips r <= 0).  Branchless.  kShear = false leaves out the shear sum
// (StepConsts::shear_live).
template <bool kShear>
__device__ __forceinline__ void pair_listed(const StepConsts& c, float4 pj, float4 vj, float mr_j, float4 pi,
                                            float4 vi, float lapm_i, ForcePart& b, CompAcc& q) {
  const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
  const float r2 = dx * dx + dy * dy + dz * dz;
  const bool pos = r2 > 0.f;
  const float inv_r = pos ? rsqrtf(r2) : 0.f;
  const float mr = pos ? mr_j : 0.f;
  const float r = r2 * inv_r;
  const float hr = c.h0f - r;
  // (d/r) * m_j (p_i/rho_i^2 + p_j/rho_j^2) (h - r)^2; times m_i and the
  // spiky coefficient at the fold
  const float fp = (pj.w * (vi.w + vj.w)) * (hr * (hr * inv_r));
  b.fx = fmaf(dx, fp, b.fx);
  b.fy = fmaf(dy, fp, b.fy);
  b.fz = fmaf(dz, fp, b.fz);
  // dv * m_j / rho_j (h - r); times m_i and the laplacian coefficient at the
  // fold
  const float dvx = vj.x - vi.x, dvy = vj.y - vi.y, dvz = vj.z - vi.z;
  const float vf = mr * hr;
  b.vx = fmaf(dvx, vf, b.vx);
  b.vy = fmaf(dvy, vf, b.vy);
  b.vz = fmaf(dvz, vf, b.vz);
  // XSPH: dv * (m_j / rho_j * poly6(r))
  const float t = c.h0sqf - r2;
  const float xw = (mr * c.poly6_cf) * (t * t * t);
  q.xsx = fmaf(dvx, xw, q.xsx);
  q.xsy = fmaf(dvy, xw, q.xsy);
  q.xsz = fmaf(dvz, xw, q.xsz);
  // strain-rate proxy: |dv| / (r + 1e-4) * m_j / rho_j
  if (kShear) {
    const float dv2 = dvx * dvx + dvy * dvy + dvz * dvz;
    const float dvn = dv2 > 0.f ? dv2 * rsqrtf(dv2) : 0.f;
    b.sh = fmaf(__fdividef(dvn, r + 1e-4f), mr, b.sh);
  }
}

// Two listed neighbours of one query at once on packed f32x2 arithmetic
// (the terms of pair_listed without the shear sum).  A candidate given with
// mass 0 and m/rho 0 adds exactly nothing, which pads a lane's odd last pair.
struct QueryPack {
  f2 px, py, pz, pw, vx, vy, vz, vw, lapm, h0, h0sq, spk, p6;
};
struct ForcePart2 {
  f2 fx, fy, fz, vx, vy, vz, xx, xy, xz;
};

__device__ __forceinline__ QueryPack query_pack(const StepConsts& c, float4 pi, float4 vi, float lapm) {
  QueryPack q;
  q.px = f2_pack(pi.x, pi.x);
  q.py = f2_pack(pi.y, pi.y);
  q.pz = f2_pack(pi.z, pi.z);
  q.pw = f2_pack(pi.w, pi.w);
  q.vx = f2_pack(vi.x, vi.x);
  q.vy = f2_pack(vi.y, vi.y);
  q.vz = f2_pack(vi.z, vi.z);
  q.vw = f2_pack(vi.w, vi.w);
  q.lapm = f2_pack(lapm, lapm);
  q.h0 = f2_pack(c.h0f, c.h0f);
  q.h0sq = f2_pack(c.h0sqf, c.h0sqf);
  q.spk = f2_pack(c.spiky_cf, c.spiky_cf);
  q.p6 = f2_pack(c.poly6_cf, c.poly6_cf);
  return q;
}

__device__ __forceinline__ void zero(ForcePart2& b) {
  const f2 z = f2_pack(0.f, 0.f);
  b.fx = b.fy = b.fz = b.vx = b.vy = b.vz = b.xx = b.xy = b.xz = z;
}

__device__ __forceinline__ void pair2_listed(const QueryPack& Q, float4 pa, float4 va, float mra, float4 pb,
                                             float4 vb, float mrb, ForcePart2& b) {
  const f2 DX = f2_sub(f2_pack(pa.x, pb.x), Q.px);
  const f2 DY = f2_sub(f2_pack(pa.y, pb.y), Q.py);
  const f2 DZ = f2_sub(f2_pack(pa.z, pb.z), Q.pz);
  const f2 R2 = f2_fma(DZ, DZ, f2_fma(DY, DY, f2_mul(DX, DX)));
  float r2a, r2b;
  f2_unpack(R2, r2a, r2b);
  const bool posa = r2a > 0.f, posb = r2b > 0.f;
  const f2 INV = f2_pack(posa ? rsqrtf(r2a) : 0.f, posb ? rsqrtf(r2b) : 0.f);
  const f2 MR = f2_pack(posa ? mra : 0.f, posb ? mrb : 0.f);
  const f2 HR = f2_sub(Q.h0, f2_mul(R2, INV));
  // (d/r) * m_i m_j (p_i/rho_i^2 + p_j/rho_j^2) * spiky(r)
  const f2 FP = f2_mul(f2_mul(f2_mul(f2_mul(Q.pw, f2_pack(pa.w, pb.w)), f2_add(Q.vw, f2_pack(va.w, vb.w))),
                              f2_mul(Q.spk, HR)),
                       f2_mul(HR, INV));
  b.fx = f2_fma(DX, FP, b.fx);
  b.fy = f2_fma(DY, FP, b.fy);
  b.fz = f2_fma(DZ, FP, b.fz);
  // dv * (m_i m_j / rho_j * lap(r))
  const f2 DVX = f2_sub(f2_pack(va.x, vb.x), Q.vx);
  const f2 DVY = f2_sub(f2_pack(va.y, vb.y), Q.vy);
  const f2 DVZ = f2_sub(f2_pack(va.z, vb.z), Q.vz);
  const f2 VF = f2_mul(f2_mul(Q.lapm, MR), HR);
  b.vx = f2_fma(DVX, VF, b.vx);
  b.vy = f2_fma(DVY, VF, b.vy);
  b.vz = f2_fma(DVZ, VF, b.vz);
  // XSPH: dv * (m_j / rho_j * poly6(r))
  const f2 T = f2_sub(Q.h0sq, R2);
  const f2 XW = f2_mul(f2_mul(MR, Q.p6), f2_mul(f2_mul(T, T), T));
  b.xx = f2_fma(DVX, XW, b.xx);
  b.xy = f2_fma(DVY, XW, b.xy);
  b.xz = f2_fma(DVZ, XW, b.xz);
}

// Folds both halves of the packed partial sums into the compensated totals.
__device__ __forceinline__ void fold2(CompAcc& q, ForcePart2& b) {
  float lo, hi;
  f2_unpack(b.fx, lo, hi);
  kahan_add(q.fpx, q.cpx, lo + hi);
  f2_unpack(b.fy, lo, hi);
  kahan_add(q.fpy, q.cpy, lo + hi);
  f2_unpack(b.fz, lo, hi);
  kahan_add(q.fpz, q.cpz, lo + hi);
  f2_unpack(b.vx, lo, hi);
  kahan_add(q.fvx, q.cvx, lo + hi);
  f2_unpack(b.vy, lo, hi);
  kahan_add(q.fvy, q.cvy, lo + hi);
  f2_unpack(b.vz, lo, hi);
  kahan_add(q.fvz, q.cvz, lo + hi);
  f2_unpack(b.xx, lo, hi);
  q.xsx += lo + hi;
  f2_unpack(b.xy, lo, hi);
  q.xsy += lo + hi;
  f2_unpack(b.xz, lo, hi);
  q.xsz += lo + hi;
  zero(b);
}

// Three CTAs per SM is the shared-memory limit (75 KB each), so registers up to
// 65536 / (3 x 256) cost no occupancy.
template <int TB, bool kShear>
__global__ void __launch_bounds__(kTT, 3) k_force_tiled(StepConsts c, TiledArgs a) {
  using T = Tile<TB>;
  extern __shared__ __align__(16) unsigned char smem[];
  // Staged neighbour records as separate 16-byte arrays (a 32-byte record
  // stride would map every record onto 4 of the 8 bank quads).
  float4* s_pos = reinterpret_cast<float4*>(smem);
  float4* s_vel = s_pos + kHaloCap;
  float* s_mr = reinterpret_cast<float*>(s_vel + kHaloCap);
  uint32_t* s_src = reinterpret_cast<uint32_t*>(s_mr + kHaloCap);
  uint32_t* s_end = s_src + T::NH;
  uint32_t* s_off = s_end + T::NH;
  uint32_t* ws = s_off + T::NH + 1;
  const float hc2 = fminf(c.h2f, c.h0sqf);
  __shared__ uint32_t s_next;
  const uint32_t ntiles = *a.num_tiles;
  for (uint32_t k = next_tile(a.queue, 1, blockIdx.x, &s_next); k < ntiles;
       k = next_tile(a.queue, 1, k + gridDim.x, &s_next)) {
    const TileGeom g = tile_geom<TB>(c, a, k);
    halo_table<TB>(c, a, g, s_src, s_end, s_off, ws);
    const int slab = a.tile_crowd[k] ? 0 : pick_slab<TB>(s_off, (uint32_t)min(c.halo_cap, kHaloCap));
    if (slab == 0) continue;  // the dense-cell pass computes this tile
    for (int x0 = 0; x0 < T::B; x0 += slab) {
    const uint32_t base = s_off[x0 * T::H * T::H];
    stage_halo<TB>(
        s_src, s_end, s_off, x0 * T::H, (x0 + slab + 2) * T::H, base,
        [&](uint32_t slot, int h, uint32_t src) {
          s_pos[slot] = tile_rel<TB>(c, a.cpos[src], h);
          s_vel[slot] = a.cvel[src];
          s_mr[slot] = a.cmr[src];
        },
        [&](uint32_t slot) {
          s_pos[slot] = make_float4(kFar, kFar, kFar, 0.f);
          s_vel[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
          s_mr[slot] = 0.f;
        });
    __syncthreads();
    const uint32_t qfirst = s_src[((x0 + 1) * T::H + 1) * T::H + 1];
    const uint32_t qlast = s_end[((x0 + slab) * T::H + T::B) * T::H + T::B];
    for (uint32_t qi = qfirst + threadIdx.x; qi < qlast; qi += kTT) {
      const int hq = own_halo_cell<TB>(a.sorted_cell[qi]);
      const uint32_t si = s_off[hq] - base + (qi - s_src[hq]);
      const float4 pi = s_pos[si];
      const float4 vi = s_vel[si];
      const float lapm_i = pi.w * c.lap_cf;
      const OwnState own = load_own(a, (int)qi);
      CompAcc q;
      ForcePart b;
      const uint32_t cnt = a.nbr_count[qi];
      if (cnt <= (uint32_t)kMaxNeighbors) {
        // Row-major list: 8 entries per 16-byte load, the next load issued
        // before the current eight pairs are computed.
        const uint4* row = reinterpret_cast<const uint4*>(a.nbr16 + (size_t)qi * kMaxNeighbors);
        uint4 cur = cnt > 0 ? row[0] : make_uint4(0, 0, 0, 0);
        for (uint32_t e0 = 0; e0 < cnt; e0 += 8) {
          const uint4 nxt = e0 + 8 < cnt ? row[(e0 >> 3) + 1] : cur;
          const uint32_t w[4] = {cur.x, cur.y, cur.z, cur.w};
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            if (e0 + u < cnt) {
              const uint32_t j = (w[u >> 1] >> (16 * (u & 1))) & 0xffffu;
              pair_listed<kShear>(c, s_pos[j], s_vel[j], s_mr[j], pi, vi, lapm_i, b, q);
            }
            if (u == 7) fold<kShear>(q, b, pi.w * c.spiky_cf, lapm_i);
          }
          cur = nxt;
        }
      } else {
        // List overflow: rescan the 27 staged cells with the cutoff test.
        for (int di = -1; di <= 1; ++di)
          for (int dj = -1; dj <= 1; ++dj) {
            const int h0 = hq + di * T::H * T::H + dj * T::H - 1;
            for (uint32_t j = s_off[h0] - base; j < s_off[h0 + 3] - base; ++j) {
              const float4 pj = s_pos[j];
              const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
              if (!(dx * dx + dy * dy + dz * dz < hc2)) continue;
              pair_listed<kShear>(c, pj, s_vel[j], s_mr[j], pi, vi, lapm_i, b, q);
              fold<kShear>(q, b, pi.w * c.spiky_cf, lapm_i);
            }
          }
      }
      finish_particle(c, a, (int)qi, q, c.boxes[g.sc], own);
    }
    __syncthreads();
    }  // slabs
  }
  const uint32_t end = a.tile_slot[ntiles];
  for (uint32_t qi = end + blockIdx.x * kTT + threadIdx.x; qi < (uint32_t)c.n; qi += gridDim.x * kTT) {
    CompAcc q;
    finish_particle(c, a, (int)qi, q, c.boxes[a.scene ? (int)a.scene[qi] : 0], load_own(a, (int)qi));
  }
}

// ---- Dense cells ---------------------------------------------------------------
//
// Tiles whose halo does not fit the staging buffer even in 1-layer slabs, or
// whose occupied cells average more than kDenseMean particles (cells of tens
// to thousands of particles, as when the fluid has collapsed onto the floor),
// are computed by warps: a task is up to 32 consecutive particles of one cell
// (one query per lane; the in-cell Morton order makes them a compact clump),
// and the warp streams each of the 27 neighbour cells in chunks of 32
// candidates (one per lane, coalesced), staged in the warp's own shared
// memory.  A chunk is skipped whole when the bounding boxes of the warp's
// queries and of the chunk's candidates are at least the cutoff apart, which
// removes about half the candidates of a crowded neighbourhood.  Tasks come
// from a device counter (one atomic per task), so no barrier joins warps.
//
// The density pass also keeps every chunk's 32 lane masks of in-range
// candidates (chunks where some lane has one), in a buffer each task reserves
// at its start for its upper bound of chunks.  The force pass of the same
// step, at the same positions, walks the kept masks in the same order instead
// of filtering again, which gives the same pairs in the same order; a task
// whose reservation did not fit filters as before.

constexpr int kWT = 256;  // threads per dense-task CTA
constexpr int kWarps = kWT / 32;
constexpr uint32_t kNoMasks = 0xffffffffu;

// Order-preserving map of f32 bits to u32 (for warp min/max reductions) and
// its inverse.  NaN maps outside [-inf, inf], which makes a box conservative.
__device__ __forceinline__ uint32_t ord_f32(float x) {
  const uint32_t b = __float_as_uint(x);
  return b ^ ((uint32_t)((int32_t)b >> 31) | 0x80000000u);
}
__device__ __forceinline__ float unord_f32(uint32_t u) {
  return __uint_as_float(u ^ (((u >> 31) - 1u) | 0x80000000u));
}

// Bounding box of the valid lanes' points (all lanes call it).
struct Box3 {
  float lo[3], hi[3];
};
__device__ __forceinline__ Box3 warp_box(float x, float y, float z, bool valid) {
  const float v[3] = {x, y, z};
  Box3 b;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const uint32_t u = ord_f32(v[k]);
    b.lo[k] = unord_f32(__reduce_min_sync(0xffffffffu, valid ? u : 0xffffffffu));
    b.hi[k] = unord_f32(__reduce_max_sync(0xffffffffu, valid ? u : 0u));
  }
  return b;
}

// True when every point of box c (offset by off) is at least sqrt(hc2) from
// every point of box q.  The gaps use the operations of the pair distance
// (f32 subtraction of offset coordinates, fma sum of squares), which round
// monotonically, so a skipped chunk holds no pair with r^2 < hc2; a NaN
// bound never skips.
__device__ __forceinline__ bool boxes_apart(const Box3& q, const Box3& c, const float off[3], float hc2) {
  float g[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float a = (c.lo[k] + off[k]) - q.hi[k];
    const float b = q.lo[k] - (c.hi[k] + off[k]);
    g[k] = fmaxf(fmaxf(a, b), 0.f);
  }
  const float d2 = fmaf(g[2], g[2], fmaf(g[1], g[1], g[0] * g[0]));
  return d2 >= hc2 * 1.0001f;
}

struct CellGeom {
  int ax, ay, az;  // box coordinates
  int sc;
};

template <int TB>
__device__ __forceinline__ CellGeom cell_geom(const StepConsts& c, const TiledArgs& a, uint32_t cell) {
  using T = Tile<TB>;
  CellGeom g;
  g.sc = a.scene ? (int)a.scene[a.cell_start[cell]] : 0;
  const SceneBox& bx = c.boxes[g.sc];
  const uint32_t rel = cell - (uint32_t)bx.cell_base;
  const int t = (int)(rel >> (3 * T::L));
  const int u = (int)(rel & ((1u << (3 * T::L)) - 1u));
  const int tz = t % bx.nt[2], ty = (t / bx.nt[2]) % bx.nt[1], tx = t / (bx.nt[2] * bx.nt[1]);
  g.ax = tx * T::B + (u >> (2 * T::L));
  g.ay = ty * T::B + ((u >> T::L) & (T::B - 1));
  g.az = tz * T::B + (u & (T::B - 1));
  return g;
}

// The warp's task: slots [q0, q0 + qn) of `cell`, its box geometry, and the
// 27 neighbour ranges held by lanes 0..26 (empty when the neighbour cell's
// box is out of reach of the queries' box).
struct DenseTask {
  uint32_t k;  // task index
  uint32_t q0, qn;
  CellGeom cg;
  uint32_t nb_s, nb_e;  // this lane's neighbour range (lane < 27)
};

template <int TB>
__device__ __forceinline__ bool next_task(const StepConsts& c, const TiledArgs& a, uint32_t* counter,
                                          uint32_t ntasks, DenseTask& t) {
  const int lane = threadIdx.x & 31;
  uint32_t k = 0;
  if (lane == 0) k = atomicAdd(counter, 1u);
  k = __shfl_sync(0xffffffffu, k, 0);
  if (k >= ntasks) return false;
  t.k = k;
  t.q0 = a.dense_q0[k];
  const uint32_t cell = a.sorted_cell[t.q0];
  t.qn = min(32u, a.cell_start[cell + 1] - t.q0);
  t.cg = cell_geom<TB>(c, a, cell);
  return true;
}

// Neighbour ranges of the task (lane nb < 27 holds neighbour nb), with
// whole cells out of reach of the query box emptied.
template <int TB>
__device__ __forceinline__ void task_neighbours(const StepConsts& c, const TiledArgs& a, DenseTask& t,
                                                const Box3& qb, float hc2) {
  const int nb = threadIdx.x & 31;
  t.nb_s = t.nb_e = 0;
  if (nb < 27) {
    const SceneBox& bx = c.boxes[t.cg.sc];
    const int dx = nb / 9 - 1, dy = (nb / 3) % 3 - 1, dz = nb % 3 - 1;
    const int lin = box_tiled_index(c, bx, t.cg.ax + dx, t.cg.ay + dy, t.cg.az + dz);
    uint32_t s0, e0;
    cell_range<TB>(a, (uint32_t)lin, s0, e0);
    // The neighbour cell's box in query-cell coordinates, widened by 1e-3 h0
    // for cell-local coordinates rounded just outside [0, h0].
    const float m = 1e-3f * c.h0f;
    Box3 cb;
    const float o[3] = {(float)dx * c.h0f, (float)dy * c.h0f, (float)dz * c.h0f};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      cb.lo[k] = -m;
      cb.hi[k] = c.h0f + m;
    }
    if (!boxes_apart(qb, cb, o, hc2)) {
      t.nb_s = s0;
      t.nb_e = e0;
    }
  }
}

__device__ __forceinline__ void neighbour_offset(const StepConsts& c, int nb, float off[3]) {
  off[0] = (float)(nb / 9 - 1) * c.h0f;
  off[1] = (float)((nb / 3) % 3 - 1) * c.h0f;
  off[2] = (float)(nb % 3 - 1) * c.h0f;
}

// Density of the dense-cell particles: per query the compensated sum of
// m_j poly6(r) over the 27 cells (world.rs:219-238), candidates in pairs on
// f32x2 arithmetic (the filter of the tiled pass without the list).
template <int TB, bool kCount, bool kExact>
__global__ void __launch_bounds__(kWT, 4) k_density_dense(StepConsts c, TiledArgs a) {
  __shared__ __align__(16) float s_pp[kWarps][32 * 4];  // 32 candidates, pair-interleaved
  const int lane = threadIdx.x & 31;
  float* sp = s_pp[threadIdx.x >> 5];
  const float4* sp4 = reinterpret_cast<const float4*>(sp);
  const uint32_t ntasks = *a.dense_count;
  const float hc2 = fminf(c.h2f, c.h0sqf);
  const f2 HC2 = f2_pack(hc2, hc2), H0SQ = f2_pack(c.h0sqf, c.h0sqf);
  unsigned cand = 0, pairs = 0;
  DenseTask t;
  while (next_task<TB>(c, a, a.dense_taken, ntasks, t)) {
    const bool qv = (uint32_t)lane < t.qn;
    const uint32_t qi = t.q0 + (uint32_t)lane;
    const float4 q = qv ? a.cpos[qi] : make_float4(kFar, kFar, kFar, 0.f);
    const Box3 qb = warp_box(q.x, q.y, q.z, qv);
    task_neighbours<TB>(c, a, t, qb, hc2);
    const f2 PX = f2_pack(q.x, q.x), PY = f2_pack(q.y, q.y), PZ = f2_pack(q.z, q.z);
    // Mask entries: reserve the task's upper bound (one entry per chunk of
    // every neighbour cell in reach).
    uint32_t mbase = kNoMasks, mcount = 0;
    if (a.mask_ctl) {
      const uint32_t bound = __reduce_add_sync(0xffffffffu, (t.nb_e - t.nb_s + 31u) >> 5);
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(a.mask_ctl, (unsigned long long)bound);
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base + bound <= a.mask_cap) mbase = (uint32_t)base;
    }
    float s = 0.f, comp = 0.f;
    for (int nb = 0; nb < 27; ++nb) {
      const uint32_t s0 = __shfl_sync(0xffffffffu, t.nb_s, nb), e0 = __shfl_sync(0xffffffffu, t.nb_e, nb);
      if (s0 >= e0) continue;
      float off[3];
      neighbour_offset(c, nb, off);
      for (uint32_t cb = s0; cb < e0; cb += 32) {
        const uint32_t j = cb + (uint32_t)lane;
        const bool cv = j < e0;
        float4 p = cv ? a.cpos[j] : make_float4(kFar, kFar, kFar, 0.f);
        const Box3 bb = warp_box(p.x, p.y, p.z, cv);
        if (boxes_apart(qb, bb, off, hc2)) continue;  // uniform
        p.x += off[0];
        p.y += off[1];
        p.z += off[2];
        put_pair_slot(sp, (uint32_t)lane, p);
        __syncwarp();
        const uint32_t m = min(32u, e0 - cb);
        if (kCount && qv) cand += m;
        f2 NPART = f2_pack(0.f, 0.f);
        // In-range bits as the force pass forms them (the sign of r^2 - hc2),
        // the chunk's first candidate shifted in first.
        uint32_t mask = 0;
#pragma unroll 4
        for (uint32_t k = 0; k < 32u; k += 2) {
          if (k >= m) break;  // uniform; slot m of an odd m holds a far dummy
          const float4 A = sp4[k];      // x0 x1 y0 y1
          const float4 B = sp4[k + 1];  // z0 z1 m0 m1
          const f2 DX = f2_sub(f2_pack(A.x, A.y), PX);
          const f2 DY = f2_sub(f2_pack(A.z, A.w), PY);
          const f2 DZ = f2_sub(f2_pack(B.x, B.y), PZ);
          const f2 R2 = f2_fma(DZ, DZ, f2_fma(DY, DY, f2_mul(DX, DX)));
          float d0, d1, n0, n1;
          f2_unpack(f2_sub(R2, HC2), d0, d1);
          if (kExact) {
            n0 = fminf(d0, 0.f);
            n1 = fminf(d1, 0.f);
          } else {
            float e0_, e1_;
            f2_unpack(f2_sub(R2, H0SQ), e0_, e1_);
            n0 = d0 < 0.f ? e0_ : 0.f;
            n1 = d1 < 0.f ? e1_ : 0.f;
          }
          if (kCount) pairs += (qv && d0 < 0.f ? 1u : 0u) + (qv && d1 < 0.f && k + 1 < m ? 1u : 0u);
          mask = __funnelshift_l(__float_as_uint(d0), mask, 1);
          mask = __funnelshift_l(__float_as_uint(d1), mask, 1);
          const f2 N = f2_pack(n0, n1);
          NPART = f2_fma(f2_mul(N, N), f2_mul(N, f2_pack(B.z, B.w)), NPART);
        }
        float p0, p1;
        f2_unpack(NPART, p0, p1);
        kahan_add(s, comp, c.poly6_cf * -(p0 + p1));
        if (mbase != kNoMasks) {
          // 2 ceil(m / 2) bits were shifted in (at least 2); bit k = candidate k.
          const uint32_t used = (m + 1u) & ~1u;
          const uint32_t bits = qv ? __brev(used < 32u ? mask << (32u - used) : mask) : 0u;
          if (__any_sync(0xffffffffu, bits != 0u)) {
            a.mask_bits[(size_t)(mbase + mcount) * 32u + (uint32_t)lane] = bits;
            if (lane == 0) a.mask_hdr[mbase + mcount] = (cb << 5) | (uint32_t)nb;
            ++mcount;
          }
        }
        __syncwarp();  // the chunk is consumed before the next one is staged
      }
    }
    if (qv) {
      write_density(c, a, (int)qi, (double)s - (double)comp);
      a.nbr_count[qi] = kNoList;
    }
    if (a.mask_ctl && lane == 0) {
      a.task_mbase[t.k] = mbase;
      a.task_mcount[t.k] = mcount;
    }
  }
  if (kCount) {
    const unsigned wc = __reduce_add_sync(0xffffffffu, cand);
    const unsigned wp = __reduce_add_sync(0xffffffffu, pairs);
    if (lane == 0) {
      atomicAdd(&a.counters[0], (unsigned long long)wc);
      atomicAdd(&a.counters[1], (unsigned long long)wp);
    }
  }
}

// Forces, integration and bounds of the dense-cell particles: per chunk each
// lane has the mask of its in-range candidates (kept by the density pass, or
// built here branch-free, candidates in pairs on f32x2 arithmetic), then the
// warp walks the masks in lockstep for as many rounds as the fullest mask has
// bits, each lane taking its own next candidate through the pair terms of the
// tiled pass.  The partial sums are folded into the compensated totals every
// 16 rounds (every 8 with the shear sum, one candidate per round) and at the
// end of the chunk, uniformly across the warp.
template <int TB, bool kShear>
__global__ void __launch_bounds__(kWT, 2) k_force_dense(StepConsts c, TiledArgs a) {
  // The chunk's 32 candidates, and in slot 32 a weightless copy of its first
  // (mass and m/rho 0) that pads the two-candidate rounds.
  __shared__ float4 s_pos[kWarps][33];
  __shared__ float4 s_vel[kWarps][33];
  __shared__ float s_mr[kWarps][33];
  __shared__ __align__(16) float s_pp[kWarps][32 * 4];  // the chunk's positions, pair-interleaved
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  float* sp = s_pp[w];
  const float4* sp4 = reinterpret_cast<const float4*>(sp);
  const uint32_t ntasks = *a.dense_count;
  const float hc2 = fminf(c.h2f, c.h0sqf);
  const f2 HC2 = f2_pack(hc2, hc2);
  DenseTask t;
  while (next_task<TB>(c, a, a.dense_taken + 1, ntasks, t)) {
    const bool qv = (uint32_t)lane < t.qn;
    const uint32_t qi = t.q0 + (uint32_t)lane;
    const float4 qp = qv ? a.cpos[qi] : make_float4(kFar, kFar, kFar, 0.f);
    const float4 qvel = qv ? a.cvel[qi] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float lapm = qp.w * c.lap_cf;
    const QueryPack Q = query_pack(c, qp, qvel, lapm);
    CompAcc acc;
    ForcePart part;
    ForcePart2 part2;
    zero(part2);
    // Stages this lane's candidate (offset position p, velocity, m/rho) in
    // its slot; lane 0 also fills the padding slot 32.
    auto stage = [&](float4 p, float4 v, float mr) {
      s_pos[w][lane] = p;
      s_vel[w][lane] = v;
      s_mr[w][lane] = mr;
      if (lane == 0) {
        s_pos[w][32] = make_float4(p.x, p.y, p.z, 0.f);
        s_vel[w][32] = v;
        s_mr[w][32] = 0.f;
      }
    };
    // The walk of one staged chunk given this lane's in-range bits (bit k =
    // candidate k; zero for a lane without a query).
    auto walk = [&](uint32_t mask) {
      if (!kShear) {
        // Two candidates per round; a lane out of candidates takes the
        // weightless padding slot.
        const int rounds = (int)(__reduce_max_sync(0xffffffffu, (unsigned)__popc(mask)) + 1) >> 1;
        for (int r = 0; r < rounds; ++r) {
          const int ka = mask != 0 ? __ffs(mask) - 1 : 32;
          mask &= mask - 1;
          const int kb = mask != 0 ? __ffs(mask) - 1 : 32;
          mask &= mask - 1;
          pair2_listed(Q, s_pos[w][ka], s_vel[w][ka], s_mr[w][ka], s_pos[w][kb], s_vel[w][kb], s_mr[w][kb],
                       part2);
          if ((r & 15) == 15) fold2(acc, part2);
        }
        if (rounds & 15) fold2(acc, part2);
      } else {
        const int rounds = __reduce_max_sync(0xffffffffu, (unsigned)__popc(mask));
        for (int r = 0; r < rounds; ++r) {
          if (mask) {
            const int k = __ffs(mask) - 1;
            mask &= mask - 1;
            pair_listed<kShear>(c, s_pos[w][k], s_vel[w][k], s_mr[w][k], qp, qvel, lapm, part, acc);
          }
          if ((r & 7) == 7) fold<kShear>(acc, part, qp.w * c.spiky_cf, lapm);
        }
        if (rounds & 7) fold<kShear>(acc, part, qp.w * c.spiky_cf, lapm);
      }
    };
    uint32_t mbase = a.task_mbase ? a.task_mbase[t.k] : kNoMasks;
    const uint32_t mcount = mbase != kNoMasks ? a.task_mcount[t.k] : 0u;
    if (mbase != kNoMasks && ((unsigned long long)mbase + mcount > a.mask_cap || mcount > (1u << 20))) {
      if (lane == 0) atomicOr(a.flags, kFlagMaskTable);
      mbase = kNoMasks;
    }
    if (mbase != kNoMasks) {
      // The density pass's chunks, in its order; the next entry's header and
      // mask are loaded while the current chunk is walked.
      uint32_t hdr = 0, bits = 0;
      if (mcount) {
        hdr = a.mask_hdr[mbase];
        bits = a.mask_bits[(size_t)mbase * 32u + (uint32_t)lane];
      }
      for (uint32_t e = 0; e < mcount; ++e) {
        const uint32_t h = hdr, mask = bits;
        if (e + 1 < mcount) {
          hdr = a.mask_hdr[mbase + e + 1];
          bits = a.mask_bits[(size_t)(mbase + e + 1) * 32u + (uint32_t)lane];
        }
        // Only candidates some lane has in range are loaded, and the chunk's
        // first (always a particle), which pads the two-candidate rounds as in
        // the filtering walk; the other slots hold far dummies, never walked.
        const uint32_t any = __reduce_or_sync(0xffffffffu, mask);  // every lane takes part
        const bool cv = lane == 0 || ((any >> lane) & 1u) != 0u;
        const uint32_t j = (h >> 5) + (uint32_t)lane;
        float off[3];
        neighbour_offset(c, (int)(h & 31u), off);
        float4 p = cv ? a.cpos[j] : make_float4(kFar, kFar, kFar, 0.f);
        p.x += off[0];
        p.y += off[1];
        p.z += off[2];
        stage(p, cv ? a.cvel[j] : make_float4(0.f, 0.f, 0.f, 0.f), cv ? a.cmr[j] : 0.f);
        __syncwarp();
        walk(mask);
        __syncwarp();  // the chunk is consumed before the next one is staged
      }
    } else {
      const Box3 qb = warp_box(qp.x, qp.y, qp.z, qv);
      task_neighbours<TB>(c, a, t, qb, hc2);
      for (int nb = 0; nb < 27; ++nb) {
        const uint32_t s0 = __shfl_sync(0xffffffffu, t.nb_s, nb), e0 = __shfl_sync(0xffffffffu, t.nb_e, nb);
        if (s0 >= e0) continue;
        float off[3];
        neighbour_offset(c, nb, off);
        for (uint32_t cb = s0; cb < e0; cb += 32) {
          const uint32_t j = cb + (uint32_t)lane;
          const bool cv = j < e0;
          float4 p = cv ? a.cpos[j] : make_float4(kFar, kFar, kFar, 0.f);
          const Box3 bb = warp_box(p.x, p.y, p.z, cv);
          if (boxes_apart(qb, bb, off, hc2)) continue;  // uniform
          p.x += off[0];
          p.y += off[1];
          p.z += off[2];
          stage(p, cv ? a.cvel[j] : make_float4(0.f, 0.f, 0.f, 0.f), cv ? a.cmr[j] : 0.f);
          put_pair_slot(sp, (uint32_t)lane, p);
          __syncwarp();
          // In-range bits (r^2 < hc2; the sign of r^2 - hc2, which is never
          // -0), shifted in so that the chunk's first candidate ends in the
          // highest bit; slots past the chunk hold far dummies (bit 0).
          uint32_t mask = 0;
#pragma unroll
          for (uint32_t k = 0; k < 32u; k += 2) {
            const float4 A = sp4[k];      // x0 x1 y0 y1
            const float4 B = sp4[k + 1];  // z0 z1 m0 m1
            const f2 DX = f2_sub(f2_pack(A.x, A.y), Q.px);
            const f2 DY = f2_sub(f2_pack(A.z, A.w), Q.py);
            const f2 DZ = f2_sub(f2_pack(B.x, B.y), Q.pz);
            const f2 R2 = f2_fma(DZ, DZ, f2_fma(DY, DY, f2_mul(DX, DX)));
            float d0, d1;
            f2_unpack(f2_sub(R2, HC2), d0, d1);
            mask = __funnelshift_l(__float_as_uint(d0), mask, 1);
            mask = __funnelshift_l(__float_as_uint(d1), mask, 1);
          }
          walk(qv ? __brev(mask) : 0u);
          __syncwarp();  // the chunk is consumed before the next one is staged
        }
      }
    }
    if (qv) finish_particle(c, a, (int)qi, acc, c.boxes[t.cg.sc]);
  }
}

constexpr size_t kDensitySmem = kHaloCap * sizeof(float4) + (3 * kNHMax + 1 + 32) * 4;
constexpr size_t kForceSmem = kHaloCap * (2 * sizeof(float4) + sizeof(float)) + (3 * kNHMax + 1 + 32) * 4;

// Resident CTAs per SM of the persistent passes (occupancy limits, computed
// once; the shared-memory opt-in is set on the same first call).
struct Occupancy {
  int sms = 1, density = 1, force = 1, dense_density = 1, dense_force = 1;
};

template <int TB>
void set_smem_limits() {
  for (auto f : {k_density_tiled<TB, false, true>, k_density_tiled<TB, true, true>, k_density_tiled<TB, false, false>,
                 k_density_tiled<TB, true, false>})
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDensitySmem);
  for (auto f : {k_force_tiled<TB, false>, k_force_tiled<TB, true>})
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kForceSmem);
}

const Occupancy& occupancy() {
  static const Occupancy o = [] {
    Occupancy r;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&r.sms, cudaDevAttrMultiProcessorCount, dev);
    set_smem_limits<4>();
    set_smem_limits<2>();
    // Both tile edges use the same shared memory and registers per CTA.
    int bd = 0, bf = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bd, k_density_tiled<4, false, true>, kTT, kDensitySmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bf, k_force_tiled<4, true>, kTT, kForceSmem);
    int dd = 0, df = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&dd, k_density_dense<4, false, true>, kWT, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&df, k_force_dense<4, true>, kWT, 0);
    r.dense_density = std::max(dd, 1);
    r.dense_force = std::max(df, 1);
    r.sms = std::max(r.sms, 1);
    r.density = std::max(bd, 1);
    r.force = std::max(bf, 1);
    return r;
  }();
  return o;
}

// The four passes of a tiled step (staged and dense-cell density, staged and
// dense-cell force) for tile edge TB.
template <int TB>
void launch_passes(const StepConsts& c, const TiledArgs& a, cudaStream_t s, const PassEvents& ev, bool exact,
                   int density_blocks, int force_blocks, int dense_d_blocks, int dense_f_blocks) {
  auto density = a.counters ? (exact ? k_density_tiled<TB, true, true> : k_density_tiled<TB, true, false>)
                            : (exact ? k_density_tiled<TB, false, true> : k_density_tiled<TB, false, false>);
  density<<<density_blocks, kTT, kDensitySmem, s>>>(c, a);
  auto dense = a.counters ? (exact ? k_density_dense<TB, true, true> : k_density_dense<TB, true, false>)
                          : (exact ? k_density_dense<TB, false, true> : k_density_dense<TB, false, false>);
  dense<<<dense_d_blocks, kWT, 0, s>>>(c, a);
  if (ev.after_density) cudaEventRecord(ev.after_density, s);
  if (c.shear_live) {
    k_force_tiled<TB, true><<<force_blocks, kTT, kForceSmem, s>>>(c, a);
    k_force_dense<TB, true><<<dense_f_blocks, kWT, 0, s>>>(c, a);
  } else {
    k_force_tiled<TB, false><<<force_blocks, kTT, kForceSmem, s>>>(c, a);
    k_force_dense<TB, false><<<dense_f_blocks, kWT, 0, s>>>(c, a);
  }
}

}  // namespace

int tiled_max_ctas_per_sm() {
  const Occupancy& o = occupancy();
  return std::max(o.density, o.force);
}

void launch_comp_tiled(const StepConsts& c, DevBuffers& b, cudaStream_t s, const PassEvents& ev,
                       const LaunchTuning& t) {
  const ParticleConsts& pc = b.pc[b.cur];
  TiledArgs a;
  a.px = b.pv0[0];
  a.py = b.pv0[1];
  a.pz = b.pv0[2];
  a.vx = b.pv0[3];
  a.vy = b.pv0[4];
  a.vz = b.pv0[5];
  a.mass = pc.mass;
  a.mat = pc.mat;
  a.cell_start = b.cell_start;
  a.tile_start = b.tile_head;
  a.sorted_cell = b.sorted_cell;
  a.tile_slot = b.tile_slot;
  a.tile_crowd = b.tile_crowd;
  a.num_tiles = b.num_tiles;
  a.cpos = b.cpos;
  a.cvel = b.cvel;
  a.cmr = b.cmr;
  a.bax = b.has_ba ? pc.ba[0] : nullptr;
  a.bay = b.has_ba ? pc.ba[1] : nullptr;
  a.baz = b.has_ba ? pc.ba[2] : nullptr;
  a.rho = b.rho;
  a.p = b.p;
  for (int k = 0; k < 3; ++k) {
    a.acc[k] = b.acc[k];
    a.xsph[k] = b.xsph[k];
  }
  a.mu = b.mu;
  for (int k = 0; k < 6; ++k) a.out_pv[k] = b.pv1[k];
  a.nbr16 = b.nbr16;
  a.nbr_count = b.nbr_count;
  a.scene = pc.scene;
  a.queue = t.queue ? b.queue : nullptr;
  a.dense_count = b.queue + 2;
  a.dense_taken = b.queue + 3;
  a.dense_q0 = b.dense_q0;
  const bool masks = t.dense_masks && b.mask_ctl != nullptr;
  a.task_mbase = masks ? b.task_mbase : nullptr;
  a.task_mcount = b.task_mcount;
  a.mask_hdr = b.mask_hdr;
  a.mask_bits = b.mask_bits;
  a.mask_ctl = masks ? b.mask_ctl : nullptr;
  a.mask_cap = b.mask_cap;
  a.stride = b.capacity;
  a.flags = b.flags;
  a.counters = b.counters;
  // Persistent grids: SM count x resident CTAs per SM (the occupancy limit,
  // or the tuned count when smaller).
  const Occupancy& o = occupancy();
  const int per_sm = t.ctas_per_sm;
  const int density_blocks = o.sms * (per_sm > 0 ? std::min(per_sm, o.density) : o.density);
  const int force_blocks = o.sms * (per_sm > 0 ? std::min(per_sm, o.force) : o.force);
  // The f32 operands (cpos, cvel) and the work-queue reset come from the
  // sort's gather; the "prep" phase of a tiled step is empty.
  if (ev.after_prep) cudaEventRecord(ev.after_prep, s);
  const int dense_d_blocks = o.sms * o.dense_density, dense_f_blocks = o.sms * o.dense_force;
  const bool exact = std::min(c.h2f, c.h0sqf) == c.h0sqf;
  if (masks) cudaMemsetAsync(b.mask_ctl, 0, sizeof(unsigned long long), s);
  if (c.tile == 2)
    launch_passes<2>(c, a, s, ev, exact, density_blocks, force_blocks, dense_d_blocks, dense_f_blocks);
  else
    launch_passes<4>(c, a, s, ev, exact, density_blocks, force_blocks, dense_d_blocks, dense_f_blocks);
  // The entries this step's tasks asked for, for the host's next sizing.
  if (masks && b.mask_demand)
    cudaMemcpyAsync(b.mask_demand, b.mask_ctl, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
}

}  // namespace phy
