// Shared definitions of the B200 SPH fluid step.
//
// Device layout (one fluid subsystem):
//   * particles live in structure-of-arrays form, sorted by (grid cell,
//     insertion index) at the start of every step; `id` maps a sorted slot
//     back to the insertion index the reference's `particles` Vec uses;
//   * the neighbour grid is a dense box of cells of edge h0 (the smoothing
//     length captured at construction, crates/phy-fluid/src/sph/world.rs:
//     94-102), linearised x-major / z-minor so that the 27-cell visit order of
//     Grid::for_each_neighbor (grid.rs:43-56: di outer, dk inner) becomes nine
//     contiguous runs of three cells in the sorted arrays;
//   * cell_start[c] .. cell_start[c+1] is the slot range of cell c.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace phy {

constexpr int kMaxMaterials = 16;
// Neighbour-list capacity per particle (in-range pairs: ~31 at rest density
// with spacing h/2, ~60 at twice the rest density, which the bottom of a
// tall column reaches with the default stiffness).
constexpr int kMaxNeighbors = 96;
// f32-compensated lists pack the 27-cell offset code under the index.
constexpr int kCodeBits = 5;
// The first kStagedNeighbors entries of a list are staged in shared memory
// and written out coalesced; further entries go straight to global memory.
constexpr int kStagedNeighbors = 40;

// Tiled form: by default a tile whose occupied cells hold more than this many
// particles on average goes to the dense-cell passes even when its halo could
// be staged (StepConsts::dense_mean, a tuning knob); from about this density
// on, neighbour lists overflow and a staged tile would rescan its cells for
// every query.
constexpr uint32_t kDenseMean = 32;

// Error bits written by device code into the per-world flag word.
enum : uint32_t {
  kFlagOutOfBox = 1u,    // a cell key fell outside the grid box
  kFlagNonFinite = 2u,   // a new position or velocity is NaN/Inf
  kFlagMaskTable = 4u,   // a dense-cell task's kept masks lie outside the mask buffer (filtered again)
};

// The grid box and wall bounds of one scene in the tiled linearisation.  A
// batch of independent scenes gives every scene its own box; the boxes'
// cells are numbered consecutively (cell_base, a multiple of the tile size),
// so one sort and one persistent pass cover all scenes, which never interact.
struct SceneBox {
  long long b0[3];   // key of the box's first cell per axis
  int nc[3];         // cells per axis (multiples of the tile edge)
  int nt[3];         // tiles per axis
  int cell_base;     // first global cell index of the box
  double lo[3], hi[3];  // bounds_min / bounds_max of the scene
};

// Everything a step kernel needs, passed by value (kernel parameter space).
struct StepConsts {
  // Captured at construction from the initial h (kernels.rs:22-35, grid.rs:27).
  double h0, h0sq, poly6_c, spiky_c, lap_c, inv_cell;
  // Live SphParams (read every step, world.rs:205, 258).
  double h, r2_guard, rest, stiff, shear_min, damp, xsph_eps, dt;
  double g[3], lo[3], hi[3];
  int n_visc_k;
  int n;
  double visc_k[kMaxMaterials], visc_n[kMaxMaterials];
  // 0 when visc_n[m] == 1 for every reachable material m < n_visc_k: then
  // mu = visc_k[m] * max(shear, shear_min)^0 = visc_k[m] exactly
  // (world.rs:319-327) and the shear sum is never observed, so the force
  // passes skip it (the same bits either way).
  int shear_live;
  // Grid box: key of cell 0 and dimensions (cells per axis).
  long long bx0, by0, bz0;
  int ncx, ncy, ncz;
  int ncells;
  // Cell linearisation: tile == 0 is x-major / z-minor over the box (the
  // reference's 27-cell order becomes 9 runs of 3 cells); tile == B (a power
  // of two) orders B^3-cell tiles x-major and the cells inside a tile
  // x-major, so a tile's particles are contiguous (ncx, ncy, ncz are then
  // multiples of B and ntx, nty, ntz count tiles).
  int tile, tile_log2;
  int ntx, nty, ntz;
  // Tiles whose halo holds more particles than this are computed from
  // global memory instead of shared memory (<= the kernels' capacity).
  int halo_cap;
  // Tiles whose occupied cells average more particles than this go to the
  // dense-cell passes.
  int dense_mean;
  // Tiled form: device table of the scene boxes (one entry for a single
  // world).  A particle's scene is its entry in ParticleConsts::scene (all 0
  // when that array is absent); ncells counts the cells of all boxes.
  const SceneBox* boxes;
  int n_scenes;
  // f32 copies for the compensated form.
  float h0f, h0sqf, poly6_cf, spiky_cf, lap_cf, hf, h2f;
};

#if defined(__CUDACC__)

// num-traits ToPrimitive::to_i64 on f64 (Some only inside (-2^63, 2^63)),
// with None mapped to 0 as in Grid::key_of (grid.rs:25-33).
__device__ __forceinline__ long long key_axis(double x, double inv) {
  double f = floor(__dmul_rn(x, inv));
  if (f > -9223372036854775808.0 && f < 9223372036854775808.0) return (long long)f;
  return 0;
}

// Linear cell index of integer key (i,j,k), or -1 when outside the box.
__device__ __forceinline__ int cell_linear(const StepConsts& c, long long i, long long j, long long k) {
  long long a = i - c.bx0, b = j - c.by0, d = k - c.bz0;
  if (a < 0 || b < 0 || d < 0 || a >= c.ncx || b >= c.ncy || d >= c.ncz) return -1;
  return (int)((a * c.ncy + b) * c.ncz + d);
}

// Tiled linear index of box coordinates (a, b, d), all inside the box.
__device__ __forceinline__ int tiled_index(const StepConsts& c, int a, int b, int d) {
  const int L = c.tile_log2, m = c.tile - 1;
  const int tile = ((a >> L) * c.nty + (b >> L)) * c.ntz + (d >> L);
  return (tile << (3 * L)) + ((((a & m) << L) + (b & m)) << L) + (d & m);
}

// Sort cell of integer key (i,j,k) under the configured linearisation, or -1
// when outside the box.
__device__ __forceinline__ int cell_index(const StepConsts& c, long long i, long long j, long long k) {
  if (c.tile == 0) return cell_linear(c, i, j, k);
  long long a = i - c.bx0, b = j - c.by0, d = k - c.bz0;
  if (a < 0 || b < 0 || d < 0 || a >= c.ncx || b >= c.ncy || d >= c.ncz) return -1;
  return tiled_index(c, (int)a, (int)b, (int)d);
}

// A particle's own cell is an "interior" cell when its 27 neighbours are all
// inside the box; the host pads the box by one cell on every side so that
// every in-box particle qualifies.
__device__ __forceinline__ bool cell_interior(const StepConsts& c, long long i, long long j, long long k) {
  long long a = i - c.bx0, b = j - c.by0, d = k - c.bz0;
  return a >= 1 && b >= 1 && d >= 1 && a < c.ncx - 1 && b < c.ncy - 1 && d < c.ncz - 1;
}

// Global tiled cell index of box coordinates (a, b, d) inside box `bx`.
__device__ __forceinline__ int box_tiled_index(const StepConsts& c, const SceneBox& bx, int a, int b, int d) {
  const int L = c.tile_log2, m = c.tile - 1;
  const int tile = ((a >> L) * bx.nt[1] + (b >> L)) * bx.nt[2] + (d >> L);
  return bx.cell_base + (tile << (3 * L)) + ((((a & m) << L) + (b & m)) << L) + (d & m);
}

// visc_k[m], visc_n[m] by unrolled selection: a dynamic index into the
// kernel-parameter arrays would force a local-memory copy of them.
__device__ __forceinline__ void material_coeffs(const StepConsts& c, int m, double& k, double& n) {
  k = c.visc_k[0];
  n = c.visc_n[0];
#pragma unroll
  for (int q = 1; q < kMaxMaterials; ++q) {
    if (q == m) {
      k = c.visc_k[q];
      n = c.visc_n[q];
    }
  }
}

// Writes the staged part of each thread's neighbour list (column-major in
// shared memory, bank = thread) to its global column-major list: at step k
// the 32 lanes of a warp store 32 consecutive words.
template <int kBlock>
__device__ __forceinline__ void flush_staged_list(const uint32_t (*s_list)[kBlock], uint32_t* lst, int stride,
                                                  uint32_t cnt, bool active) {
  const unsigned am = __activemask();
  const uint32_t mine = active ? (cnt < (uint32_t)kStagedNeighbors ? cnt : (uint32_t)kStagedNeighbors) : 0u;
  const uint32_t kmax = __reduce_max_sync(am, mine);
  for (uint32_t k = 0; k < kmax; ++k)
    if (k < mine) lst[(size_t)k * stride] = s_list[k][threadIdx.x];
}

#endif  // __CUDACC__

}  // namespace phy
