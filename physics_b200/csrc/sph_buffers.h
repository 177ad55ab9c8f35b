// Device buffers of one fluid subsystem and the host-side launchers.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "phy_fluid.h"
#include "sph_common.cuh"

namespace phy {

// Per-particle constants carried through the sort (double-buffered: the sort
// gathers set `cur` into set `cur ^ 1`).
struct ParticleConsts {
  double* mass = nullptr;
  uint32_t* mat = nullptr;
  uint32_t* id = nullptr;   // insertion index
  double* ba[3] = {nullptr, nullptr, nullptr};  // body_acc, optional
  uint16_t* scene = nullptr;  // scene of a batched world, optional
};

struct DevBuffers {
  int capacity = 0;        // particles
  int cell_capacity = 0;   // grid cells (excluding the overflow cell)
  // Positions/velocities.  pv0: sorted state read by the passes.
  // pv1: output of the force pass (same order as pv0) and upload target.
  double* pv0[6] = {};
  double* pv1[6] = {};
  ParticleConsts pc[2];
  int cur = 0;
  bool has_ba = false;
  // Step outputs, sorted order.
  double* rho = nullptr;
  double* p = nullptr;
  double* pr2 = nullptr;   // p / (rho*rho)
  double* mr = nullptr;    // mass / rho
  double* acc[3] = {};
  double* xsph[3] = {};
  double* mu = nullptr;
  // f32-compensated form: per-particle packed operands.
  float4* cpos = nullptr;  // cell-local x, y, z (f32) and mass
  float4* cvel = nullptr;  // vx, vy, vz (f32) and p/rho^2 (f32)
  float* cmr = nullptr;    // mass/rho (f32)
  // Neighbour lists written by the density pass and read by the force pass:
  // entry k of particle i at nbr[k * capacity + i] (column-major, so a warp's
  // k-th entries are contiguous); nbr_count[i] may exceed kMaxNeighbors, in
  // which case the force pass rescans the 27 cells for that particle.
  uint32_t* nbr = nullptr;
  uint32_t* nbr_count = nullptr;
  // Tiled form: 16-bit neighbour slots (shared-memory staging order of the
  // tile's halo), row-major: the kMaxNeighbors entries of sorted slot i at
  // nbr16[i * kMaxNeighbors ..].
  uint16_t* nbr16 = nullptr;
  // Tiled sort: cell of each sorted slot (before the gather: the particles
  // grouped by cell), particles per tile scanned to tile starts (tile_head)
  // over the cell box's tiles plus the overflow bucket (tile_scan_entries);
  // the tile of every list entry, the first slot of every occupied tile
  // (+ end), and the device-side tile count.
  uint32_t* sorted_cell = nullptr;
  uint32_t* tile_head = nullptr;
  size_t tile_scan_entries = 0;
  uint32_t* tile_of = nullptr;
  uint32_t* tile_slot = nullptr;
  uint32_t* large_cells = nullptr;  // cells of more than kOrderSmall particles (capacity / 64 + 64)
  uint8_t* tile_crowd = nullptr;  // 1: tile above kDenseMean per occupied cell
  uint32_t* num_tiles = nullptr;
  // Scene boxes of the tiled linearisation (one entry for a single world),
  // the work counters of the persistent passes ([0] density tiles, [1] force
  // tiles, [2] dense-cell task count, [3] density tasks taken, [4] force tasks
  // taken), and the dense-cell tasks (first slot of up to 32 particles of one
  // cell of a tile too dense to stage).
  SceneBox* boxes = nullptr;
  uint32_t* queue = nullptr;
  uint32_t* dense_q0 = nullptr;
  // In-range masks of the dense-cell density pass, read back by the force
  // pass of the same step instead of filtering again: per task its first
  // entry (kNoMasks: none stored) and entry count; per entry the chunk's
  // first sorted slot << 5 | neighbour cell, and 32 lane masks.  mask_ctl
  // counts the entries the tasks reserved (their upper bounds, stored or
  // not), so the host can grow mask_cap; mask_demand is its pinned host copy.
  uint32_t* task_mbase = nullptr;
  uint32_t* task_mcount = nullptr;
  uint32_t* mask_hdr = nullptr;
  uint32_t* mask_bits = nullptr;
  unsigned long long mask_cap = 0;  // entries
  unsigned long long* mask_ctl = nullptr;
  unsigned long long* mask_demand = nullptr;
  // Sort scratch.
  uint32_t* cell_of = nullptr;
  uint32_t* rank = nullptr;
  uint32_t* tmp = nullptr;
  uint32_t* perm = nullptr;
  // Tiled form: in-cell order key of every particle (Morton code of its
  // quantised position inside the cell, then its insertion index).
  unsigned long long* okey = nullptr;
  uint32_t* cell_start = nullptr;  // cell_capacity + 2 entries
  uint32_t* block_sums = nullptr;
  int block_sums_capacity = 0;
  // Insertion-order staging for uploads and downloads (f64 and u32 views).
  double* stage = nullptr;   // 8 * capacity doubles
  uint32_t* flags = nullptr; // error bits, device
  uint32_t* order_count = nullptr;  // sort: cells of more than kOrderSmall particles (device count)
  unsigned long long* counters = nullptr;  // candidates, pairs (device)
  // Optional outputs of the f64 plain force pass for the adjoint's tape: the
  // raw viscous force and the strain-rate proxy of every sorted slot.
  double* tape_fv[3] = {nullptr, nullptr, nullptr};
  double* tape_shear = nullptr;
};

// grid.cu
void launch_sort(const StepConsts& c, DevBuffers& b, cudaStream_t s, int block = 256);
// The cells of the current positions without moving the state: cell_start
// over the box and perm[s] = the particle at sorted slot s in (cell,
// insertion index) order.  c.tile must be 0 (x-major cells).  The
// out-of-box bit goes to `flags` (not the step's error bits).
void launch_cell_index(const StepConsts& c, DevBuffers& b, uint32_t* flags, cudaStream_t s);

// couple.cu: FluidWorld::couple_points over np points (10 doubles each on the
// device: pos xyz, vel xyz, mass, force xyz) after launch_cell_index; updates
// the fluid velocities in pv1 and the forces of the points inside the bounds.
// Throws CudaError with `what` and the CUDA message unless e is cudaSuccess
// (fluid_world.cu).
void cuda_check(cudaError_t e, const char* what);

// Scratch of couple_points (owned by the world, grown on demand): per-point
// cell tables, candidate counts and offsets, neighbourhood overlaps with the
// points just before, candidate indices and masses.
struct CouplePointsScratch {
  uint32_t* tab = nullptr;
  uint32_t* totals = nullptr;
  uint32_t* off = nullptr;
  uint32_t* idx = nullptr;
  double* m = nullptr;
  uint16_t* conf = nullptr;
  size_t cap_tab = 0, cap_totals = 0, cap_off = 0, cap_idx = 0, cap_m = 0, cap_conf = 0;
  void release();
};
void launch_couple_points(const StepConsts& c, DevBuffers& b, double* d_pts, int np, double dt, double drag,
                          double soft_density, cudaStream_t s, CouplePointsScratch& scratch);

// couple.cu: FluidWorld::couple_heat against a heat grid of nx*ny*nz cells
// (x fastest), origin and cell size.  The scratch arena (size from
// couple_heat_scratch_bytes) starts with the grid's temperatures (cells
// doubles, uploaded by the caller) and sources (cells doubles, in/out); the
// particles' body accelerations (allocated) take the buoyancy terms.
struct HeatGrid {
  uint64_t nx, ny, nz;
  double origin[3];
  double cell;
  double t_ref, beta, heat_gain;
};
size_t couple_heat_scratch_bytes(int n, uint64_t cells);
// couple.cu: FluidWorld::couple_bodies over nb host bodies (PhyCoupleBody,
// include/phy_fluid.h; velocities updated in place) with their vertex /
// height data and face indices; uses `scratch` of couple_bodies_scratch_bytes
// and synchronises the stream.  Returns 0, or -1 on a CUDA error.
struct CoupleBodiesLaunch {
  unsigned char* scratch;
  PhyCoupleBody* bodies;
  int nb;
  const double* data;
  uint64_t n_data;
  const uint32_t* faces;
  uint64_t n_faces;
  double particle_vol;  // params.mass / rest_density (world.rs:424)
};
size_t couple_bodies_scratch_bytes(int n, int nb, uint64_t n_data, uint64_t n_faces);
int launch_couple_bodies(const StepConsts& c, DevBuffers& b, const CoupleBodiesLaunch& l, cudaStream_t s);
void launch_couple_heat(const StepConsts& c, DevBuffers& b, const HeatGrid& g, unsigned char* scratch,
                        cudaStream_t s);
void launch_unsort_f64(const DevBuffers& b, int n, const double* src_sorted, double* dst_orig,
                       cudaStream_t s);
void launch_unsort_u32(const DevBuffers& b, int n, const uint32_t* src_sorted, double* dst_orig,
                       cudaStream_t s);
void launch_iota(uint32_t* dst, int n, cudaStream_t s);
void launch_fill_f64(double* dst, double v, int n, cudaStream_t s);
void launch_interleave3(const double* x, const double* y, const double* z, double* dst, int n,
                        cudaStream_t s);
void launch_deinterleave3(const double* src, double* x, double* y, double* z, int n,
                          cudaStream_t s);
void launch_u32_from_f64(const double* src, uint32_t* dst, int n, cudaStream_t s);

// Optional events recorded between the passes (phase timing); any may be null.
struct PassEvents {
  cudaEvent_t after_prep = nullptr;
  cudaEvent_t after_density = nullptr;
};

// step_plain.cu
void launch_plain_passes(const StepConsts& c, DevBuffers& b, cudaStream_t s, const PassEvents& ev);

// step_comp.cu
void launch_comp_passes(const StepConsts& c, DevBuffers& b, cudaStream_t s, const PassEvents& ev);

size_t scan_block_sums_needed(int count);
// Entries of the tiled sort's tile scans for a box of ncells cells (tiles of 8
// cells or more, plus the overflow bucket, in whole scan tiles).
size_t tile_scan_length(int ncells);
// Scan-tile sums the tile scan needs (two per scan tile) for a box of ncells.
size_t tile_scan_sums_needed(int ncells);

// Launch knobs (results do not depend on them): resident CTAs per SM of the
// tiled passes' persistent grids (0 = the occupancy limit), their tile
// distribution (static stride or a device work queue) and the block size of
// the sort's per-particle kernels.
struct LaunchTuning {
  int ctas_per_sm = 0;
  int queue = 0;
  int sort_block = 256;
  int dense_masks = 1;  // 1: the dense-cell force pass walks the density pass's masks
};

// step_tiled.cu: the FP32-compensated passes over staged 4x4x4-cell tiles.
void launch_comp_tiled(const StepConsts& c, DevBuffers& b, cudaStream_t s, const PassEvents& ev,
                       const LaunchTuning& t);
int tiled_max_ctas_per_sm();

}  // namespace phy
