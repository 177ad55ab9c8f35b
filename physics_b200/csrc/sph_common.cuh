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

// Error bits written by device code into the per-world flag word.
enum : uint32_t {
  kFlagOutOfBox = 1u,    // a cell key fell outside the grid box
  kFlagNonFinite = 2u,   // a new position or velocity is NaN/Inf
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
  // Grid box: key of cell 0 and dimensions (cells per axis).
  long long bx0, by0, bz0;
  int ncx, ncy, ncz;
  int ncells;
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

// A particle's own cell is an "interior" cell when its 27 neighbours are all
// inside the box; the host pads the box by one cell on every side so that
// every in-box particle qualifies.
__device__ __forceinline__ bool cell_interior(const StepConsts& c, long long i, long long j, long long k) {
  long long a = i - c.bx0, b = j - c.by0, d = k - c.bz0;
  return a >= 1 && b >= 1 && d >= 1 && a < c.ncx - 1 && b < c.ncy - 1 && d < c.ncz - 1;
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

#endif  // __CUDACC__

}  // namespace phy
