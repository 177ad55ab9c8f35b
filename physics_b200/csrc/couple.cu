// Two-way coupling of point masses with the fluid on the device:
// FluidWorld::couple_points (crates/phy-fluid/src/sph/world.rs:691-752).
//
// Semantics reproduced bit for bit (f64, no FMA contraction: this file is
// built with -fmad=false):
//   * the grid is rebuilt from the current positions (world.rs:700) and the
//     27 cells of a point are visited with di outermost, dk innermost, the
//     particles of a cell in ascending insertion index (grid.rs:43-56);
//   * points run one after another: each samples the mass-weighted mean
//     fluid velocity of its cells (v_sum += vel_j * m_j, w_sum += m_j, in
//     visit order), gets f = -g (rho0 vol) + (v_f - v) (drag m), and shares
//     -f dt among those fluid particles by m_j / sum(m) before the next point
//     samples (world.rs:702-751);
//   * a point outside the bounds is skipped and its force left unwritten.
//
// One CTA walks the points in order.  Per point, its candidates are staged
// through shared memory by all threads and summed in visit order by one
// thread (the reference's sequential sums); the reaction is then applied by
// all threads in parallel (every fluid particle lies in one cell, so the
// updates are disjoint).
#include <cuda_runtime.h>

#include "sph_buffers.h"

namespace phy {

namespace {

constexpr int kCT = 256;        // threads of the coupling CTA
constexpr int kCChunk = 1024;   // candidates staged per chunk

struct CoupleArgs {
  const uint32_t* cell_start;
  const uint32_t* perm;  // sorted slot -> particle, (cell, insertion index) order
  double* vx;
  double* vy;
  double* vz;
  const double* mass;
  double* pts;  // 10 doubles per point: pos xyz, vel xyz, mass, force xyz
  int np;
  double dt, drag, soft_density;
};

// Particle at flat candidate index `flat` of the point's 27 cells.
__device__ __forceinline__ uint32_t candidate(const CoupleArgs& a, const uint32_t* s_beg, const uint32_t* s_pre,
                                              uint32_t flat) {
  int u = 0;
  while (s_pre[u + 1] <= flat) ++u;  // flat < s_pre[27]: ends at a non-empty cell
  return a.perm[s_beg[u] + (flat - s_pre[u])];
}

__global__ void __launch_bounds__(kCT) k_couple_points(StepConsts c, CoupleArgs a) {
  __shared__ uint32_t s_beg[27];
  __shared__ uint32_t s_pre[28];
  __shared__ double s_v[3][kCChunk];
  __shared__ double s_m[kCChunk];
  __shared__ double s_r[4];  // reaction xyz, sum of masses
  __shared__ int s_in;
  const int t = threadIdx.x;
  for (int k = 0; k < a.np; ++k) {
    double* q = a.pts + 10 * (size_t)k;
    if (t == 0) {
      const double x = q[0], y = q[1], z = q[2];
      // world.rs:704-711 (a NaN coordinate passes, as there).
      const bool in = !(x < c.lo[0] || x > c.hi[0] || y < c.lo[1] || y > c.hi[1] || z < c.lo[2] || z > c.hi[2]);
      s_in = in ? 1 : 0;
      if (in) {
        const long long kx = key_axis(x, c.inv_cell), ky = key_axis(y, c.inv_cell), kz = key_axis(z, c.inv_cell);
        uint32_t acc = 0;
        int u = 0;
        for (int di = -1; di <= 1; ++di)
          for (int dj = -1; dj <= 1; ++dj)
            for (int dk = -1; dk <= 1; ++dk, ++u) {
              const int lin = cell_linear(c, kx + di, ky + dj, kz + dk);
              const uint32_t beg = lin >= 0 ? a.cell_start[lin] : 0u;
              const uint32_t cnt = lin >= 0 ? a.cell_start[lin + 1] - beg : 0u;
              s_beg[u] = beg;
              s_pre[u] = acc;
              acc += cnt;
            }
        s_pre[27] = acc;
      }
    }
    __syncthreads();
    if (!s_in) {
      __syncthreads();  // every thread has read s_in before thread 0 rewrites it
      continue;
    }
    const uint32_t total = s_pre[27];
    double sx = 0.0, sy = 0.0, sz = 0.0, sw = 0.0;  // thread 0's sums
    for (uint32_t base = 0; base < total; base += kCChunk) {
      const uint32_t m = min((uint32_t)kCChunk, total - base);
      for (uint32_t e = t; e < m; e += kCT) {
        const uint32_t i = candidate(a, s_beg, s_pre, base + e);
        s_v[0][e] = a.vx[i];
        s_v[1][e] = a.vy[i];
        s_v[2][e] = a.vz[i];
        s_m[e] = a.mass[i];
      }
      __syncthreads();
      if (t == 0)
        for (uint32_t e = 0; e < m; ++e) {
          const double w = s_m[e];
          sx = sx + s_v[0][e] * w;
          sy = sy + s_v[1][e] * w;
          sz = sz + s_v[2][e] * w;
          sw = sw + w;
        }
      __syncthreads();
    }
    if (t == 0) {
      double vfx = 0.0, vfy = 0.0, vfz = 0.0;
      if (sw > 0.0) {
        vfx = sx / sw;
        vfy = sy / sw;
        vfz = sz / sw;
      }
      const double pm = q[6];
      const double vol = a.soft_density > 0.0 ? pm / a.soft_density : 0.0;
      const double rv = c.rest * vol;
      const double dm = a.drag * pm;
      const double fx = -c.g[0] * rv + (vfx - q[3]) * dm;
      const double fy = -c.g[1] * rv + (vfy - q[4]) * dm;
      const double fz = -c.g[2] * rv + (vfz - q[5]) * dm;
      q[7] = fx;
      q[8] = fy;
      q[9] = fz;
      s_r[0] = -fx * a.dt;
      s_r[1] = -fy * a.dt;
      s_r[2] = -fz * a.dt;
      s_r[3] = sw;  // sum of the masses in visit order, as the reference's second pass
    }
    __syncthreads();
    const double msum = s_r[3];
    if (msum > 0.0)
      for (uint32_t flat = t; flat < total; flat += kCT) {
        const uint32_t i = candidate(a, s_beg, s_pre, flat);
        const double frac = a.mass[i] / msum;
        a.vx[i] = a.vx[i] + s_r[0] * frac;
        a.vy[i] = a.vy[i] + s_r[1] * frac;
        a.vz[i] = a.vz[i] + s_r[2] * frac;
      }
    __syncthreads();
  }
}

}  // namespace

void launch_couple_points(const StepConsts& c, DevBuffers& b, double* d_pts, int np, double dt, double drag,
                          double soft_density, cudaStream_t s) {
  CoupleArgs a;
  a.cell_start = b.cell_start;
  a.perm = b.perm;
  a.vx = b.pv1[3];
  a.vy = b.pv1[4];
  a.vz = b.pv1[5];
  a.mass = b.pc[b.cur].mass;
  a.pts = d_pts;
  a.np = np;
  a.dt = dt;
  a.drag = drag;
  a.soft_density = soft_density;
  k_couple_points<<<1, kCT, 0, s>>>(c, a);
}

}  // namespace phy
