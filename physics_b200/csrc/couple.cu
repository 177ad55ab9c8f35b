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
// through shared memory and summed in visit order by one thread (the
// reference's sequential sums); the reaction is then applied in parallel
// (every fluid particle lies in one cell, so the updates are disjoint).
// Consecutive points whose neighbourhoods are pairwise disjoint run at once,
// one warp each (k_couple_points_grouped); k_couple_points is the one-point-
// at-a-time form, used when the grouped walk's shared memory is unavailable.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

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

// The point's force from its ordered sums (world.rs:712-736), written to
// q[7..9]; r = the reaction -f dt and the sum of the masses (the reference's
// second pass sums them in the same order).
__device__ __forceinline__ void point_force(const StepConsts& c, const CoupleArgs& a, double* q, double sx,
                                            double sy, double sz, double sw, double* r) {
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
  r[0] = -fx * a.dt;
  r[1] = -fy * a.dt;
  r[2] = -fz * a.dt;
  r[3] = sw;
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
    if (t < 32) {
      // Warp 0: lane u < 27 reads cell u of the visit order (u = 9 (di+1) +
      // 3 (dj+1) + (dk+1)); a shuffle scan gives the cells' first candidates.
      const double x = q[0], y = q[1], z = q[2];
      // world.rs:704-711 (a NaN coordinate passes, as there).
      const bool in = !(x < c.lo[0] || x > c.hi[0] || y < c.lo[1] || y > c.hi[1] || z < c.lo[2] || z > c.hi[2]);
      if (t == 0) s_in = in ? 1 : 0;
      if (in) {
        const long long kx = key_axis(x, c.inv_cell), ky = key_axis(y, c.inv_cell), kz = key_axis(z, c.inv_cell);
        uint32_t beg = 0, cnt = 0;
        if (t < 27) {
          const int lin = cell_linear(c, kx + t / 9 - 1, ky + (t / 3) % 3 - 1, kz + t % 3 - 1);
          if (lin >= 0) {
            beg = a.cell_start[lin];
            cnt = a.cell_start[lin + 1] - beg;
          }
        }
        uint32_t incl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
          if (t >= o) incl += y;
        }
        if (t < 27) {
          s_beg[t] = beg;
          s_pre[t] = incl - cnt;
        }
        if (t == 26) s_pre[27] = incl;
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
    if (t == 0) point_force(c, a, q, sx, sy, sz, sw, s_r);
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

// Grouped form of the same walk.  Only velocities change from one point to
// the next, so everything else is prepared in parallel first: one warp per
// point finds its 27 cell ranges and whether its neighbourhood overlaps those
// of the kGW - 1 points before it (k_point_tables), and, after a prefix sum
// of the candidate counts, writes its candidates' particle indices and masses
// in visit order (k_point_candidates).  Two points whose centre cells are
// more than 2 apart on some axis have disjoint 27-cell neighbourhoods, so
// they read and write disjoint particles: a run of consecutive points that
// are pairwise disjoint (a group) gives the same velocities and forces
// whether its points run one after another or at once.  The walk (one CTA)
// takes the groups in order and runs a group's points at once, one warp
// each: the lanes stage the candidates' products v_j m_j in the warp's
// shared buffer (the same f64 products), lane 0 adds them in visit order
// (the reference's sequential sums), and the lanes apply the reaction to the
// candidates they hold (v_j + share, with the velocities they gathered).
// Points with more than kPB candidates have no list and read their
// candidates through their cell table.
constexpr int kGW = 16;         // warps of the walk: points per group at most
constexpr int kPer = 8;         // candidates a lane holds per chunk
constexpr int kWB = 32 * kPer;  // candidates per chunk of a warp
constexpr int kPB = 4096;       // candidates a point may have for a list
constexpr int kTabU = 56;       // u32 per point table: in, total, beg[27], cnt[27]

// world.rs:704-711 (a NaN coordinate passes, as there).
__device__ __forceinline__ bool point_in(const StepConsts& c, const double* q) {
  const double x = q[0], y = q[1], z = q[2];
  return !(x < c.lo[0] || x > c.hi[0] || y < c.lo[1] || y > c.hi[1] || z < c.lo[2] || z > c.hi[2]);
}

// One warp per point w of the batch: in-bounds flag, candidate count and
// cell ranges, and conf[w]: bit m (1 <= m < kGW) when the neighbourhood of
// point w overlaps that of point w - m (both in bounds, centre cells at most
// 2 apart on every axis).
__global__ void __launch_bounds__(256) k_point_tables(StepConsts c, CoupleArgs a, int nb, uint32_t* tab,
                                                      uint32_t* totals, uint16_t* conf) {
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= nb) return;
  const double* q = a.pts + 10 * (size_t)w;
  const bool in = point_in(c, q);
  const long long kx = key_axis(q[0], c.inv_cell), ky = key_axis(q[1], c.inv_cell),
                  kz = key_axis(q[2], c.inv_cell);
  uint32_t beg = 0, cnt = 0;
  if (in && lane < 27) {
    const int lin = cell_linear(c, kx + lane / 9 - 1, ky + (lane / 3) % 3 - 1, kz + lane % 3 - 1);
    if (lin >= 0) {
      beg = a.cell_start[lin];
      cnt = a.cell_start[lin + 1] - beg;
    }
  }
  bool overlap = false;
  if (in && lane >= 1 && lane < kGW && w - lane >= 0) {
    const double* p = a.pts + 10 * (size_t)(w - lane);
    if (point_in(c, p)) {
      const long long dx = key_axis(p[0], c.inv_cell) - kx, dy = key_axis(p[1], c.inv_cell) - ky,
                      dz = key_axis(p[2], c.inv_cell) - kz;
      overlap = dx >= -2 && dx <= 2 && dy >= -2 && dy <= 2 && dz >= -2 && dz <= 2;
    }
  }
  const uint32_t bits = __ballot_sync(0xffffffffu, overlap);
  const uint32_t total = __reduce_add_sync(0xffffffffu, cnt);
  uint32_t* t = tab + (size_t)w * kTabU;
  if (lane < 27) {
    t[2 + lane] = beg;
    t[29 + lane] = cnt;
  }
  if (lane == 0) {
    t[0] = in ? 1u : 0u;
    t[1] = total;
    totals[w] = in && total <= (uint32_t)kPB ? total : 0u;
    conf[w] = (uint16_t)bits;
  }
}

// One warp per point: the candidates of a point that has a list, in visit
// order (cell after cell, ascending slot: ascending insertion index), from
// off[w].
__global__ void __launch_bounds__(256) k_point_candidates(CoupleArgs a, int nb, const uint32_t* tab,
                                                          const uint32_t* off, uint32_t* idx, double* m) {
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= nb) return;
  const uint32_t* t = tab + (size_t)w * kTabU;
  if (!t[0] || t[1] > (uint32_t)kPB) return;
  uint32_t o = off[w];
  for (int u = 0; u < 27; ++u) {
    const uint32_t beg = t[2 + u], cnt = t[29 + u];
    for (uint32_t e = lane; e < cnt; e += 32) {
      const uint32_t i = a.perm[beg + e];
      idx[o + e] = i;
      m[o + e] = a.mass[i];
    }
    o += cnt;
  }
}

struct PointLists {
  const uint32_t* tab;
  const uint32_t* off;
  const uint32_t* idx;
  const double* m;
  const uint16_t* conf;
};

// Cell table of a point without a list (its warp's copy).
struct WarpTable {
  uint32_t beg[27];
  uint32_t pre[28];
};

// One warp: all of point j's work in the walk.  `pw` is the warp's buffer of
// 2 kWB products, `r` its reaction and mass sum.
__device__ __forceinline__ void walk_point(const StepConsts& c, const CoupleArgs& a, const PointLists& L, int j,
                                           double2* pw, WarpTable& T, double* r) {
  const int lane = threadIdx.x & 31;
  const uint32_t* t = L.tab + (size_t)j * kTabU;
  if (!t[0]) return;  // outside the bounds: skipped, force left unwritten
  const uint32_t total = t[1];
  const bool listed = total <= (uint32_t)kPB;
  const uint32_t o = listed ? L.off[j] : 0u;
  if (!listed) {
    const uint32_t beg = lane < 27 ? t[2 + lane] : 0u, cnt = lane < 27 ? t[29 + lane] : 0u;
    uint32_t incl = cnt;
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += v;
    }
    if (lane < 27) {
      T.beg[lane] = beg;
      T.pre[lane] = incl - cnt;
    }
    if (lane == 26) T.pre[27] = incl;
    __syncwarp();
  }
  double sx = 0.0, sy = 0.0, sz = 0.0, sw = 0.0;  // lane 0's sums
  uint32_t ci[kPer];
  double cm[kPer], cx[kPer], cy[kPer], cz[kPer];
  for (uint32_t base = 0; base < total; base += kWB) {
    const uint32_t cnt = min((uint32_t)kWB, total - base);
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const uint32_t e = (uint32_t)lane + 32u * k;
      if (e < cnt) {
        const uint32_t i = listed ? L.idx[o + base + e] : candidate(a, T.beg, T.pre, base + e);
        const double m = listed ? L.m[o + base + e] : a.mass[i];
        const double vx = a.vx[i], vy = a.vy[i], vz = a.vz[i];
        pw[2 * e] = make_double2(vx * m, vy * m);
        pw[2 * e + 1] = make_double2(vz * m, m);
        ci[k] = i;
        cm[k] = m;
        cx[k] = vx;
        cy[k] = vy;
        cz[k] = vz;
      }
    }
    __syncwarp();
    if (lane == 0) {
      // Eight candidates' products are loaded before they are added, so the
      // loads overlap while the four sums still add in candidate order.
      uint32_t e = 0;
      for (; e + 8 <= cnt; e += 8) {
        double2 P[8], R[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          P[u] = pw[2 * (e + u)];
          R[u] = pw[2 * (e + u) + 1];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          sx = sx + P[u].x;
          sy = sy + P[u].y;
          sz = sz + R[u].x;
          sw = sw + R[u].y;
        }
      }
      for (; e < cnt; ++e) {
        const double2 P = pw[2 * e], R = pw[2 * e + 1];
        sx = sx + P.x;
        sy = sy + P.y;
        sz = sz + R.x;
        sw = sw + R.y;
      }
    }
    __syncwarp();  // the chunk is summed before the next one is staged
  }
  if (lane == 0) point_force(c, a, a.pts + 10 * (size_t)j, sx, sy, sz, sw, r);
  __syncwarp();
  const double msum = r[3];
  if (!(msum > 0.0)) return;
  const double rx = r[0], ry = r[1], rz = r[2];
  if (total <= (uint32_t)kWB) {
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const uint32_t e = (uint32_t)lane + 32u * k;
      if (e < total) {
        const double frac = cm[k] / msum;
        a.vx[ci[k]] = cx[k] + rx * frac;
        a.vy[ci[k]] = cy[k] + ry * frac;
        a.vz[ci[k]] = cz[k] + rz * frac;
      }
    }
  } else {
    for (uint32_t e = lane; e < total; e += 32) {
      const uint32_t i = listed ? L.idx[o + e] : candidate(a, T.beg, T.pre, e);
      const double frac = (listed ? L.m[o + e] : a.mass[i]) / msum;
      a.vx[i] = a.vx[i] + rx * frac;
      a.vy[i] = a.vy[i] + ry * frac;
      a.vz[i] = a.vz[i] + rz * frac;
    }
  }
}

// The walk over the nb points of a batch: group after group, a group being
// the longest run (at most kGW) of points after its first whose
// neighbourhoods overlap none of the run's earlier points.
__global__ void __launch_bounds__(kGW * 32, 1) k_couple_points_grouped(StepConsts c, CoupleArgs a, int nb,
                                                                       PointLists L) {
  extern __shared__ __align__(16) unsigned char smem[];
  double2* s_pw = reinterpret_cast<double2*>(smem);                    // [kGW][2 kWB]
  uint16_t* s_conf = reinterpret_cast<uint16_t*>(s_pw + 2 * kWB * kGW);  // [nb]
  __shared__ WarpTable s_tab[kGW];
  __shared__ double s_r[kGW][4];
  __shared__ int s_group;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = threadIdx.x; k < nb; k += kGW * 32) s_conf[k] = L.conf[k];
  __syncthreads();
  for (int j = 0; j < nb;) {
    if (warp == 0) {
      // Lane l < kGW stops the group before point j + l when that point
      // overlaps one of j .. j + l - 1 (conf bits 1..l) or is past the batch.
      bool stop = false;
      if (lane >= 1 && lane < kGW) stop = j + lane >= nb || (s_conf[j + lane] & ((2u << lane) - 1u)) != 0u;
      const uint32_t b = __ballot_sync(0xffffffffu, stop) | (1u << kGW);
      if (lane == 0) s_group = __ffs((int)(b >> 1));
    }
    __syncthreads();
    const int g = s_group;
    if (warp < g) walk_point(c, a, L, j + warp, s_pw + (size_t)warp * 2 * kWB, s_tab[warp], s_r[warp]);
    __syncthreads();  // the group's reactions are applied before the next group gathers
    j += g;
  }
}

constexpr size_t kGroupedSmemFixed = (size_t)kGW * 2 * kWB * sizeof(double2);

// ---- couple_heat (world.rs:555-678) ------------------------------------------------
//
// Per particle (parallel): the trilinear temperature of the heat grid at its
// position gives body_acc += -g * beta * (T - t_ref); its source amount
// heat_gain * |v| * dt and source cell are stored by insertion index.  The
// reference adds the sources to the grid particle after particle, so a cell's
// sum is taken in insertion order: a stable radix sort of the (cell,
// insertion index) pairs by cell, then one sequential sum per cell.

struct HeatArgs {
  uint64_t nx, ny, nz;  // grid cells per axis (x fastest in memory)
  double ox, oy, oz, dx;
  const double* u;  // temperatures
  double t_ref, beta, gain, dt;
  const uint32_t* id;  // sorted slot -> insertion index
  const double* px;
  const double* py;
  const double* pz;
  const double* vx;
  const double* vy;
  const double* vz;
  double* bax;
  double* bay;
  double* baz;
  uint32_t* key;  // by insertion index: source cell, or nx*ny*nz for none
  double* val;    // by insertion index: source amount
  int n;
};

// num-traits ToPrimitive::to_usize of an f64, None -> 0.
__device__ __forceinline__ uint64_t to_usize_or_zero(double f) {
  return (f > -1.0 && f < 18446744073709551616.0) ? (uint64_t)f : 0ull;
}

// ScalarField::sample (phy-field grid.rs:203-208): indices clamped to the grid.
__device__ __forceinline__ double heat_sample(const HeatArgs& h, uint64_t x, uint64_t y, uint64_t z) {
  x = x < h.nx - 1 ? x : h.nx - 1;
  y = y < h.ny - 1 ? y : h.ny - 1;
  z = z < h.nz - 1 ? z : h.nz - 1;
  return h.u[x + h.nx * (y + h.ny * z)];
}

// HeatField::sample_trilinear (phy-field heat.rs:130-171).
__device__ double heat_trilinear(const HeatArgs& h, uint64_t cx, uint64_t cy, uint64_t cz, double fx, double fy,
                                 double fz) {
  const uint64_t x1 = cx + 1 < h.nx - 1 ? cx + 1 : h.nx - 1;
  const uint64_t y1 = cy + 1 < h.ny - 1 ? cy + 1 : h.ny - 1;
  const uint64_t z1 = cz + 1 < h.nz - 1 ? cz + 1 : h.nz - 1;
  const double c000 = heat_sample(h, cx, cy, cz), c100 = heat_sample(h, x1, cy, cz);
  const double c010 = heat_sample(h, cx, y1, cz), c110 = heat_sample(h, x1, y1, cz);
  const double c001 = heat_sample(h, cx, cy, z1), c101 = heat_sample(h, x1, cy, z1);
  const double c011 = heat_sample(h, cx, y1, z1), c111 = heat_sample(h, x1, y1, z1);
  const double x00 = c000 + (c100 - c000) * fx;
  const double x10 = c010 + (c110 - c010) * fx;
  const double x01 = c001 + (c101 - c001) * fx;
  const double x11 = c011 + (c111 - c011) * fx;
  const double y0 = x00 + (x10 - x00) * fy;
  const double y1v = x01 + (x11 - x01) * fy;
  return y0 + (y1v - y0) * fz;
}

__global__ void __launch_bounds__(kCT) k_heat_particles(StepConsts c, HeatArgs h) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= h.n) return;
  const uint32_t none = (uint32_t)(h.nx * h.ny * h.nz);
  uint32_t key = none;
  double val = 0.0;
  const double x = h.px[s], y = h.py[s], z = h.pz[s];
  // world.rs:635-645: only particles inside the fluid bounds.
  if (!(x < c.lo[0] || x > c.hi[0] || y < c.lo[1] || y > c.hi[1] || z < c.lo[2] || z > c.hi[2])) {
    // to_idx (world.rs:577-598); dims.saturating_sub(1), dims >= 1 here.
    const bool in = !(x < h.ox || x > h.ox + h.dx * (double)(h.nx - 1) || y < h.oy ||
                      y > h.oy + h.dx * (double)(h.ny - 1) || z < h.oz || z > h.oz + h.dx * (double)(h.nz - 1));
    uint64_t cx = 0, cy = 0, cz = 0;
    double temp = h.t_ref;
    if (in) {
      const double fx = floor((x - h.ox) / h.dx), fy = floor((y - h.oy) / h.dx), fz = floor((z - h.oz) / h.dx);
      cx = to_usize_or_zero(fx);
      cy = to_usize_or_zero(fy);
      cz = to_usize_or_zero(fz);
      temp = heat_trilinear(h, cx, cy, cz, (x - h.ox) / h.dx - fx, (y - h.oy) / h.dx - fy, (z - h.oz) / h.dx - fz);
    }
    const double dT = temp - h.t_ref;
    h.bax[s] = h.bax[s] + -c.g[0] * h.beta * dT;
    h.bay[s] = h.bay[s] + -c.g[1] * h.beta * dT;
    h.baz[s] = h.baz[s] + -c.g[2] * h.beta * dT;
    if (h.gain > 0.0 && in && cx < h.nx && cy < h.ny && cz < h.nz) {
      const double vx = h.vx[s], vy = h.vy[s], vz = h.vz[s];
      const double speed = sqrt((vx * vx + vy * vy) + vz * vz);
      key = (uint32_t)(cx + h.nx * (cy + h.ny * cz));
      val = h.gain * speed * h.dt;
    }
  }
  const uint32_t i = h.id[s];
  h.key[i] = key;
  h.val[i] = val;
}

// Stable LSD radix sort of 32-bit keys with a 32-bit payload, 8 bits a pass.
// Block b owns keys [b * kRTile, (b + 1) * kRTile); hist[d * nblocks + b]
// counts digit d in block b, and its exclusive scan (digit-major) is the
// first output slot of block b's keys of digit d.
constexpr int kRT = 256;
constexpr int kRRounds = 32;
constexpr int kRTile = kRT * kRRounds;

__global__ void __launch_bounds__(kRT) k_radix_hist(const uint32_t* key, int n, int shift, uint32_t* hist,
                                                     int nblocks) {
  __shared__ uint32_t s_h[256];
  const int t = threadIdx.x;
  s_h[t] = 0;
  __syncthreads();
  const int base = blockIdx.x * kRTile;
  for (int r = 0; r < kRRounds; ++r) {
    const int e = base + r * kRT + t;
    if (e < n) atomicAdd(&s_h[(key[e] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(size_t)t * nblocks + blockIdx.x] = s_h[t];
}

// In-place exclusive scan of len values by one block (each thread scans a
// contiguous run).
__global__ void __launch_bounds__(1024) k_scan_single(uint32_t* v, int len) {
  __shared__ uint32_t s_part[1024];
  const int t = threadIdx.x;
  const int per = (len + 1023) / 1024;
  const int lo = min(t * per, len), hi = min(lo + per, len);
  uint32_t sum = 0;
  for (int i = lo; i < hi; ++i) sum += v[i];
  s_part[t] = sum;
  __syncthreads();
  if (t == 0) {
    uint32_t run = 0;
    for (int k = 0; k < 1024; ++k) {
      const uint32_t x = s_part[k];
      s_part[k] = run;
      run += x;
    }
  }
  __syncthreads();
  uint32_t run = s_part[t];
  for (int i = lo; i < hi; ++i) {
    const uint32_t x = v[i];
    v[i] = run;
    run += x;
  }
}

// Scatter with ranks stable in key order: round r takes keys base + r*256 ..
// +255; a key's rank among equal digits is (earlier rounds) + (earlier warps
// of this round) + (earlier lanes of its warp).
__global__ void __launch_bounds__(kRT) k_radix_scatter(const uint32_t* key_in, const uint32_t* val_in,
                                                        uint32_t* key_out, uint32_t* val_out, int n, int shift,
                                                        const uint32_t* off, int nblocks) {
  __shared__ uint32_t s_w[kRT / 32][256];
  __shared__ uint32_t s_run[256];
  __shared__ uint32_t s_base[256];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  s_run[t] = 0;
  s_base[t] = off[(size_t)t * nblocks + blockIdx.x];
  const int base = blockIdx.x * kRTile;
  for (int r = 0; r < kRRounds; ++r) {
    for (int w = 0; w < kRT / 32; ++w) s_w[w][t] = 0;
    __syncthreads();
    const int e = base + r * kRT + t;
    const bool valid = e < n;
    const uint32_t k = valid ? key_in[e] : 0u;
    const uint32_t d = valid ? (k >> shift) & 255u : 256u;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t lower = __popc(peers & ((1u << lane) - 1u));
    if (valid && lower == 0) s_w[warp][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t pre = 0;
      for (int w = 0; w < warp; ++w) pre += s_w[w][d];
      const uint32_t dst = s_base[d] + s_run[d] + pre + lower;
      key_out[dst] = k;
      val_out[dst] = val_in[e];
    }
    __syncthreads();
    uint32_t tot = 0;
    for (int w = 0; w < kRT / 32; ++w) tot += s_w[w][t];
    s_run[t] += tot;
    __syncthreads();
  }
}

// One sequential sum per source cell, in insertion order (the segment of the
// sorted keys), onto the cell's current source value.
__global__ void __launch_bounds__(kCT) k_heat_deposit(const uint32_t* key, const uint32_t* idx, const double* val,
                                                       int n, uint32_t none, double* src) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const uint32_t k = key[e];
  if (k == none || (e > 0 && key[e - 1] == k)) return;
  double sum = src[k];
  for (int j = e; j < n && key[j] == k; ++j) sum = sum + val[idx[j]];
  src[k] = sum;
}

__global__ void k_iota_u32(uint32_t* v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = (uint32_t)i;
}

// ---- couple_bodies (world.rs:414-503) ------------------------------------------------
//
// Containment is tested against each particle's position at the start of its
// turn, so the particles inside some body are found in parallel; the bodies'
// velocities then change particle after particle, so those particles are
// processed by one thread in insertion order (a radix sort of the flagged
// insertion indices), with the reference's loop over the bodies.

struct V3d {
  double x, y, z;
};
__device__ __forceinline__ V3d v3(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ V3d operator+(V3d a, V3d b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3d operator-(V3d a, V3d b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3d operator*(V3d a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3d operator/(V3d a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ double vdot(V3d a, V3d b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ double vnorm(V3d a) { return sqrt((a.x * a.x + a.y * a.y) + a.z * a.z); }
__device__ __forceinline__ V3d vnormalize(V3d a) { return a / vnorm(a); }
__device__ __forceinline__ V3d vcross(V3d a, V3d b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Unit quaternion (i, j, k, w) times a vector, nalgebra 0.33.3's formula:
// t = 2 (q.v x v); q v = (t * q.w + q.v x t) + v; the inverse negates q.v.
__device__ V3d qrot(const double* q, V3d v, bool inverse) {
  const double s = inverse ? -1.0 : 1.0;
  const V3d u = v3(s * q[0], s * q[1], s * q[2]);
  const V3d t = vcross(u, v) * 2.0;
  return (t * q[3] + vcross(u, t)) + v;
}

struct BodyArgs {
  PhyCoupleBody* bodies;
  int nb;
  const double* data;
  const uint32_t* faces;
  double* displaced;  // nb
};

__device__ __forceinline__ V3d body_pos(const PhyCoupleBody& b) { return v3(b.pos[0], b.pos[1], b.pos[2]); }
__device__ __forceinline__ V3d to_local(const PhyCoupleBody& b, V3d p) { return qrot(b.rot, p - body_pos(b), true); }
__device__ __forceinline__ V3d to_world(const PhyCoupleBody& b, V3d p) { return qrot(b.rot, p, false) + body_pos(b); }

// A leaf shape (sphere, capsule, box, convex, heightfield): a body's own, or
// one sub shape of a compound body.
struct ShapeRef {
  int shape;
  double size[3];
  uint32_t data_first, data_count, face_first, face_count;
};

__device__ __forceinline__ ShapeRef shape_of(const PhyCoupleBody& b) {
  return {b.shape, {b.size[0], b.size[1], b.size[2]}, b.data_first, b.data_count, b.face_first, b.face_count};
}

// Sub shape q of compound body b (a 16-double record in the data array:
// shape, size, offset, quaternion, then its own data ranges).
__device__ __forceinline__ ShapeRef sub_shape(const BodyArgs& a, const PhyCoupleBody& b, uint32_t q, V3d& off,
                                              double rot[4]) {
  const double* r = a.data + b.data_first + 16 * (size_t)q;
  off = v3(r[4], r[5], r[6]);
  for (int k = 0; k < 4; ++k) rot[k] = r[7 + k];
  return {(int)r[0], {r[1], r[2], r[3]}, (uint32_t)r[11], (uint32_t)r[12], (uint32_t)r[13], (uint32_t)r[14]};
}

__device__ V3d support_leaf(const BodyArgs& a, const ShapeRef& b, V3d dir) {  // shape.rs:198-236
  switch (b.shape) {
    case PHY_SHAPE_SPHERE:
      return vnormalize(dir) * b.size[0];
    case PHY_SHAPE_CAPSULE: {
      const V3d n = vnormalize(dir);
      const V3d end = dir.y > 0.0 ? v3(0.0, b.size[0], 0.0) : dir.y < 0.0 ? v3(0.0, -b.size[0], 0.0) : v3(0, 0, 0);
      return end + n * b.size[1];
    }
    case PHY_SHAPE_BOX:
      return v3(dir.x >= 0.0 ? b.size[0] : -b.size[0], dir.y >= 0.0 ? b.size[1] : -b.size[1],
                dir.z >= 0.0 ? b.size[2] : -b.size[2]);
    case PHY_SHAPE_CONVEX: {
      const double* v = a.data + b.data_first;
      V3d best = v3(v[0], v[1], v[2]);
      double best_dot = vdot(best, dir);
      for (uint32_t k = 1; k < b.data_count; ++k) {
        const V3d c = v3(v[3 * k], v[3 * k + 1], v[3 * k + 2]);
        const double d = vdot(c, dir);
        if (d > best_dot) {
          best_dot = d;
          best = c;
        }
      }
      return best;
    }
    default:
      return v3(0, 0, 0);
  }
}

// Shape::Compound: the sub shape farthest along dir, in body coordinates;
// the search starts from the first sub shape's offset at dot 0
// (shape.rs:238-254).
__device__ V3d support_local(const BodyArgs& a, const PhyCoupleBody& b, V3d dir) {
  if (b.shape != PHY_SHAPE_COMPOUND) return support_leaf(a, shape_of(b), dir);
  V3d best = v3(0, 0, 0);
  double best_dot = 0.0;
  for (uint32_t q = 0; q < b.data_count; ++q) {
    V3d off;
    double rot[4];
    const ShapeRef sub = sub_shape(a, b, q, off, rot);
    if (q == 0) best = off;
    const V3d s = support_leaf(a, sub, qrot(rot, dir, true));
    const V3d ws = off + qrot(rot, s, false);
    const double d = vdot(ws, dir);
    if (d > best_dot) {
      best_dot = d;
      best = ws;
    }
  }
  return best;
}

__device__ bool contains_leaf(const BodyArgs& a, const ShapeRef& b, V3d p) {  // shape.rs:287-318
  switch (b.shape) {
    case PHY_SHAPE_SPHERE:
      return vnorm(p) <= b.size[0];
    case PHY_SHAPE_CAPSULE: {
      const double h = b.size[0], r = b.size[1];
      const double y = p.y < -h ? -h : (p.y > h ? h : p.y);
      const double cx = p.x * p.x + (p.y - y) * (p.y - y) + p.z * p.z;
      return cx <= r * r;
    }
    case PHY_SHAPE_BOX:
      return fabs(p.x) <= b.size[0] && fabs(p.y) <= b.size[1] && fabs(p.z) <= b.size[2];
    case PHY_SHAPE_CONVEX: {
      const double* v = a.data + b.data_first;
      const uint32_t* f = a.faces + 3 * (size_t)b.face_first;
      for (uint32_t k = 0; k < b.face_count; ++k) {
        const uint32_t i0 = f[3 * k], i1 = f[3 * k + 1], i2 = f[3 * k + 2];
        const V3d pa = v3(v[3 * i0], v[3 * i0 + 1], v[3 * i0 + 2]);
        const V3d pb = v3(v[3 * i1], v[3 * i1 + 1], v[3 * i1 + 2]);
        const V3d pc = v3(v[3 * i2], v[3 * i2 + 1], v[3 * i2 + 2]);
        if (vdot(p - pa, vcross(pb - pa, pc - pa)) > 0.0) return false;
      }
      return true;
    }
    default:
      return false;
  }
}

// Shape::Compound: any sub shape contains p in its own coordinates
// (shape.rs:319-322).
__device__ bool contains_local(const BodyArgs& a, const PhyCoupleBody& b, V3d p) {
  if (b.shape != PHY_SHAPE_COMPOUND) return contains_leaf(a, shape_of(b), p);
  for (uint32_t q = 0; q < b.data_count; ++q) {
    V3d off;
    double rot[4];
    const ShapeRef sub = sub_shape(a, b, q, off, rot);
    if (contains_leaf(a, sub, qrot(rot, p - off, true))) return true;
  }
  return false;
}

__device__ double volume_leaf(const BodyArgs& a, const ShapeRef& b) {  // world.rs:506-530
  const double pi = 3.14159265358979323846;
  switch (b.shape) {
    case PHY_SHAPE_SPHERE:
      return 4.0 / 3.0 * pi * b.size[0] * b.size[0] * b.size[0];
    case PHY_SHAPE_CAPSULE:
      return pi * b.size[1] * b.size[1] * 2.0 * b.size[0] + 4.0 / 3.0 * pi * b.size[1] * b.size[1] * b.size[1];
    case PHY_SHAPE_BOX:
      return b.size[0] * b.size[1] * b.size[2] * 8.0;
    case PHY_SHAPE_HEIGHTFIELD: {
      const double hx = b.size[0] * b.size[2], hz = b.size[1] * b.size[2];
      double sum = 0.0;
      for (uint32_t k = 0; k < b.data_count; ++k) sum = sum + a.data[b.data_first + k];
      const double hy = b.data_count == 0 ? 0.0 : sum / (double)b.data_count;
      return hx * hz * fabs(hy);
    }
    default:
      return 0.0;
  }
}

// Shape::Compound: the sub shapes' volumes folded from 0 in order
// (world.rs:531-534).
__device__ double body_volume(const BodyArgs& a, const PhyCoupleBody& b) {
  if (b.shape != PHY_SHAPE_COMPOUND) return volume_leaf(a, shape_of(b));
  double v = 0.0;
  for (uint32_t q = 0; q < b.data_count; ++q) {
    V3d off;
    double rot[4];
    v = v + volume_leaf(a, sub_shape(a, b, q, off, rot));
  }
  return v;
}


// world.rs:755-773
__device__ void push_out(const BodyArgs& a, const PhyCoupleBody& b, V3d& pos, V3d& vel) {
  const V3d local = to_local(b, pos);
  const V3d dir = vnorm(local) > 1e-9 ? vnormalize(local) : v3(0.0, 1.0, 0.0);
  const V3d sd = support_local(a, b, dir);
  pos = to_world(b, sd);
  const V3d v_rel = vel - v3(b.vel[0], b.vel[1], b.vel[2]);
  const V3d n = vnormalize(to_world(b, vnormalize(sd)) - body_pos(b));
  const double vn = vdot(v_rel, n);
  if (vn < 0.0) vel = vel - n * vn;
}

// Flags the particles inside any body: their insertion index and slot are
// appended (in no particular order) to key / val, the count to *count.
// mask[s] = the bit of the one body that holds slot s (bodies 0..31); a
// particle inside two or more bodies sets *multi.
__global__ void __launch_bounds__(kCT) k_body_flags(BodyArgs a, int n, const double* px, const double* py,
                                                     const double* pz, const uint32_t* id, uint32_t* key,
                                                     uint32_t* val, uint32_t* count, uint32_t* mask,
                                                     uint32_t* multi) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const V3d p = v3(px[s], py[s], pz[s]);
  int hits = 0, first = 0;
  for (int bi = 0; bi < a.nb; ++bi)
    if (contains_local(a, a.bodies[bi], to_local(a.bodies[bi], p))) {
      if (hits == 0) first = bi;
      ++hits;
    }
  if (hits == 0) return;
  if (hits > 1) atomicOr(multi, 1u);
  mask[s] = first < 32 ? 1u << first : 0u;
  const uint32_t k = atomicAdd(count, 1u);
  key[k] = id[s];
  val[k] = (uint32_t)s;
}

// One particle's contact with one body that holds it (the body of the
// reference's inner loop, world.rs:452-481): a static body pushes the particle
// out; a dynamic body takes the normal impulse of an approaching particle,
// counts its displaced volume and pushes it out (push_out's velocity replaces
// the particle's, as there).
__device__ __forceinline__ void body_contact(const BodyArgs& a, PhyCoupleBody& body, int bi, V3d p_world,
                                             double m_p, double particle_vol, V3d& pos, V3d& vel, V3d& v_p) {
  constexpr double restitution = 0.0;
  const V3d local = to_local(body, p_world);
  const V3d n = vnorm(local) > 1e-9 ? vnormalize(local) : v3(0.0, 1.0, 0.0);
  if (body.inv_mass <= 0.0) {
    push_out(a, body, pos, vel);
    v_p = vel;
    return;
  }
  const double v_rel_n = vdot(v_p - v3(body.vel[0], body.vel[1], body.vel[2]), n);
  if (v_rel_n < 0.0) {
    const double inv_sum = (1.0 / m_p) + body.inv_mass;
    const double j_mag = -(1.0 + restitution) * v_rel_n / inv_sum;
    const V3d j = n * j_mag;
    v_p = v_p + j / m_p;
    body.vel[0] = body.vel[0] + -j.x * body.inv_mass;  // apply_impulse(-j) (shape.rs:461-463)
    body.vel[1] = body.vel[1] + -j.y * body.inv_mass;
    body.vel[2] = body.vel[2] + -j.z * body.inv_mass;
  }
  a.displaced[bi] = a.displaced[bi] + particle_vol;
  push_out(a, body, pos, vel);
  v_p = vel;
}

// The reference's loops over the flagged particles (insertion order) and the
// bodies, then the buoyancy impulses (one CTA of kCT threads).  A body's
// velocity changes particle after particle, so the loops are ordered; but
// when every flagged particle lies in exactly one body (of at most 32), the
// bodies share no particle and each body's own sequence runs on its own
// thread: the warps first list each body's particles in insertion order (into
// `lists`), then thread b walks body b's.  Otherwise one thread runs the loops
// as written.  Both give the same bits.
__global__ void __launch_bounds__(kCT) k_body_contacts(StepConsts c, BodyArgs a, const uint32_t* slots, int m,
                                                        const double* mass, double* px, double* py, double* pz,
                                                        double* vx, double* vy, double* vz, double dt,
                                                        double particle_vol, const uint32_t* mask,
                                                        const uint32_t* multi, uint32_t* lists) {
  __shared__ uint32_t s_cnt[32];
  __shared__ uint32_t s_off[33];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const double rho_f = c.rest;
  if (t == 0)
    for (int bi = 0; bi < a.nb; ++bi) a.displaced[bi] = 0.0;
  __syncthreads();
  const bool by_body = a.nb <= 32 && *multi == 0u;  // uniform
  if (!by_body) {
    if (t == 0)
      for (int k = 0; k < m; ++k) {
        const uint32_t s = slots[k];
        const V3d p_world = v3(px[s], py[s], pz[s]);
        V3d pos = p_world;
        V3d vel = v3(vx[s], vy[s], vz[s]);
        V3d v_p = vel;
        const double m_p = mass[s];
        for (int bi = 0; bi < a.nb; ++bi) {
          PhyCoupleBody& body = a.bodies[bi];
          if (!contains_local(a, body, to_local(body, p_world))) continue;
          body_contact(a, body, bi, p_world, m_p, particle_vol, pos, vel, v_p);
        }
        px[s] = pos.x;
        py[s] = pos.y;
        pz[s] = pos.z;
        vx[s] = v_p.x;
        vy[s] = v_p.y;
        vz[s] = v_p.z;
      }
  } else {
    const int nw = blockDim.x >> 5;
    for (int bb = warp; bb < a.nb; bb += nw) {
      uint32_t cnt = 0;
      for (int k0 = 0; k0 < m; k0 += 32) {
        const int k = k0 + lane;
        cnt += __popc(__ballot_sync(0xffffffffu, k < m && mask[slots[k]] == (1u << bb)));
      }
      if (lane == 0) s_cnt[bb] = cnt;
    }
    __syncthreads();
    if (t == 0) {
      s_off[0] = 0;
      for (int bi = 0; bi < a.nb; ++bi) s_off[bi + 1] = s_off[bi] + s_cnt[bi];
    }
    __syncthreads();
    for (int bb = warp; bb < a.nb; bb += nw) {
      uint32_t o = s_off[bb];
      for (int k0 = 0; k0 < m; k0 += 32) {
        const int k = k0 + lane;
        const bool hit = k < m && mask[slots[k]] == (1u << bb);
        const uint32_t bal = __ballot_sync(0xffffffffu, hit);
        if (hit) lists[o + __popc(bal & ((1u << lane) - 1u))] = slots[k];
        o += __popc(bal);
      }
    }
    __syncthreads();
    if (t < a.nb) {
      PhyCoupleBody& body = a.bodies[t];
      for (uint32_t e = s_off[t]; e < s_off[t + 1]; ++e) {
        const uint32_t s = lists[e];
        const V3d p_world = v3(px[s], py[s], pz[s]);
        V3d pos = p_world;
        V3d vel = v3(vx[s], vy[s], vz[s]);
        V3d v_p = vel;
        body_contact(a, body, t, p_world, mass[s], particle_vol, pos, vel, v_p);
        px[s] = pos.x;
        py[s] = pos.y;
        pz[s] = pos.z;
        vx[s] = v_p.x;
        vy[s] = v_p.y;
        vz[s] = v_p.z;
      }
    }
  }
  __syncthreads();
  if (t == 0)
    for (int bi = 0; bi < a.nb; ++bi) {
      PhyCoupleBody& body = a.bodies[bi];
      if (body.inv_mass <= 0.0) continue;
      const double vol_b = body_volume(a, body);
      const double v_sub = a.displaced[bi] > 0.0 ? vol_b : 0.0;
      const double rv = rho_f * v_sub;
      body.vel[0] = body.vel[0] + -c.g[0] * rv * dt * body.inv_mass;
      body.vel[1] = body.vel[1] + -c.g[1] * rv * dt * body.inv_mass;
      body.vel[2] = body.vel[2] + -c.g[2] * rv * dt * body.inv_mass;
    }
}

}  // namespace

size_t couple_bodies_scratch_bytes(int n, int nb, uint64_t n_data, uint64_t n_faces) {
  return (size_t)nb * sizeof(PhyCoupleBody) + 8 * (size_t)nb + 8 * (size_t)n_data + 4 * (size_t)n_faces +
         20 * (size_t)n + 1024 * (size_t)((n + kRTile - 1) / kRTile) + 512;
}

int launch_couple_bodies(const StepConsts& c, DevBuffers& b, const CoupleBodiesLaunch& l, cudaStream_t s) {
  const int n = c.n;
  if (cudaMemcpyAsync(l.scratch, l.bodies, (size_t)l.nb * sizeof(PhyCoupleBody), cudaMemcpyHostToDevice, s) !=
      cudaSuccess)
    return -1;
  const size_t nbk = (size_t)((n + kRTile - 1) / kRTile);
  unsigned char* base = l.scratch;
  PhyCoupleBody* bodies = reinterpret_cast<PhyCoupleBody*>(base);
  double* displaced = reinterpret_cast<double*>(bodies + l.nb);
  double* data = displaced + l.nb;
  uint32_t* faces = reinterpret_cast<uint32_t*>(data + l.n_data);
  uint32_t* key0 = faces + l.n_faces;
  uint32_t* key1 = key0 + n;
  uint32_t* val0 = key1 + n;
  uint32_t* val1 = val0 + n;
  uint32_t* mask = val1 + n;  // by slot: the bit of the one body holding it
  uint32_t* hist = mask + n;
  uint32_t* count = hist + 256 * nbk;
  uint32_t* multi = count + 1;
  if (l.n_data && cudaMemcpyAsync(data, l.data, l.n_data * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return -1;
  if (l.n_faces &&
      cudaMemcpyAsync(faces, l.faces, l.n_faces * sizeof(uint32_t), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return -1;
  BodyArgs a;
  a.bodies = bodies;
  a.nb = l.nb;
  a.data = data;
  a.faces = faces;
  a.displaced = displaced;
  const ParticleConsts& pc = b.pc[b.cur];
  cudaMemsetAsync(count, 0, 2 * sizeof(uint32_t), s);  // count and multi
  const int blocks = (n + kCT - 1) / kCT;
  k_body_flags<<<blocks, kCT, 0, s>>>(a, n, b.pv1[0], b.pv1[1], b.pv1[2], pc.id, key0, val0, count, mask, multi);
  uint32_t m = 0;
  if (cudaMemcpyAsync(&m, count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return -1;
  uint32_t *kin = key0, *kout = key1, *vin = val0, *vout = val1;
  if (m > 1) {
    const int mb = (int)((m + kRTile - 1) / kRTile);
    int bits = 0;
    while (bits < 32 && ((uint32_t)(n - 1) >> bits) != 0u) ++bits;
    for (int shift = 0; shift < bits; shift += 8) {
      k_radix_hist<<<mb, kRT, 0, s>>>(kin, (int)m, shift, hist, mb);
      k_scan_single<<<1, 1024, 0, s>>>(hist, 256 * mb);
      k_radix_scatter<<<mb, kRT, 0, s>>>(kin, vin, kout, vout, (int)m, shift, hist, mb);
      uint32_t* t = kin;
      kin = kout;
      kout = t;
      t = vin;
      vin = vout;
      vout = t;
    }
  }
  // kout is free after the sort: it takes the per-body lists.
  k_body_contacts<<<1, kCT, 0, s>>>(c, a, vin, (int)m, pc.mass, b.pv1[0], b.pv1[1], b.pv1[2], b.pv1[3], b.pv1[4],
                                     b.pv1[5], c.dt, l.particle_vol, mask, multi, kout);
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(l.bodies, bodies, (size_t)l.nb * sizeof(PhyCoupleBody), cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return -1;
  return 0;
}

size_t couple_heat_scratch_bytes(int n, uint64_t cells) {
  const size_t nb = (size_t)((n + kRTile - 1) / kRTile);
  return 16 * (size_t)cells + 8 * (size_t)n + 16 * (size_t)n + 1024 * nb + 256;
}

void launch_couple_heat(const StepConsts& c, DevBuffers& b, const HeatGrid& g, unsigned char* scratch,
                        cudaStream_t s) {
  const int n = c.n;
  const uint64_t cells = g.nx * g.ny * g.nz;
  const size_t nb = (size_t)((n + kRTile - 1) / kRTile);
  double* u = reinterpret_cast<double*>(scratch);
  double* src = u + cells;
  double* val = src + cells;
  uint32_t* key0 = reinterpret_cast<uint32_t*>(val + n);
  uint32_t* key1 = key0 + n;
  uint32_t* id0 = key1 + n;
  uint32_t* id1 = id0 + n;
  uint32_t* hist = id1 + n;
  const ParticleConsts& pc = b.pc[b.cur];
  HeatArgs h;
  h.nx = g.nx;
  h.ny = g.ny;
  h.nz = g.nz;
  h.ox = g.origin[0];
  h.oy = g.origin[1];
  h.oz = g.origin[2];
  h.dx = g.cell;
  h.u = u;
  h.t_ref = g.t_ref;
  h.beta = g.beta;
  h.gain = g.heat_gain;
  h.dt = c.dt;
  h.id = pc.id;
  h.px = b.pv1[0];
  h.py = b.pv1[1];
  h.pz = b.pv1[2];
  h.vx = b.pv1[3];
  h.vy = b.pv1[4];
  h.vz = b.pv1[5];
  h.bax = pc.ba[0];
  h.bay = pc.ba[1];
  h.baz = pc.ba[2];
  h.key = key0;
  h.val = val;
  h.n = n;
  const int blocks = (n + kCT - 1) / kCT;
  k_heat_particles<<<blocks, kCT, 0, s>>>(c, h);
  if (!(g.heat_gain > 0.0)) return;
  const uint32_t none = (uint32_t)cells;
  int bits = 0;
  while (bits < 32 && (none >> bits) != 0u) ++bits;  // keys 0 .. none
  k_iota_u32<<<blocks, kCT, 0, s>>>(id0, n);
  uint32_t *kin = key0, *kout = key1, *iin = id0, *iout = id1;
  for (int shift = 0; shift < bits; shift += 8) {
    k_radix_hist<<<(int)nb, kRT, 0, s>>>(kin, n, shift, hist, (int)nb);
    k_scan_single<<<1, 1024, 0, s>>>(hist, (int)(256 * nb));
    k_radix_scatter<<<(int)nb, kRT, 0, s>>>(kin, iin, kout, iout, n, shift, hist, (int)nb);
    uint32_t* tk = kin;
    kin = kout;
    kout = tk;
    uint32_t* ti = iin;
    iin = iout;
    iout = ti;
  }
  k_heat_deposit<<<blocks, kCT, 0, s>>>(kin, iin, val, n, none, src);
}

namespace {

// Grows a device array to hold `count` elements (contents dropped).
template <class T>
void scratch_grow(T*& p, size_t& cap, size_t count, cudaStream_t s) {
  if (count <= cap && p) return;
  if (p) {
    cuda_check(cudaStreamSynchronize(s), "couple scratch sync");
    cudaFree(p);
    p = nullptr;
  }
  cap = std::max<size_t>(count, 1);
  cuda_check(cudaMalloc((void**)&p, cap * sizeof(T)), "cudaMalloc");
}

}  // namespace

void CouplePointsScratch::release() {
  for (uint32_t** p : {&tab, &totals, &off, &idx}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  if (m) cudaFree(m);
  m = nullptr;
  if (conf) cudaFree(conf);
  conf = nullptr;
  cap_tab = cap_totals = cap_off = cap_idx = cap_m = cap_conf = 0;
}

void launch_couple_points(const StepConsts& c, DevBuffers& b, double* d_pts, int np, double dt, double drag,
                          double soft_density, cudaStream_t s, CouplePointsScratch& sc) {
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
  // Points run in batches (one ordered walk per batch, in order on the
  // stream), which bounds the candidate lists and the walk's shared memory.
  constexpr int kBatch = 16384;
  static const bool smem_ok = [] {
    return cudaFuncSetAttribute(k_couple_points_grouped, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(kGroupedSmemFixed + kBatch * sizeof(uint16_t))) == cudaSuccess;
  }();
  if (!smem_ok) {
    k_couple_points<<<1, kCT, 0, s>>>(c, a);
    return;
  }
  std::vector<uint32_t> totals, off;
  for (int p0 = 0; p0 < np; p0 += kBatch) {
    const int nb = std::min(kBatch, np - p0);
    CoupleArgs ab = a;
    ab.pts = d_pts + 10 * (size_t)p0;
    scratch_grow(sc.tab, sc.cap_tab, (size_t)nb * kTabU, s);
    scratch_grow(sc.totals, sc.cap_totals, (size_t)nb, s);
    scratch_grow(sc.conf, sc.cap_conf, (size_t)nb, s);
    const int warps_per_block = 256 / 32, blocks = (nb + warps_per_block - 1) / warps_per_block;
    k_point_tables<<<blocks, 256, 0, s>>>(c, ab, nb, sc.tab, sc.totals, sc.conf);
    cuda_check(cudaGetLastError(), "point tables");
    totals.resize(nb);
    cuda_check(cudaMemcpyAsync(totals.data(), sc.totals, nb * sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
               "point totals");
    cuda_check(cudaStreamSynchronize(s), "point totals sync");
    off.resize(nb + 1);
    uint64_t sum = 0;
    for (int k = 0; k < nb; ++k) {
      off[k] = (uint32_t)sum;
      sum += totals[k];
    }
    off[nb] = (uint32_t)sum;  // at most kBatch * kPB candidates: fits 32 bits
    scratch_grow(sc.off, sc.cap_off, (size_t)nb + 1, s);
    scratch_grow(sc.idx, sc.cap_idx, (size_t)sum, s);
    scratch_grow(sc.m, sc.cap_m, (size_t)sum, s);
    cuda_check(cudaMemcpyAsync(sc.off, off.data(), (nb + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, s),
               "point offsets");
    k_point_candidates<<<blocks, 256, 0, s>>>(ab, nb, sc.tab, sc.off, sc.idx, sc.m);
    PointLists L{sc.tab, sc.off, sc.idx, sc.m, sc.conf};
    k_couple_points_grouped<<<1, kGW * 32, kGroupedSmemFixed + (size_t)nb * sizeof(uint16_t), s>>>(c, ab, nb, L);
    cuda_check(cudaGetLastError(), "couple points");
    // The offsets' host copy must outlive the upload.
    cuda_check(cudaStreamSynchronize(s), "couple points sync");
  }
}

}  // namespace phy
