// The f64 "plain" SPH passes: bit-identical to the reference's
// FluidWorld<f64>::step (crates/phy-fluid/src/sph/world.rs:183-397).
//
// Arithmetic contract: every floating-point operation is an explicit
// round-to-nearest intrinsic in the reference's evaluation order (this file
// is also compiled with -fmad=false), division and square root are the
// IEEE-exact double operations, and each particle's neighbour reduction runs
// sequentially in the reference's visit order (27 cells, di outer / dk inner,
// ascending insertion index within a cell).  One thread owns one particle, so
// the result does not depend on scheduling and repeats bit-exactly.
//
// Two exact shortcuts are used:
//   * a candidate whose squared distance exceeds `r2_guard` (the first double
//     above h*h) is skipped before the square root: sqrt(r2) >= h follows,
//     so `r < h` is false exactly as in the reference; NaN distances are
//     never skipped by it;
//   * p_j/(rho_j*rho_j) and m_j/rho_j, which the reference evaluates per pair
//     from the same operands, are evaluated once per particle in the density
//     pass (same expression, same value).
#include <cuda_runtime.h>

#include "sph_buffers.h"

namespace phy {

namespace {

constexpr int kThreads = 128;

// Kernels<T> (crates/phy-fluid/src/kernels.rs:39-65).
__device__ __forceinline__ double poly6(const StepConsts& c, double r) {
  if (r >= c.h0) return 0.0;
  double diff = __dsub_rn(c.h0sq, __dmul_rn(r, r));
  return __dmul_rn(__dmul_rn(__dmul_rn(c.poly6_c, diff), diff), diff);
}
__device__ __forceinline__ double spiky_grad_mag(const StepConsts& c, double r) {
  if (r >= c.h0 || r <= 0.0) return 0.0;
  double diff = __dsub_rn(c.h0, r);
  return __dmul_rn(__dmul_rn(c.spiky_c, diff), diff);
}
__device__ __forceinline__ double visc_lap(const StepConsts& c, double r) {
  if (r >= c.h0) return 0.0;
  return __dmul_rn(c.lap_c, __dsub_rn(c.h0, r));
}
// nalgebra Vector3::norm_squared: (x*x + y*y) + z*z.
__device__ __forceinline__ double norm2(double x, double y, double z) {
  return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

struct PlainArgs {
  const double* __restrict__ px;
  const double* __restrict__ py;
  const double* __restrict__ pz;
  const double* __restrict__ vx;
  const double* __restrict__ vy;
  const double* __restrict__ vz;
  const double* __restrict__ mass;
  const uint32_t* __restrict__ mat;
  const uint32_t* __restrict__ cell_start;
  double* bax;  // body_acc (nullable; zeroed after use)
  double* bay;
  double* baz;
  double* rho;
  double* p;
  double* pr2;
  double* mr;
  double* acc[3];
  double* xsph[3];
  double* mu;
  double* out_pv[6];
  uint32_t* nbr;
  uint32_t* nbr_count;
  int stride;  // column stride of nbr (the buffer capacity)
  uint32_t* flags;
  unsigned long long* counters;
  double* fv_out[3];  // nullable: raw viscous force (adjoint tape)
  double* shear_out;  // nullable: strain-rate proxy (adjoint tape)
};

// compute_density_pressure (world.rs:204-246).  Also records, in visit
// order, every candidate j != i that the force loop will not skip on the
// `r >= h` test: those with r < h and those whose distance is NaN (the
// reference's force loop does not skip NaN distances, world.rs:297).
template <bool kCount>
__global__ void __launch_bounds__(kThreads) k_density_plain(StepConsts c, PlainArgs a) {
  __shared__ uint32_t s_list[kStagedNeighbors][kThreads];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.n) return;
  const double xi = a.px[i], yi = a.py[i], zi = a.pz[i];
  const long long kx = key_axis(xi, c.inv_cell);
  const long long ky = key_axis(yi, c.inv_cell);
  const long long kz = key_axis(zi, c.inv_cell);
  double rho = 0.0;
  unsigned cand = 0, pairs = 0;
  uint32_t cnt = 0;
  uint32_t* lst = a.nbr + i;
  if (cell_interior(c, kx, ky, kz)) {
    const int base = cell_linear(c, kx - 1, ky - 1, kz - 1);
    for (int di = 0; di < 3; ++di) {
      for (int dj = 0; dj < 3; ++dj) {
        const int c0 = base + (di * c.ncy + dj) * c.ncz;
        const int s = (int)a.cell_start[c0], e = (int)a.cell_start[c0 + 3];
        if (kCount) cand += (unsigned)(e - s);
        for (int j = s; j < e; ++j) {
          // na_distance(p_i, p_j) = |p_i - p_j| (world.rs:777-779).
          double r2 = norm2(__dsub_rn(xi, a.px[j]), __dsub_rn(yi, a.py[j]), __dsub_rn(zi, a.pz[j]));
          if (r2 > c.r2_guard) continue;
          double r = __dsqrt_rn(r2);
          if (r < c.h) {
            rho = __dadd_rn(rho, __dmul_rn(a.mass[j], poly6(c, r)));
            if (kCount) ++pairs;
          }
          if (!(r >= c.h) && j != i) {
            if (cnt < (uint32_t)kStagedNeighbors)
              s_list[cnt][threadIdx.x] = (uint32_t)j;
            else if (cnt < (uint32_t)kMaxNeighbors)
              lst[(size_t)cnt * a.stride] = (uint32_t)j;
            ++cnt;
          }
        }
      }
    }
  }
  flush_staged_list<kThreads>(s_list, lst, a.stride, cnt, true);
  a.nbr_count[i] = cnt;
  double over = __dsub_rn(rho, c.rest);
  double pr = over > 0.0 ? __dmul_rn(c.stiff, over) : 0.0;
  a.rho[i] = rho;
  a.p[i] = pr;
  a.pr2[i] = __ddiv_rn(pr, __dmul_rn(rho, rho));
  a.mr[i] = __ddiv_rn(a.mass[i], rho);
  if (kCount) {
    const unsigned am = __activemask();
    const unsigned wc = __reduce_add_sync(am, cand);
    const unsigned wp = __reduce_add_sync(am, pairs);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(am) - 1)) {
      atomicAdd(&a.counters[0], (unsigned long long)wc);
      atomicAdd(&a.counters[1], (unsigned long long)wp);
    }
  }
}

struct PlainAcc {
  double fpx = 0.0, fpy = 0.0, fpz = 0.0;
  double fvx = 0.0, fvy = 0.0, fvz = 0.0;
  double xsx = 0.0, xsy = 0.0, xsz = 0.0;
  double shear = 0.0;
};

// One neighbour of compute_forces' loop body (world.rs:291-316), in the
// reference's expression order.  kShear = false leaves out the shear sum
// (StepConsts::shear_live: every reachable visc_n is 1, so mu never reads it).
template <bool kShear>
__device__ __forceinline__ void plain_pair(const StepConsts& c, const PlainArgs& a, int j, double xi, double yi,
                                           double zi, double vxi, double vyi, double vzi, double m_i,
                                           double pr2_i, PlainAcc& q) {
  // d = pos[j] - p_i; r = |d|; skip r >= h or r <= 0 (world.rs:295-299).
  const double dx = __dsub_rn(a.px[j], xi);
  const double dy = __dsub_rn(a.py[j], yi);
  const double dz = __dsub_rn(a.pz[j], zi);
  const double r2 = norm2(dx, dy, dz);
  if (r2 > c.r2_guard) return;
  const double r = __dsqrt_rn(r2);
  if (r >= c.h || r <= 0.0) return;
  const double rho_j = a.rho[j];
  const double m_j = a.mass[j];
  const double mm = __dmul_rn(m_i, m_j);
  // f_press += (d / r) * (coef * grad)   (world.rs:303-306)
  const double grad = spiky_grad_mag(c, r);
  const double coef = __dmul_rn(mm, __dadd_rn(pr2_i, a.pr2[j]));
  const double cg = __dmul_rn(coef, grad);
  q.fpx = __dadd_rn(q.fpx, __dmul_rn(__ddiv_rn(dx, r), cg));
  q.fpy = __dadd_rn(q.fpy, __dmul_rn(__ddiv_rn(dy, r), cg));
  q.fpz = __dadd_rn(q.fpz, __dmul_rn(__ddiv_rn(dz, r), cg));
  // f_visc_raw += (v_j - v_i) * (m_i * m_j / rho_j * lap)   (308-309)
  const double dvx = __dsub_rn(a.vx[j], vxi);
  const double dvy = __dsub_rn(a.vy[j], vyi);
  const double dvz = __dsub_rn(a.vz[j], vzi);
  const double vf = __dmul_rn(__ddiv_rn(mm, rho_j), visc_lap(c, r));
  q.fvx = __dadd_rn(q.fvx, __dmul_rn(dvx, vf));
  q.fvy = __dadd_rn(q.fvy, __dmul_rn(dvy, vf));
  q.fvz = __dadd_rn(q.fvz, __dmul_rn(dvz, vf));
  // xsph += (v_j - v_i) * (m_j / rho_j * w)   (311-312)
  const double mr_j = a.mr[j];
  const double xw = __dmul_rn(mr_j, poly6(c, r));
  q.xsx = __dadd_rn(q.xsx, __dmul_rn(dvx, xw));
  q.xsy = __dadd_rn(q.xsy, __dmul_rn(dvy, xw));
  q.xsz = __dadd_rn(q.xsz, __dmul_rn(dvz, xw));
  // shear += |v_j - v_i| / (r + 1e-4) * (m_j / rho_j)   (314-315)
  if (kShear) {
    const double dvn = __dsqrt_rn(norm2(dvx, dvy, dvz));
    q.shear = __dadd_rn(q.shear, __dmul_rn(__ddiv_rn(dvn, __dadd_rn(r, 1e-4)), mr_j));
  }
}

// compute_forces (world.rs:252-347) fused with integrate (352-363) and
// enforce_bounds (366-397).  The neighbours come from the density pass's list
// (same visit order); a particle whose list overflowed rescans its 27 cells.
template <bool kShear>
__global__ void __launch_bounds__(kThreads) k_force_plain(StepConsts c, PlainArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.n) return;
  const double xi = a.px[i], yi = a.py[i], zi = a.pz[i];
  const double vxi = a.vx[i], vyi = a.vy[i], vzi = a.vz[i];
  const double rho_i = a.rho[i], pr2_i = a.pr2[i], m_i = a.mass[i];
  PlainAcc q;
  const uint32_t cnt = a.nbr_count[i];
  if (cnt <= (uint32_t)kMaxNeighbors) {
    const uint32_t* lst = a.nbr + i;
    for (uint32_t k = 0; k < cnt; ++k)
      plain_pair<kShear>(c, a, (int)lst[(size_t)k * a.stride], xi, yi, zi, vxi, vyi, vzi, m_i, pr2_i, q);
  } else {
    const long long kx = key_axis(xi, c.inv_cell);
    const long long ky = key_axis(yi, c.inv_cell);
    const long long kz = key_axis(zi, c.inv_cell);
    const int base = cell_linear(c, kx - 1, ky - 1, kz - 1);  // interior: cnt > 0 needs a neighbour search
    for (int di = 0; di < 3; ++di) {
      for (int dj = 0; dj < 3; ++dj) {
        const int c0 = base + (di * c.ncy + dj) * c.ncz;
        const int s = (int)a.cell_start[c0], e = (int)a.cell_start[c0 + 3];
        for (int j = s; j < e; ++j)
          if (j != i) plain_pair<kShear>(c, a, j, xi, yi, zi, vxi, vyi, vzi, m_i, pr2_i, q);
      }
    }
  }
  // Power-law effective viscosity (world.rs:319-327).
  const uint32_t m = a.mat[i];
  const int midx = (int)m < c.n_visc_k ? (int)m : 0;
  double kc, nn;
  material_coeffs(c, midx, kc, nn);
  const double ex = __dsub_rn(nn, 1.0);
  const double sreg = q.shear > c.shear_min ? q.shear : c.shear_min;
  const double mu = __dmul_rn(kc, ex == 0.0 ? 1.0 : pow(sreg, ex));
  // acc = (f_press + f_visc_raw * mu) / rho_i if rho_i > 0 (329-336).
  double ax = 0.0, ay = 0.0, az = 0.0;
  if (rho_i > 0.0) {
    ax = __ddiv_rn(__dadd_rn(q.fpx, __dmul_rn(q.fvx, mu)), rho_i);
    ay = __ddiv_rn(__dadd_rn(q.fpy, __dmul_rn(q.fvy, mu)), rho_i);
    az = __ddiv_rn(__dadd_rn(q.fpz, __dmul_rn(q.fvz, mu)), rho_i);
  }
  a.acc[0][i] = ax;
  a.acc[1][i] = ay;
  a.acc[2][i] = az;
  a.xsph[0][i] = q.xsx;
  a.xsph[1][i] = q.xsy;
  a.xsph[2][i] = q.xsz;
  a.mu[i] = mu;
  if (a.shear_out) {
    a.fv_out[0][i] = q.fvx;
    a.fv_out[1][i] = q.fvy;
    a.fv_out[2][i] = q.fvz;
    a.shear_out[i] = q.shear;
  }
  // integrate (352-363): a = (acc + g) + body_acc; v += a dt; v += xsph eps; x += v dt.
  double bx = 0.0, by = 0.0, bz = 0.0;
  if (a.bax) {
    bx = a.bax[i];
    by = a.bay[i];
    bz = a.baz[i];
    a.bax[i] = 0.0;
    a.bay[i] = 0.0;
    a.baz[i] = 0.0;
  }
  double p3[3] = {xi, yi, zi};
  double v3[3] = {vxi, vyi, vzi};
  const double acc3[3] = {ax, ay, az};
  const double xs3[3] = {q.xsx, q.xsy, q.xsz};
  const double b3[3] = {bx, by, bz};
  bool finite = true;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double ak = __dadd_rn(__dadd_rn(acc3[k], c.g[k]), b3[k]);
    double v = __dadd_rn(v3[k], __dmul_rn(ak, c.dt));
    v = __dadd_rn(v, __dmul_rn(xs3[k], c.xsph_eps));
    double x = __dadd_rn(p3[k], __dmul_rn(v, c.dt));
    // enforce_bounds: clamp and reflect with damping.
    if (x < c.lo[k]) {
      x = c.lo[k];
      v = __dmul_rn(-v, c.damp);
    } else if (x > c.hi[k]) {
      x = c.hi[k];
      v = __dmul_rn(-v, c.damp);
    }
    finite = finite && isfinite(x) && isfinite(v);
    p3[k] = x;
    v3[k] = v;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    a.out_pv[k][i] = p3[k];
    a.out_pv[3 + k][i] = v3[k];
  }
  if (!finite) atomicOr(a.flags, kFlagNonFinite);
}

}  // namespace

void launch_plain_passes(const StepConsts& c, DevBuffers& b, cudaStream_t s, const PassEvents& ev) {
  const ParticleConsts& pc = b.pc[b.cur];
  PlainArgs a;
  a.px = b.pv0[0];
  a.py = b.pv0[1];
  a.pz = b.pv0[2];
  a.vx = b.pv0[3];
  a.vy = b.pv0[4];
  a.vz = b.pv0[5];
  a.mass = pc.mass;
  a.mat = pc.mat;
  a.cell_start = b.cell_start;
  a.bax = b.has_ba ? pc.ba[0] : nullptr;
  a.bay = b.has_ba ? pc.ba[1] : nullptr;
  a.baz = b.has_ba ? pc.ba[2] : nullptr;
  a.rho = b.rho;
  a.p = b.p;
  a.pr2 = b.pr2;
  a.mr = b.mr;
  for (int k = 0; k < 3; ++k) {
    a.acc[k] = b.acc[k];
    a.xsph[k] = b.xsph[k];
  }
  a.mu = b.mu;
  for (int k = 0; k < 6; ++k) a.out_pv[k] = b.pv1[k];
  a.nbr = b.nbr;
  a.nbr_count = b.nbr_count;
  a.stride = b.capacity;
  a.flags = b.flags;
  a.counters = b.counters;
  for (int k = 0; k < 3; ++k) a.fv_out[k] = b.tape_fv[k];
  a.shear_out = b.tape_shear;
  const int grid = (c.n + kThreads - 1) / kThreads;
  if (ev.after_prep) cudaEventRecord(ev.after_prep, s);
  if (a.counters)
    k_density_plain<true><<<grid, kThreads, 0, s>>>(c, a);
  else
    k_density_plain<false><<<grid, kThreads, 0, s>>>(c, a);
  if (ev.after_density) cudaEventRecord(ev.after_density, s);
  if (c.shear_live)
    k_force_plain<true><<<grid, kThreads, 0, s>>>(c, a);
  else
    k_force_plain<false><<<grid, kThreads, 0, s>>>(c, a);
}

}  // namespace phy
