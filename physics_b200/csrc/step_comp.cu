// The FP32-compensated SPH passes.
//
// Same step as the reference's FluidWorld<f64>::step (crates/phy-fluid/src/
// sph/world.rs:183-397) with the pairwise kernel math in f32:
//   * pair geometry comes from cell-local f32 coordinates: every particle
//     stores (x - kx*h0, y - ky*h0, z - kz*h0) as floats, so a neighbour's
//     offset is (dcell * h0) + (local_j - local_i) with |local| < h0 and an
//     absolute rounding error of about h0 * 2^-24, independent of how far
//     the scene lies from the origin;
//   * density and the pressure / viscous force components are summed with
//     Kahan compensation, and rho - rho0 is formed in f64 from the
//     compensated (sum, correction) pair;
//   * cell keys, positions, velocities, integration and bounds stay f64.
// Neighbours are visited in the reference's order, so the result is
// deterministic run to run.
#include <cuda_runtime.h>

#include "sph_buffers.h"

namespace phy {

namespace {

constexpr int kThreads = 128;

__device__ __forceinline__ void kahan_add(float& s, float& c, float x) {
  float y = x - c;
  float t = s + y;
  c = (t - s) - y;
  s = t;
}

struct CompArgs {
  const double* __restrict__ px;
  const double* __restrict__ py;
  const double* __restrict__ pz;
  const double* __restrict__ vx;
  const double* __restrict__ vy;
  const double* __restrict__ vz;
  const double* __restrict__ mass;
  const uint32_t* __restrict__ mat;
  const uint32_t* __restrict__ cell_start;
  float4* cpos;
  float4* cvel;
  float* cmr;
  double* bax;
  double* bay;
  double* baz;
  double* rho;
  double* p;
  double* acc[3];
  double* xsph[3];
  double* mu;
  double* out_pv[6];
  uint32_t* nbr;
  uint32_t* nbr_count;
  int stride;
  uint32_t* flags;
  unsigned long long* counters;
};

// Cell-local f32 operands of every particle.
__global__ void __launch_bounds__(kThreads) k_prep_comp(StepConsts c, CompArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.n) return;
  const double x = a.px[i], y = a.py[i], z = a.pz[i];
  const long long kx = key_axis(x, c.inv_cell);
  const long long ky = key_axis(y, c.inv_cell);
  const long long kz = key_axis(z, c.inv_cell);
  float lx = (float)(x - (double)kx * c.h0);
  float ly = (float)(y - (double)ky * c.h0);
  float lz = (float)(z - (double)kz * c.h0);
  a.cpos[i] = make_float4(lx, ly, lz, (float)a.mass[i]);
  a.cvel[i] = make_float4((float)a.vx[i], (float)a.vy[i], (float)a.vz[i], 0.0f);
}

// Density pass.  rho_i = poly6_c * sum_j m_j (h0^2 - r^2)^3 over r < min(h, h0):
// each cell's terms are summed with plain FMAs (a handful of terms), and the
// 27 cell sums are added with Kahan compensation.  In-range neighbours (and
// NaN distances) are listed as (j << kCodeBits) | cell code, code = 9 di +
// 3 dj + dk, for the force pass (i itself included: its r^2 is exactly 0).
template <bool kCount>
__global__ void __launch_bounds__(kThreads) k_density_comp(StepConsts c, CompArgs a) {
  __shared__ uint32_t s_list[kStagedNeighbors][kThreads];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.n) return;
  const double xi = a.px[i], yi = a.py[i], zi = a.pz[i];
  const long long kx = key_axis(xi, c.inv_cell);
  const long long ky = key_axis(yi, c.inv_cell);
  const long long kz = key_axis(zi, c.inv_cell);
  const float4 pi = a.cpos[i];
  // Squared cutoff: r < h (live) and poly6's r < h0 (captured).
  const float hc2 = fminf(c.h2f, c.h0sqf);
  float s = 0.0f, comp = 0.0f;
  unsigned cand = 0, pairs = 0;
  uint32_t cnt = 0;
  uint32_t* lst = a.nbr + i;
  if (cell_interior(c, kx, ky, kz)) {
    const int base = cell_linear(c, kx - 1, ky - 1, kz - 1);
    for (int di = 0; di < 3; ++di) {
      const float ox = (float)(di - 1) * c.h0f - pi.x;
      for (int dj = 0; dj < 3; ++dj) {
        const float oy = (float)(dj - 1) * c.h0f - pi.y;
        const int c0 = base + (di * c.ncy + dj) * c.ncz;
        for (int dk = 0; dk < 3; ++dk) {
          const float oz = (float)(dk - 1) * c.h0f - pi.z;
          const uint32_t code = (uint32_t)(9 * di + 3 * dj + dk);
          const int s0 = (int)a.cell_start[c0 + dk], e0 = (int)a.cell_start[c0 + dk + 1];
          if (kCount) cand += (unsigned)(e0 - s0);
          float part = 0.0f;
          for (int j = s0; j < e0; ++j) {
            const float4 q = a.cpos[j];
            const float dx = ox + q.x, dy = oy + q.y, dz = oz + q.z;
            const float r2 = dx * dx + dy * dy + dz * dz;
            const float t = r2 < hc2 ? c.h0sqf - r2 : 0.0f;
            part = fmaf(t * t, t * q.w, part);
            if (kCount) pairs += r2 < hc2 ? 1u : 0u;
            if (!(r2 >= hc2)) {
              const uint32_t e = ((uint32_t)j << kCodeBits) | code;
              if (cnt < (uint32_t)kStagedNeighbors)
                s_list[cnt][threadIdx.x] = e;
              else if (cnt < (uint32_t)kMaxNeighbors)
                lst[(size_t)cnt * a.stride] = e;
              ++cnt;
            }
          }
          kahan_add(s, comp, c.poly6_cf * part);
        }
      }
    }
  }
  flush_staged_list<kThreads>(s_list, lst, a.stride, cnt, true);
  a.nbr_count[i] = cnt;
  const double rho = (double)s - (double)comp;
  const double over = rho - c.rest;
  const double pr = over > 0.0 ? c.stiff * over : 0.0;
  a.rho[i] = rho;
  a.p[i] = pr;
  a.cvel[i].w = (float)(pr / (rho * rho));
  a.cmr[i] = (float)(a.mass[i] / rho);
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

struct CompAcc {
  float fpx = 0.f, fpy = 0.f, fpz = 0.f, cpx = 0.f, cpy = 0.f, cpz = 0.f;
  float fvx = 0.f, fvy = 0.f, fvz = 0.f, cvx = 0.f, cvy = 0.f, cvz = 0.f;
  float xsx = 0.f, xsy = 0.f, xsz = 0.f, shear = 0.f;
};

// One neighbour: d = offset of j's cell + (local_j - local_i).
__device__ __forceinline__ void comp_pair(const StepConsts& c, const CompArgs& a, int j, float dx, float dy,
                                          float dz, float m_j, float4 vi, float m_i, float pr2_i, CompAcc& q) {
  const float r2 = dx * dx + dy * dy + dz * dz;
  if (!(r2 < fminf(c.h2f, c.h0sqf)) || r2 <= 0.0f) return;
  const float4 vj = a.cvel[j];
  const float mr_j = a.cmr[j];
  const float inv_r = rsqrtf(r2);
  const float r = r2 * inv_r;
  const float hr = c.h0f - r;
  // Symmetric pressure: (d/r) * (m_i m_j (p_i/rho_i^2 + p_j/rho_j^2) * spiky(r)).
  const float fp = (m_i * m_j) * (pr2_i + vj.w) * (c.spiky_cf * hr * hr) * inv_r;
  kahan_add(q.fpx, q.cpx, dx * fp);
  kahan_add(q.fpy, q.cpy, dy * fp);
  kahan_add(q.fpz, q.cpz, dz * fp);
  // Viscosity (raw, mu applied later): dv * (m_i m_j / rho_j * lap(r)).
  const float dvx = vj.x - vi.x, dvy = vj.y - vi.y, dvz = vj.z - vi.z;
  const float vf = m_i * mr_j * (c.lap_cf * hr);
  kahan_add(q.fvx, q.cvx, dvx * vf);
  kahan_add(q.fvy, q.cvy, dvy * vf);
  kahan_add(q.fvz, q.cvz, dvz * vf);
  // XSPH: dv * (m_j/rho_j * poly6(r)).
  const float t = c.h0sqf - r2;
  const float xw = mr_j * (c.poly6_cf * t * t * t);
  q.xsx += dvx * xw;
  q.xsy += dvy * xw;
  q.xsz += dvz * xw;
  // Strain-rate proxy: |dv| / (r + 1e-4) * m_j/rho_j.
  const float dvn = sqrtf(dvx * dvx + dvy * dvy + dvz * dvz);
  q.shear += __fdividef(dvn, r + 1e-4f) * mr_j;
}

__global__ void __launch_bounds__(kThreads) k_force_comp(StepConsts c, CompArgs a) {
  __shared__ float4 s_off[27];  // cell offsets (di-1, dj-1, dk-1) * h0
  if (threadIdx.x < 27) {
    const int t = threadIdx.x;
    s_off[t] = make_float4((float)(t / 9 - 1) * c.h0f, (float)((t / 3) % 3 - 1) * c.h0f,
                           (float)(t % 3 - 1) * c.h0f, 0.f);
  }
  __syncthreads();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.n) return;
  const double xi = a.px[i], yi = a.py[i], zi = a.pz[i];
  const double vxi = a.vx[i], vyi = a.vy[i], vzi = a.vz[i];
  const double rho_i = a.rho[i];
  const float4 pi = a.cpos[i];
  const float4 vi = a.cvel[i];
  const float m_i = pi.w, pr2_i = vi.w;
  CompAcc q;
  const uint32_t cnt = a.nbr_count[i];
  if (cnt <= (uint32_t)kMaxNeighbors) {
    const uint32_t* lst = a.nbr + i;
    for (uint32_t k = 0; k < cnt; ++k) {
      const uint32_t e = lst[(size_t)k * a.stride];
      const int j = (int)(e >> kCodeBits);
      const float4 off = s_off[e & ((1u << kCodeBits) - 1u)];
      const float4 pj = a.cpos[j];
      comp_pair(c, a, j, (off.x - pi.x) + pj.x, (off.y - pi.y) + pj.y, (off.z - pi.z) + pj.z, pj.w, vi, m_i,
                pr2_i, q);
    }
  } else {
    const long long kx = key_axis(xi, c.inv_cell);
    const long long ky = key_axis(yi, c.inv_cell);
    const long long kz = key_axis(zi, c.inv_cell);
    const int base = cell_linear(c, kx - 1, ky - 1, kz - 1);
    for (int di = 0; di < 3; ++di) {
      for (int dj = 0; dj < 3; ++dj) {
        const int c0 = base + (di * c.ncy + dj) * c.ncz;
        for (int dk = 0; dk < 3; ++dk) {
          const float4 off = s_off[9 * di + 3 * dj + dk];
          const int s0 = (int)a.cell_start[c0 + dk], e0 = (int)a.cell_start[c0 + dk + 1];
          for (int j = s0; j < e0; ++j) {
            if (j == i) continue;
            const float4 pj = a.cpos[j];
            comp_pair(c, a, j, (off.x - pi.x) + pj.x, (off.y - pi.y) + pj.y, (off.z - pi.z) + pj.z, pj.w, vi,
                      m_i, pr2_i, q);
          }
        }
      }
    }
  }
  const uint32_t m = a.mat[i];
  const int midx = (int)m < c.n_visc_k ? (int)m : 0;
  double kc, nn;
  material_coeffs(c, midx, kc, nn);
  const double ex = nn - 1.0;
  const double sh = (double)q.shear;
  const double sreg = sh > c.shear_min ? sh : c.shear_min;
  const double mu = kc * (ex == 0.0 ? 1.0 : pow(sreg, ex));
  double ax = 0.0, ay = 0.0, az = 0.0;
  if (rho_i > 0.0) {
    const double fx = ((double)q.fpx - (double)q.cpx) + ((double)q.fvx - (double)q.cvx) * mu;
    const double fy = ((double)q.fpy - (double)q.cpy) + ((double)q.fvy - (double)q.cvy) * mu;
    const double fz = ((double)q.fpz - (double)q.cpz) + ((double)q.fvz - (double)q.cvz) * mu;
    ax = fx / rho_i;
    ay = fy / rho_i;
    az = fz / rho_i;
  }
  a.acc[0][i] = ax;
  a.acc[1][i] = ay;
  a.acc[2][i] = az;
  a.xsph[0][i] = q.xsx;
  a.xsph[1][i] = q.xsy;
  a.xsph[2][i] = q.xsz;
  a.mu[i] = mu;
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
  const double xs3[3] = {(double)q.xsx, (double)q.xsy, (double)q.xsz};
  const double b3[3] = {bx, by, bz};
  bool finite = true;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double ak = (acc3[k] + c.g[k]) + b3[k];
    double v = v3[k] + ak * c.dt;
    v = v + xs3[k] * c.xsph_eps;
    double x = p3[k] + v * c.dt;
    if (x < c.lo[k]) {
      x = c.lo[k];
      v = -v * c.damp;
    } else if (x > c.hi[k]) {
      x = c.hi[k];
      v = -v * c.damp;
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

void launch_comp_passes(const StepConsts& c, DevBuffers& b, cudaStream_t s, const PassEvents& ev) {
  const ParticleConsts& pc = b.pc[b.cur];
  CompArgs a;
  a.px = b.pv0[0];
  a.py = b.pv0[1];
  a.pz = b.pv0[2];
  a.vx = b.pv0[3];
  a.vy = b.pv0[4];
  a.vz = b.pv0[5];
  a.mass = pc.mass;
  a.mat = pc.mat;
  a.cell_start = b.cell_start;
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
  a.nbr = b.nbr;
  a.nbr_count = b.nbr_count;
  a.stride = b.capacity;
  a.flags = b.flags;
  a.counters = b.counters;
  const int grid = (c.n + kThreads - 1) / kThreads;
  k_prep_comp<<<grid, kThreads, 0, s>>>(c, a);
  if (ev.after_prep) cudaEventRecord(ev.after_prep, s);
  if (a.counters)
    k_density_comp<true><<<grid, kThreads, 0, s>>>(c, a);
  else
    k_density_comp<false><<<grid, kThreads, 0, s>>>(c, a);
  if (ev.after_density) cudaEventRecord(ev.after_density, s);
  k_force_comp<<<grid, kThreads, 0, s>>>(c, a);
}

}  // namespace phy
