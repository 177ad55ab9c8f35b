// Reverse-mode adjoint of the f64 plain SPH step
// (FluidWorld<f64>::step, crates/phy-fluid/src/sph/world.rs:183-397).
//
// The forward step of one particle i (d = x_j - x_i, r = |d|, u = d / r,
// dv = v_j - v_i, j over the step's neighbours with 0 < r < h):
//   rho_i   = sum_{r<h} m_j W(r)                       (self included)
//   p_i     = k max(0, rho_i - rho0),  pi_i = p_i / rho_i^2
//   fp_i    = sum u m_i m_j (pi_i + pi_j) G(r)          G = spiky gradient
//   fv_i    = sum dv m_i m_j / rho_j L(r)               L = viscosity Laplacian
//   xs_i    = sum dv m_j / rho_j W(r)
//   s_i     = sum |dv| / (r + 1e-4) m_j / rho_j
//   mu_i    = visc_k[m] max(s_i, shear_min)^(n-1)
//   acc_i   = (fp_i + fv_i mu_i) / rho_i
//   v'      = v + ((acc + g) + b) dt + xs eps;  x' = x + v' dt;  walls clamp
//             x' and reflect v' with damping.
// The reverse sweep holds the step's neighbour sets and every branch (wall
// contacts, max(0, .), shear_min) fixed, as the forward took them, and is
// exact for that piecewise-smooth map.
//
// Gradient flow (one reverse step, all arrays in the step's sorted order):
//   k_adj_integrate   dL/dx', dL/dv' -> direct dL/dx, dL/dv, the seeds of the
//                     pair sums (dL/dfp, dL/dfv, dL/dxs, dL/ds), the direct
//                     dL/drho and the visc_k[0] term;
//   k_adj_force       for each particle i, over its neighbours j, the
//                     derivatives of i's own pair terms (i's seeds) and of j's
//                     pair terms that involve i (j's seeds) — the neighbour
//                     relation is symmetric, so every contribution to i is
//                     gathered by i and no atomics are needed; its epilogue
//                     closes dL/drho_i through pi_i and p_i and the stiffness
//                     term;
//   k_adj_density     the density sums: dL/dx_i += sum W'(r) (x_i - x_j) / r
//                     (m_j dL/drho_i + m_i dL/drho_j), then the scatter back to
//                     insertion order.
// The parameter gradients are per-particle terms summed by a fixed-order
// reduction, so a gradient repeats bit-exactly run to run.
//
// The forward quantities the reverse needs (sorted state, rho, p, pi, m/rho,
// acc, xsph, mu, fv and s, the cell ranges) are recorded by re-running the
// forward step from checkpoints; the wall decisions are recomputed here with
// the forward's exact operation order.
#include <cuda_runtime.h>

#include "adjoint.h"

namespace phy {

namespace {

constexpr int kThreads = 128;
constexpr double kShearEps = 1e-4;  // world.rs:259 (r + 1e-4 in the strain proxy)

__device__ __forceinline__ double norm2(double x, double y, double z) {
  return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

// Kernel values and radial derivatives at r (< h0; zero beyond, as the
// forward's kernels).
struct KernelDerivs {
  double G, Gp, L, Lp, W, Wp;
};

__device__ __forceinline__ KernelDerivs kernel_derivs(const StepConsts& c, double r) {
  KernelDerivs k;
  if (r >= c.h0) {
    k.G = k.Gp = k.L = k.Lp = k.W = k.Wp = 0.0;
    return k;
  }
  const double hr = c.h0 - r;
  const double q = c.h0sq - r * r;
  k.G = c.spiky_c * hr * hr;
  k.Gp = -2.0 * c.spiky_c * hr;
  k.L = c.lap_c * hr;
  k.Lp = -c.lap_c;
  k.W = c.poly6_c * q * q * q;
  k.Wp = -6.0 * c.poly6_c * r * q * q;
  return k;
}

__global__ void __launch_bounds__(kThreads) k_adj_integrate(StepConsts c, AdjTape t, AdjWork w) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= c.n) return;
  const uint32_t ins = t.id[s];
  const double x3[3] = {t.x[0][s], t.x[1][s], t.x[2][s]};
  const double v3[3] = {t.v[0][s], t.v[1][s], t.v[2][s]};
  const double acc3[3] = {t.acc[0][s], t.acc[1][s], t.acc[2][s]};
  const double xs3[3] = {t.xsph[0][s], t.xsph[1][s], t.xsph[2][s]};
  double accb[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    // The forward's integrate and enforce_bounds, operation for operation, to
    // recover the wall decision (body accelerations are zero on a tape).
    const double ak = __dadd_rn(__dadd_rn(acc3[a], c.g[a]), 0.0);
    double v = __dadd_rn(v3[a], __dmul_rn(ak, c.dt));
    v = __dadd_rn(v, __dmul_rn(xs3[a], c.xsph_eps));
    const double x = __dadd_rn(x3[a], __dmul_rn(v, c.dt));
    const bool wall = x < c.lo[a] || x > c.hi[a];
    const double xb_out = w.gx_ins[a][ins], vb_out = w.gv_ins[a][ins];
    const double xb1 = wall ? 0.0 : xb_out;
    double vb2 = wall ? -c.damp * vb_out : vb_out;
    vb2 += xb1 * c.dt;
    w.gx[a][s] = xb1;
    w.gv[a][s] = vb2;
    w.Y[a][s] = vb2 * c.xsph_eps;
    accb[a] = vb2 * c.dt;
  }
  const double rho = t.rho[s], mu = t.mu[s];
  double rbar = 0.0, mub = 0.0;
  if (rho > 0.0) {
    const double inv = 1.0 / rho;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      w.P[a][s] = accb[a] * inv;
      w.Q[a][s] = accb[a] * mu * inv;
      mub += accb[a] * t.fv[a][s] * inv;
      rbar -= accb[a] * acc3[a] * inv;
    }
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      w.P[a][s] = 0.0;
      w.Q[a][s] = 0.0;
    }
  }
  // mu = kc * (n == 1 ? 1 : max(s, shear_min)^(n-1))  (world.rs:319-327)
  const uint32_t m = t.mat[s];
  const int midx = (int)m < c.n_visc_k ? (int)m : 0;
  double kc, nn;
  material_coeffs(c, midx, kc, nn);
  const double ex = nn - 1.0;
  const double shear = t.shear[s];
  const double sreg = shear > c.shear_min ? shear : c.shear_min;
  const double fac = ex == 0.0 ? 1.0 : pow(sreg, ex);
  w.cc[s] = midx == 0 ? mub * fac : 0.0;
  w.sig[s] = (ex != 0.0 && shear > c.shear_min) ? mub * kc * ex * pow(sreg, ex - 1.0) : 0.0;
  w.rbar[s] = rbar;
}

// Lanes per particle of the pair kernels: a particle's neighbours are dealt
// round-robin to kLanes consecutive lanes of a warp, whose partial sums are
// then combined by a fixed shuffle tree (deterministic).
constexpr int kLanes = 4;

// Visits lane `q`'s share of the step's force/density neighbours of slot i:
// its recorded list, or the 27 cells when the list overflowed (and, for a
// particle outside the grid box, nothing).  `f(j)` applies the pair tests.
template <class F>
__device__ __forceinline__ void for_each_listed(const StepConsts& c, const AdjTape& t, int i, int q, double xi,
                                                double yi, double zi, F&& f) {
  const uint32_t cnt = t.nbr_count[i];
  if (cnt <= (uint32_t)kMaxNeighbors) {
    for (uint32_t k = q; k < cnt; k += kLanes) f((int)t.nbr[(size_t)k * c.n + i]);
    return;
  }
  const long long kx = key_axis(xi, c.inv_cell), ky = key_axis(yi, c.inv_cell), kz = key_axis(zi, c.inv_cell);
  if (!cell_interior(c, kx, ky, kz)) return;
  const int base = cell_linear(c, kx - 1, ky - 1, kz - 1);
  for (int di = 0; di < 3; ++di)
    for (int dj = 0; dj < 3; ++dj) {
      const int c0 = base + (di * c.ncy + dj) * c.ncz;
      const int s0 = (int)t.cell_start[c0], e0 = (int)t.cell_start[c0 + 3];
      for (int j = s0 + q; j < e0; j += kLanes)
        if (j != i) f(j);
    }
}

// Sum over the kLanes lanes of a particle (all lanes receive the total).
__device__ __forceinline__ double lane_sum(double v) {
#pragma unroll
  for (int o = 1; o < kLanes; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(kThreads) k_adj_force(StepConsts c, AdjTape t, AdjWork w) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = g / kLanes, q = g % kLanes;
  const bool live = i < c.n;  // whole particles per warp: kLanes divides 32
  const int ii = live ? i : 0;
  const double xi = t.x[0][ii], yi = t.x[1][ii], zi = t.x[2][ii];
  const double vxi = t.v[0][ii], vyi = t.v[1][ii], vzi = t.v[2][ii];
  const double m_i = t.mass[ii], pr2_i = t.pr2[ii], mr_i = t.mr[ii];
  const double Pi[3] = {w.P[0][ii], w.P[1][ii], w.P[2][ii]};
  const double Qi[3] = {w.Q[0][ii], w.Q[1][ii], w.Q[2][ii]};
  const double Yi[3] = {w.Y[0][ii], w.Y[1][ii], w.Y[2][ii]};
  const double sig_i = w.sig[ii];
  double gx[3] = {0.0, 0.0, 0.0}, gv[3] = {0.0, 0.0, 0.0};
  double pibar = 0.0, rsum = 0.0;
  if (live) for_each_listed(c, t, i, q, xi, yi, zi, [&](int j) {
    // The forward's neighbour test (d = p_j - p_i, world.rs:295-299).
    const double d[3] = {__dsub_rn(t.x[0][j], xi), __dsub_rn(t.x[1][j], yi), __dsub_rn(t.x[2][j], zi)};
    const double r2 = norm2(d[0], d[1], d[2]);
    if (r2 > c.r2_guard) return;
    const double r = __dsqrt_rn(r2);
    if (r >= c.h || r <= 0.0) return;
    const KernelDerivs k = kernel_derivs(c, r);
    const double inv_r = __drcp_rn(r);
    const double u[3] = {d[0] * inv_r, d[1] * inv_r, d[2] * inv_r};
    const double dv[3] = {t.v[0][j] - vxi, t.v[1][j] - vyi, t.v[2][j] - vzi};
    const double dv2 = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
    const double inv_dvn = dv2 > 0.0 ? rsqrt(dv2) : 0.0;
    const double dvn = dv2 * inv_dvn;
    const double m_j = t.mass[j], mr_j = t.mr[j];
    const double mm = m_i * m_j;
    const double A = mm * (pr2_i + t.pr2[j]);
    const double inv_re = __drcp_rn(r + kShearEps);
    const double Pj[3] = {w.P[0][j], w.P[1][j], w.P[2][j]};
    const double Qj[3] = {w.Q[0][j], w.Q[1][j], w.Q[2][j]};
    const double Yj[3] = {w.Y[0][j], w.Y[1][j], w.Y[2][j]};
    const double sig_j = w.sig[j];
    // Own terms (i's seeds): variables d, dv, pi_i, pi_j, rho_j.
    const double uP = u[0] * Pi[0] + u[1] * Pi[1] + u[2] * Pi[2];
    const double dvQ = dv[0] * Qi[0] + dv[1] * Qi[1] + dv[2] * Qi[2];
    const double dvY = dv[0] * Yi[0] + dv[1] * Yi[1] + dv[2] * Yi[2];
    const double B = m_i * mr_j;  // m_i m_j / rho_j
    const double AGr = A * k.G * inv_r;
    const double radial_own = (A * k.Gp - AGr) * uP + dvQ * B * k.Lp + dvY * mr_j * k.Wp -
                              sig_i * dvn * mr_j * inv_re * inv_re;
    const double sv_own = sig_i * mr_j * inv_re * inv_dvn;
    // Cross terms (j's seeds; from j's side d' = -d, u' = -u, dv' = -dv, and
    // rho_i is the neighbour density).
    const double uPj = -(u[0] * Pj[0] + u[1] * Pj[1] + u[2] * Pj[2]);
    const double dvQj = -(dv[0] * Qj[0] + dv[1] * Qj[1] + dv[2] * Qj[2]);
    const double dvYj = -(dv[0] * Yj[0] + dv[1] * Yj[1] + dv[2] * Yj[2]);
    const double Bi = m_j * mr_i;  // m_i m_j / rho_i
    const double radial_x = (A * k.Gp - AGr) * uPj + dvQj * Bi * k.Lp + dvYj * mr_i * k.Wp -
                            sig_j * dvn * mr_i * inv_re * inv_re;
    const double sv_x = sig_j * mr_i * inv_re * inv_dvn;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      // d(own)/d d and d(own)/d dv; x_i enters d with a minus sign.
      const double gd_own = radial_own * u[a] + AGr * Pi[a];
      const double gdv_own = Qi[a] * B * k.L + Yi[a] * mr_j * k.W + sv_own * dv[a];
      // d(cross)/d d' (u' = -u) and d(cross)/d dv' (dv' = -dv); x_i enters d' with a plus sign.
      const double gd_x = -radial_x * u[a] + AGr * Pj[a];
      const double gdv_x = Qj[a] * Bi * k.L + Yj[a] * mr_i * k.W - sv_x * dv[a];
      gx[a] += gd_x - gd_own;
      gv[a] += gdv_x - gdv_own;
    }
    pibar += mm * k.G * (uP + uPj);
    // d/d rho_i of j's terms, times rho_i^2 (divided once below).
    rsum += dvQj * mm * k.L + dvYj * m_i * k.W + sig_j * dvn * m_i * inv_re;
  });
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    gx[a] = lane_sum(gx[a]);
    gv[a] = lane_sum(gv[a]);
  }
  pibar = lane_sum(pibar);
  rsum = lane_sum(rsum);
  if (!live || q != 0) return;
  // pi_i = p_i / rho_i^2, p_i = k max(0, rho_i - rho0).
  const double rho_i = t.rho[i], p_i = t.p[i];
  const double inv_r2 = 1.0 / (rho_i * rho_i);
  const double pbar = pibar * inv_r2;
  double rbar = w.rbar[i] - rsum * inv_r2 - 2.0 * pibar * p_i * inv_r2 / rho_i;
  const double over = rho_i - c.rest;
  double kk = 0.0;
  if (over > 0.0) {
    rbar += pbar * c.stiff;
    kk = pbar * over;
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    w.gx[a][i] += gx[a];
    w.gv[a][i] += gv[a];
  }
  w.rbar_tot[i] = rbar;
  w.kk[i] = kk;
}

__global__ void __launch_bounds__(kThreads) k_adj_density(StepConsts c, AdjTape t, AdjWork w) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = g / kLanes, q = g % kLanes;
  const bool live = i < c.n;
  const int ii = live ? i : 0;
  const double xi = t.x[0][ii], yi = t.x[1][ii], zi = t.x[2][ii];
  const double m_i = t.mass[ii], rb_i = w.rbar_tot[ii];
  double gd[3] = {0.0, 0.0, 0.0};
  if (live) for_each_listed(c, t, i, q, xi, yi, zi, [&](int j) {
    // The forward's density test (p_i - p_j, world.rs:226-229); r = 0 pairs
    // (self, coincident particles) have W'(0) = 0.
    const double d[3] = {__dsub_rn(xi, t.x[0][j]), __dsub_rn(yi, t.x[1][j]), __dsub_rn(zi, t.x[2][j])};
    const double r2 = norm2(d[0], d[1], d[2]);
    if (r2 > c.r2_guard) return;
    const double r = __dsqrt_rn(r2);
    if (!(r < c.h) || r <= 0.0 || r >= c.h0) return;
    const double qq = c.h0sq - r2;
    // W'(r) / r = -6 poly6_c (h0^2 - r^2)^2
    const double f = -6.0 * c.poly6_c * qq * qq * (t.mass[j] * rb_i + m_i * w.rbar_tot[j]);
#pragma unroll
    for (int a = 0; a < 3; ++a) gd[a] += f * d[a];
  });
#pragma unroll
  for (int a = 0; a < 3; ++a) gd[a] = lane_sum(gd[a]);
  if (!live || q != 0) return;
  const uint32_t ins = t.id[i];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    w.gx_ins[a][ins] = w.gx[a][i] + gd[a];
    w.gv_ins[a][ins] = w.gv[a][i];
  }
}

// acc[0] += sum a[0..n), acc[1] += sum b[0..n): one block, fixed order.
__global__ void __launch_bounds__(1024) k_adj_sum2(int n, const double* __restrict__ a,
                                                   const double* __restrict__ b, double* acc) {
  __shared__ double sa[1024], sb[1024];
  double x = 0.0, y = 0.0;
  for (int k = threadIdx.x; k < n; k += 1024) {
    x += a[k];
    y += b[k];
  }
  sa[threadIdx.x] = x;
  sb[threadIdx.x] = y;
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      sa[threadIdx.x] += sa[threadIdx.x + o];
      sb[threadIdx.x] += sb[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    acc[0] += sa[0];
    acc[1] += sb[0];
  }
}

}  // namespace

void launch_adjoint_step(const StepConsts& c, const AdjTape& t, const AdjWork& w, cudaStream_t s) {
  if (c.n == 0) return;
  static_assert(32 % kLanes == 0, "a particle's lanes share a warp");
  const int grid = (c.n + kThreads - 1) / kThreads;
  const int pair_grid = (int)(((long long)c.n * kLanes + kThreads - 1) / kThreads);
  k_adj_integrate<<<grid, kThreads, 0, s>>>(c, t, w);
  k_adj_force<<<pair_grid, kThreads, 0, s>>>(c, t, w);
  k_adj_density<<<pair_grid, kThreads, 0, s>>>(c, t, w);
  // param_acc = {d/d stiffness, d/d visc_k[0]}
  k_adj_sum2<<<1, 1024, 0, s>>>(c.n, w.kk, w.cc, w.param_acc);
}

}  // namespace phy
