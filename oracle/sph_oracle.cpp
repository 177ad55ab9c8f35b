// TEST INFRASTRUCTURE ONLY — the CPU oracle for the SPH fluid step.
//
// This file restates, in plain C++17, the reference's weakly-compressible SPH
// step `FluidWorld<T>::step` (jojo240607/physics, crate phy-fluid) so that the
// CUDA product can be checked against it.  It is never linked into the
// product library and nothing in `physics_b200/` loads it; only the tests,
// `__graft_entry__.smoke()` and the CPU-baseline leg of `bench.py` do.
//
// Parity status: the reference is Rust and cannot be compiled here (no
// cargo/rustc, crates not vendored), and its own tests hold no golden vectors
// for this path.  The restatement is therefore pinned only against the
// reference's property tests and the analytic known answers derivable from
// its definitions (see tests/test_oracle.py) — parity against
// reference-generated outputs is UNPINNED.
//
// Arithmetic contract (follows the reference expression by expression):
//   * no FMA contraction (build with -ffp-contract=off), IEEE division/sqrt;
//   * evaluation order left-to-right exactly as the Rust source groups it;
//   * |v| = sqrt((x*x + y*y) + z*z): nalgebra 0.33.3 `Matrix::norm` =
//     `norm_squared().sqrt()`, and its `dotx` special-cases 3-vectors as
//     `a + b + c` of the component products (nalgebra is a crates.io
//     dependency, absent here; this is its published algorithm);
//   * neighbour visit order: 27 cells with di outermost, dk innermost, and the
//     particles of a cell in ascending insertion index (HashMap of Vec pushed
//     in index order).
//
// The density and force passes optionally run on OpenMP threads, mirroring the
// reference's rayon per-particle maps; results do not depend on the thread
// count because every particle's reduction is sequential and write-disjoint.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;  // std::f64::consts::PI

struct V3 {
  double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3& operator+=(V3& a, V3 b) {
  a.x = a.x + b.x;
  a.y = a.y + b.y;
  a.z = a.z + b.z;
  return a;
}
// nalgebra Vector3::norm (see header).
inline double norm(V3 a) { return std::sqrt((a.x * a.x + a.y * a.y) + a.z * a.z); }
inline double norm_squared(V3 a) { return (a.x * a.x + a.y * a.y) + a.z * a.z; }

}  // namespace

extern "C" {

// Same field layout as `PhySphParams` in include/phy_fluid.h.
// Mirrors SphParams<T> (crates/phy-fluid/src/sph/params.rs:12-86).
struct OrcParams {
  double rest_density, stiffness, viscosity, shear_min, mass, h;
  double gravity[3], bounds_min[3], bounds_max[3];
  double boundary_damp, xsph_eps;
  uint32_t n_visc_k, n_visc_n;
  double visc_k[16], visc_n[16];
};

}  // extern "C"

namespace {

// Particle<T> (crates/phy-fluid/src/particle.rs:17-46).
struct Particle {
  V3 pos{0, 0, 0}, vel{0, 0, 0}, acc{0, 0, 0}, body_acc{0, 0, 0};
  double rho = 0, p = 0, mass = 0;
  uint64_t material = 0;
  double mu_eff = 0;
  V3 xsph{0, 0, 0};
};

// Kernels<T> (crates/phy-fluid/src/kernels.rs:20-66): coefficients captured from h.
struct Kernels {
  double h, h2, poly6_coeff, spiky_grad_coeff, visc_lap_coeff;
  explicit Kernels(double hh) {
    h = hh;
    h2 = hh * hh;
    double h3 = h2 * hh;
    double h6 = h3 * h3;
    double h9 = h6 * h3;
    poly6_coeff = 315.0 / (64.0 * kPi * h9);       // kernels.rs:31
    spiky_grad_coeff = (-45.0) / (kPi * h6);       // kernels.rs:32
    visc_lap_coeff = 45.0 / (kPi * h6);            // kernels.rs:33
  }
  double poly6(double r) const {  // kernels.rs:39-45
    if (r >= h) return 0.0;
    double diff = h2 - r * r;
    return poly6_coeff * diff * diff * diff;
  }
  double spiky_grad_mag(double r) const {  // kernels.rs:50-56
    if (r >= h || r <= 0.0) return 0.0;
    double diff = h - r;
    return spiky_grad_coeff * diff * diff;
  }
  double visc_lap(double r) const {  // kernels.rs:60-65
    if (r >= h) return 0.0;
    return visc_lap_coeff * (h - r);
  }
};

// num-traits `ToPrimitive::to_i64` for f64: Some only inside (-2^63, 2^63).
inline int64_t to_i64_or_zero(double v) {
  if (v > -9223372036854775808.0 && v < 9223372036854775808.0) return (int64_t)v;
  return 0;
}

struct Key {
  int64_t i, j, k;
  bool operator==(const Key& o) const { return i == o.i && j == o.j && k == o.k; }
};
struct KeyHash {
  size_t operator()(const Key& a) const {
    uint64_t h = (uint64_t)a.i * 0x9E3779B97F4A7C15ull;
    h ^= (uint64_t)a.j * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
    h ^= (uint64_t)a.k * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
    return (size_t)h;
  }
};

// Grid<T> (crates/phy-fluid/src/sph/grid.rs:10-56).
struct Grid {
  double cell;
  std::unordered_map<Key, std::vector<uint32_t>, KeyHash> map;
  explicit Grid(double c) : cell(c) {}
  Key key_of(V3 p) const {  // grid.rs:25-33
    double inv = 1.0 / cell;
    return {to_i64_or_zero(std::floor(p.x * inv)), to_i64_or_zero(std::floor(p.y * inv)),
            to_i64_or_zero(std::floor(p.z * inv))};
  }
  void build(const std::vector<Particle>& ps) {  // grid.rs:35-40
    map.clear();
    for (size_t i = 0; i < ps.size(); ++i) map[key_of(ps[i].pos)].push_back((uint32_t)i);
  }
  template <class F>
  void for_each_neighbor(V3 p, F&& f) const {  // grid.rs:43-56
    Key c = key_of(p);
    for (int64_t di = -1; di <= 1; ++di)
      for (int64_t dj = -1; dj <= 1; ++dj)
        for (int64_t dk = -1; dk <= 1; ++dk) {
          auto it = map.find(Key{c.i + di, c.j + dj, c.k + dk});
          if (it == map.end()) continue;
          for (uint32_t id : it->second) f((size_t)id);
        }
  }
};

// Per-pass counters used by the roofline accounting (candidates visited and
// pairs inside the support radius).
struct Counters {
  uint64_t candidates = 0, pairs = 0;
};

// FluidWorld<f64> (crates/phy-fluid/src/sph/world.rs:21-397).
struct World {
  OrcParams params;
  std::vector<Particle> particles;
  Kernels kernels;
  Grid grid;
  int nthreads = 1;
  Counters counters;

  explicit World(const OrcParams& p) : params(p), kernels(p.h), grid(p.h) {}  // world.rs:94-102

  // world.rs:148-169
  double lattice_mass(double s) const {
    double h = params.h;
    double hs = h / s;
    int n_shell = (int)std::ceil(hs) + 1;
    double sum_w = 0.0;
    for (int i = -n_shell; i <= n_shell; ++i)
      for (int j = -n_shell; j <= n_shell; ++j)
        for (int l = -n_shell; l <= n_shell; ++l) {
          double rr = std::sqrt((double)(i * i + j * j + l * l));
          double r = s * rr;
          if (r < h) sum_w = sum_w + kernels.poly6(r);
        }
    if (sum_w > 0.0) return params.rest_density / sum_w;
    return params.mass;
  }

  // world.rs:124-144 (float-accumulated loops, z innermost).
  void fill_box(V3 mn, V3 mx, double spacing, double margin) {
    V3 lo = mn + V3{margin, margin, margin};
    V3 hi = mx - V3{margin, margin, margin};
    double d = spacing;
    double mass = lattice_mass(d);
    double x = lo.x;
    while (x <= hi.x) {
      double y = lo.y;
      while (y <= hi.y) {
        double z = lo.z;
        while (z <= hi.z) {
          Particle pt;
          pt.pos = {x, y, z};
          pt.mass = mass;
          particles.push_back(pt);
          z = z + d;
        }
        y = y + d;
      }
      x = x + d;
    }
  }

  void step(double dt) {  // world.rs:183-192
    if (particles.empty()) return;
    grid.build(particles);
    compute_density_pressure();
    compute_forces();
    integrate(dt);
    enforce_bounds();
  }

  void compute_density_pressure() {  // world.rs:204-246
    const double h = params.h;
    const size_t n = particles.size();
    const double rest = params.rest_density, stiff = params.stiffness;
    std::vector<V3> pos(n);
    std::vector<double> mass(n);
    for (size_t i = 0; i < n; ++i) {
      pos[i] = particles[i].pos;
      mass[i] = particles[i].mass;
    }
    std::vector<double> rho_out(n), p_out(n);
    uint64_t cand = 0, pairs = 0;
#pragma omp parallel for schedule(static) num_threads(nthreads) reduction(+ : cand, pairs)
    for (long long ii = 0; ii < (long long)n; ++ii) {
      size_t i = (size_t)ii;
      V3 p_i = pos[i];
      double rho = 0.0;
      grid.for_each_neighbor(p_i, [&](size_t j) {
        double r = norm(p_i - pos[j]);  // na_distance, world.rs:777-779
        ++cand;
        if (r < h) {
          rho = rho + mass[j] * kernels.poly6(r);
          ++pairs;
        }
      });
      double over = rho - rest;
      double p = over > 0.0 ? stiff * over : 0.0;
      rho_out[i] = rho;
      p_out[i] = p;
    }
    for (size_t i = 0; i < n; ++i) {
      particles[i].rho = rho_out[i];
      particles[i].p = p_out[i];
    }
    counters.candidates += cand;
    counters.pairs += pairs;
  }

  void compute_forces() {  // world.rs:252-347
    const size_t n = particles.size();
    const double h = params.h;
    const double r_eps = 1e-4;
    const double shear_min = params.shear_min;
    std::vector<V3> pos(n), vel(n);
    std::vector<double> rho(n), pr(n), mass(n);
    std::vector<uint64_t> mat(n);
    for (size_t i = 0; i < n; ++i) {
      pos[i] = particles[i].pos;
      vel[i] = particles[i].vel;
      rho[i] = particles[i].rho;
      pr[i] = particles[i].p;
      mass[i] = particles[i].mass;
      mat[i] = particles[i].material;
    }
    std::vector<V3> acc_out(n), xsph_out(n);
    std::vector<double> mu_out(n);
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (long long ii = 0; ii < (long long)n; ++ii) {
      size_t i = (size_t)ii;
      V3 p_i = pos[i], v_i = vel[i];
      double rho_i = rho[i], p_i_p = pr[i], m_i = mass[i];
      V3 f_press{0, 0, 0}, f_visc_raw{0, 0, 0}, xsph{0, 0, 0};
      double shear = 0.0;
      grid.for_each_neighbor(p_i, [&](size_t j) {
        if (j == i) return;
        V3 d = pos[j] - p_i;
        double r = norm(d);
        if (r >= h || r <= 0.0) return;
        double rho_j = rho[j];
        double p_j = pr[j];
        double grad = kernels.spiky_grad_mag(r);
        V3 dir = d / r;
        double coef = m_i * mass[j] * (p_i_p / (rho_i * rho_i) + p_j / (rho_j * rho_j));
        f_press += dir * (coef * grad);
        double lap = kernels.visc_lap(r);
        f_visc_raw += (vel[j] - v_i) * (m_i * mass[j] / rho_j * lap);
        double w = kernels.poly6(r);
        xsph += (vel[j] - v_i) * (mass[j] / rho_j * w);
        double dv = norm(vel[j] - v_i);
        shear = shear + dv / (r + r_eps) * (mass[j] / rho_j);
      });
      // world.rs:319-327; visc_k/visc_n are indexed like Rust slices.
      uint64_t m_idx = mat[i] < params.n_visc_k ? mat[i] : 0;
      double kc = params.visc_k[m_idx];
      double nn = params.visc_n[m_idx];
      double sreg = shear > shear_min ? shear : shear_min;
      double mu_eff = kc * std::pow(sreg, nn - 1.0);
      V3 f_visc = f_visc_raw * mu_eff;
      V3 acc = rho_i > 0.0 ? (f_press + f_visc) / rho_i : V3{0, 0, 0};
      acc_out[i] = acc;
      mu_out[i] = mu_eff;
      xsph_out[i] = xsph;
    }
    for (size_t i = 0; i < n; ++i) {
      particles[i].acc = acc_out[i];
      particles[i].mu_eff = mu_out[i];
      particles[i].xsph = xsph_out[i];
    }
  }

  void integrate(double dt) {  // world.rs:352-363
    V3 g{params.gravity[0], params.gravity[1], params.gravity[2]};
    double eps = params.xsph_eps;
    for (auto& pt : particles) {
      V3 a = pt.acc + g + pt.body_acc;
      pt.vel += a * dt;
      pt.vel += pt.xsph * eps;
      pt.pos += pt.vel * dt;
      pt.body_acc = {0, 0, 0};
    }
  }

  void enforce_bounds() {  // world.rs:366-397
    const double* lo = params.bounds_min;
    const double* hi = params.bounds_max;
    double damp = params.boundary_damp;
    for (auto& pt : particles) {
      double p[3] = {pt.pos.x, pt.pos.y, pt.pos.z};
      double v[3] = {pt.vel.x, pt.vel.y, pt.vel.z};
      for (int a = 0; a < 3; ++a) {
        if (p[a] < lo[a]) {
          p[a] = lo[a];
          v[a] = -v[a] * damp;
        } else if (p[a] > hi[a]) {
          p[a] = hi[a];
          v[a] = -v[a] * damp;
        }
      }
      pt.pos = {p[0], p[1], p[2]};
      pt.vel = {v[0], v[1], v[2]};
    }
  }

  // world.rs:555-678 against a heat grid (HeatFieldLike of phy-field):
  // trilinear temperature -> body_acc += -g * beta * (T - t_ref) for the
  // particles inside the bounds, and heat_gain * |v| * dt added to the
  // source of the particle's cell, particle after particle.  (The reference
  // also installs a velocity sampler closure into the field; that part
  // belongs to the field's own step.)
  struct HeatGrid {
    uint64_t nx, ny, nz;
    V3 origin;
    double dx;
    const double* u;
    double* src;
    uint64_t idx(uint64_t x, uint64_t y, uint64_t z) const { return x + nx * (y + ny * z); }  // grid.rs:80-82
    double sample(uint64_t x, uint64_t y, uint64_t z) const {  // grid.rs:203-208
      return u[idx(x < nx - 1 ? x : nx - 1, y < ny - 1 ? y : ny - 1, z < nz - 1 ? z : nz - 1)];
    }
    double sample_trilinear(uint64_t cx, uint64_t cy, uint64_t cz, double fx, double fy, double fz) const {
      // heat.rs:130-171
      const uint64_t x1 = cx + 1 < nx - 1 ? cx + 1 : nx - 1, y1 = cy + 1 < ny - 1 ? cy + 1 : ny - 1,
                     z1 = cz + 1 < nz - 1 ? cz + 1 : nz - 1;
      const double c000 = sample(cx, cy, cz), c100 = sample(x1, cy, cz), c010 = sample(cx, y1, cz),
                   c110 = sample(x1, y1, cz), c001 = sample(cx, cy, z1), c101 = sample(x1, cy, z1),
                   c011 = sample(cx, y1, z1), c111 = sample(x1, y1, z1);
      const double x00 = c000 + (c100 - c000) * fx;
      const double x10 = c010 + (c110 - c010) * fx;
      const double x01 = c001 + (c101 - c001) * fx;
      const double x11 = c011 + (c111 - c011) * fx;
      const double y0 = x00 + (x10 - x00) * fy;
      const double y1v = x01 + (x11 - x01) * fy;
      return y0 + (y1v - y0) * fz;
    }
    void add_source(uint64_t x, uint64_t y, uint64_t z, double v) {  // grid.rs:125-130
      if (x < nx && y < ny && z < nz) src[idx(x, y, z)] = src[idx(x, y, z)] + v;
    }
  };

  // num-traits ToPrimitive::to_usize of an f64 with None -> 0.
  static uint64_t to_usize_or_zero(double f) {
    return (f > -1.0 && f < 18446744073709551616.0) ? (uint64_t)f : 0;
  }

  void couple_heat(HeatGrid& heat, double dt, double t_ref, double beta, double heat_gain) {
    if (particles.empty()) return;
    const V3 g{params.gravity[0], params.gravity[1], params.gravity[2]};
    const double* lo = params.bounds_min;
    const double* hi = params.bounds_max;
    const V3 hmin = heat.origin;
    const double dx = heat.dx;
    // dims.saturating_sub(1) as T
    const double nxm1 = heat.nx > 0 ? (double)(heat.nx - 1) : 0.0, nym1 = heat.ny > 0 ? (double)(heat.ny - 1) : 0.0,
                 nzm1 = heat.nz > 0 ? (double)(heat.nz - 1) : 0.0;
    auto to_idx = [&](V3 p, uint64_t* c, double* t) {  // world.rs:577-598
      if (p.x < hmin.x || p.x > hmin.x + dx * nxm1 || p.y < hmin.y || p.y > hmin.y + dx * nym1 || p.z < hmin.z ||
          p.z > hmin.z + dx * nzm1)
        return false;
      const double fx = std::floor((p.x - hmin.x) / dx), fy = std::floor((p.y - hmin.y) / dx),
                   fz = std::floor((p.z - hmin.z) / dx);
      c[0] = to_usize_or_zero(fx);
      c[1] = to_usize_or_zero(fy);
      c[2] = to_usize_or_zero(fz);
      t[0] = (p.x - hmin.x) / dx - fx;
      t[1] = (p.y - hmin.y) / dx - fy;
      t[2] = (p.z - hmin.z) / dx - fz;
      return true;
    };
    for (auto& pt : particles) {
      const V3 p = pt.pos;
      if (p.x < lo[0] || p.x > hi[0] || p.y < lo[1] || p.y > hi[1] || p.z < lo[2] || p.z > hi[2]) continue;
      uint64_t c[3];
      double t[3];
      const double temp = to_idx(p, c, t) ? heat.sample_trilinear(c[0], c[1], c[2], t[0], t[1], t[2]) : t_ref;
      const double dT = temp - t_ref;
      pt.body_acc += V3{-g.x * beta * dT, -g.y * beta * dT, -g.z * beta * dT};
      if (heat_gain > 0.0) {
        const double speed = norm(pt.vel);
        if (to_idx(p, c, t)) heat.add_source(c[0], c[1], c[2], heat_gain * speed * dt);
      }
    }
  }

  // Rigid bodies for couple_bodies (phy-rigid shape.rs:138-372): the pose
  // (pos, unit quaternion rot = (i, j, k, w) as nalgebra stores it), the
  // linear velocity, inv_mass, and the shape: 0 sphere {r}, 1 capsule
  // {half_height, r} along local y, 2 box {half extents}, 3 convex (vertices,
  // index faces), 4 heightfield {nx, nz, cell} + heights, 5 compound: sub
  // shapes (shape.rs:176-192), each with its own offset and rotation
  // relative to the body (the sub shapes' own pose fields).
  struct Body {
    int shape = 0;
    double size[3] = {0, 0, 0};
    V3 pos{0, 0, 0};
    double rot[4] = {0, 0, 0, 1};
    V3 vel{0, 0, 0};
    double inv_mass = 0;
    std::vector<V3> verts;
    std::vector<uint32_t> faces;  // 3 per face, indices into verts
    std::vector<double> heights;
    std::vector<Body> subs;  // compound: sub shapes, pos = offset, rot = quat
  };

  static double dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
  static V3 cross(V3 a, V3 b) {  // nalgebra Vector3::cross
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
  }
  static V3 normalize(V3 a) { return a / norm(a); }
  // nalgebra 0.33.3 UnitQuaternion * Vector3 (its published formula):
  // t = 2 (q.v x v); q v = (t * q.w + q.v x t) + v.  inverse() is the
  // conjugate.
  static V3 qrot(const double* q, V3 v, bool inverse) {
    const double s = inverse ? -1.0 : 1.0;
    const V3 u{s * q[0], s * q[1], s * q[2]};
    const V3 t = cross(u, v) * 2.0;
    return (t * q[3] + cross(u, t)) + v;
  }
  static V3 to_local(const Body& b, V3 p) { return qrot(b.rot, p - b.pos, true); }   // shape.rs:433-436
  static V3 to_world(const Body& b, V3 p) { return qrot(b.rot, p, false) + b.pos; }  // shape.rs:438-440

  static V3 support_local(const Body& b, V3 dir) {  // shape.rs:198-256
    switch (b.shape) {
      case 0:
        return normalize(dir) * b.size[0];
      case 1: {
        const V3 n = normalize(dir);
        const V3 end = dir.y > 0.0 ? V3{0.0, b.size[0], 0.0} : dir.y < 0.0 ? V3{0.0, -b.size[0], 0.0} : V3{0, 0, 0};
        return end + n * b.size[1];
      }
      case 2:
        return {dir.x >= 0.0 ? b.size[0] : -b.size[0], dir.y >= 0.0 ? b.size[1] : -b.size[1],
                dir.z >= 0.0 ? b.size[2] : -b.size[2]};
      case 3: {
        V3 best = b.verts[0];
        double best_dot = dot(b.verts[0], dir);
        for (size_t k = 1; k < b.verts.size(); ++k) {
          const double d = dot(b.verts[k], dir);
          if (d > best_dot) {
            best_dot = d;
            best = b.verts[k];
          }
        }
        return best;
      }
      case 5: {
        // The sub shape farthest along dir, in body coordinates; the search
        // starts from the first sub shape's offset at dot 0 (shape.rs:238-254).
        V3 best = b.subs[0].pos;
        double best_dot = 0.0;
        for (const Body& sub : b.subs) {
          const V3 d_local = qrot(sub.rot, dir, true);
          const V3 sp = support_local(sub, d_local);
          const V3 ws = sub.pos + qrot(sub.rot, sp, false);
          const double d = dot(ws, dir);
          if (d > best_dot) {
            best_dot = d;
            best = ws;
          }
        }
        return best;
      }
      default:
        return {0, 0, 0};
    }
  }

  static bool contains_local(const Body& b, V3 p) {  // shape.rs:287-325
    switch (b.shape) {
      case 0:
        return norm(p) <= b.size[0];
      case 1: {
        const double h = b.size[0], r = b.size[1];
        const double y = p.y < -h ? -h : (p.y > h ? h : p.y);
        const double cx = p.x * p.x + (p.y - y) * (p.y - y) + p.z * p.z;
        return cx <= r * r;
      }
      case 2:
        return std::fabs(p.x) <= b.size[0] && std::fabs(p.y) <= b.size[1] && std::fabs(p.z) <= b.size[2];
      case 3:
        for (size_t f = 0; f + 2 < b.faces.size(); f += 3) {
          const V3 a = b.verts[b.faces[f]], bb = b.verts[b.faces[f + 1]], c = b.verts[b.faces[f + 2]];
          const V3 n = cross(bb - a, c - a);
          if (dot(p - a, n) > 0.0) return false;
        }
        return true;
      case 5:  // any sub shape contains p in its own coordinates (shape.rs:319-322)
        for (const Body& sub : b.subs)
          if (contains_local(sub, qrot(sub.rot, p - sub.pos, true))) return true;
        return false;
      default:
        return false;
    }
  }

  static double body_volume(const Body& b) {  // world.rs:506-540
    switch (b.shape) {
      case 0:
        return 4.0 / 3.0 * kPi * b.size[0] * b.size[0] * b.size[0];
      case 1:
        return kPi * b.size[1] * b.size[1] * 2.0 * b.size[0] + 4.0 / 3.0 * kPi * b.size[1] * b.size[1] * b.size[1];
      case 2:
        return b.size[0] * b.size[1] * b.size[2] * 8.0;
      case 4: {
        const double hx = b.size[0] * b.size[2], hz = b.size[1] * b.size[2];
        double sum = 0.0;
        for (double h : b.heights) sum = sum + h;
        const double hy = b.heights.empty() ? 0.0 : sum / (double)b.heights.size();
        return hx * hz * std::fabs(hy);
      }
      case 5: {  // sum of the sub shapes' volumes, folded from 0 in order (world.rs:531-534)
        double v = 0.0;
        for (const Body& sub : b.subs) v = v + body_volume(sub);
        return v;
      }
      default:
        return 0.0;
    }
  }

  static void push_out(Particle& pt, const Body& b) {  // world.rs:755-773
    const V3 local = to_local(b, pt.pos);
    const V3 dir = norm(local) > 1e-9 ? normalize(local) : V3{0.0, 1.0, 0.0};
    const V3 support_dir = support_local(b, dir);
    pt.pos = to_world(b, support_dir);
    const V3 v_rel = pt.vel - b.vel;
    const V3 n = normalize(to_world(b, normalize(support_dir)) - b.pos);
    const double vn = dot(v_rel, n);
    if (vn < 0.0) pt.vel = pt.vel - n * vn;
  }

  // world.rs:414-503: symmetric soft contact and buoyancy with rigid bodies,
  // particle after particle (each body's velocity takes the impulses of the
  // particles before).  As in the reference, a dynamic contact's impulse on
  // the particle is overwritten by push_out's velocity, while the body keeps
  // its share.
  void couple_bodies(std::vector<Body>& bodies, double dt) {
    if (particles.empty() || bodies.empty()) return;
    const double rho_f = params.rest_density;
    const V3 g{params.gravity[0], params.gravity[1], params.gravity[2]};
    const double particle_vol = params.mass / rho_f;
    const double restitution = 0.0;
    std::vector<double> displaced(bodies.size(), 0.0);
    for (auto& pt : particles) {
      const V3 p_world = pt.pos;
      V3 v_p = pt.vel;
      const double m_p = pt.mass;
      for (size_t bi = 0; bi < bodies.size(); ++bi) {
        Body& body = bodies[bi];
        const V3 local = to_local(body, p_world);
        if (!contains_local(body, local)) continue;
        const V3 n = norm(local) > 1e-9 ? normalize(local) : V3{0.0, 1.0, 0.0};
        if (body.inv_mass <= 0.0) {
          push_out(pt, body);
          v_p = pt.vel;
          continue;
        }
        const double v_rel_n = dot(v_p - body.vel, n);
        if (v_rel_n < 0.0) {
          const double inv_sum = (1.0 / m_p) + body.inv_mass;
          const double j_mag = -(1.0 + restitution) * v_rel_n / inv_sum;
          const V3 j = n * j_mag;
          v_p = v_p + j / m_p;
          body.vel = body.vel + V3{-j.x, -j.y, -j.z} * body.inv_mass;  // apply_impulse (shape.rs:461-463)
        }
        displaced[bi] = displaced[bi] + particle_vol;
        push_out(pt, body);
        v_p = pt.vel;
      }
      pt.vel = v_p;
    }
    for (size_t bi = 0; bi < bodies.size(); ++bi) {
      Body& body = bodies[bi];
      if (body.inv_mass <= 0.0) continue;
      const double vol_b = body_volume(body);
      const double v_sub = displaced[bi] > 0.0 ? vol_b : 0.0;
      const V3 buoy = V3{-g.x, -g.y, -g.z} * (rho_f * v_sub);
      body.vel = body.vel + (buoy * dt) * body.inv_mass;
    }
  }

  // world.rs:691-752: point masses (pos, vel, mass in; force out) coupled to
  // the fluid one after another.  A point outside the bounds is skipped and
  // its force left as it was; each point's reaction -f*dt is shared among the
  // fluid particles of its 27 cells by mass, and the next point samples the
  // updated velocities.
  void couple_points(size_t np, const V3* ppos, const V3* pvel, const double* pmass, V3* pforce, double dt,
                     double drag, double soft_density) {
    if (np == 0 || particles.empty()) return;
    const double rho_f = params.rest_density;
    const V3 g{params.gravity[0], params.gravity[1], params.gravity[2]};
    const double* lo = params.bounds_min;
    const double* hi = params.bounds_max;
    grid.build(particles);
    std::vector<size_t> idxs;
    for (size_t k = 0; k < np; ++k) {
      const V3 p = ppos[k];
      if (p.x < lo[0] || p.x > hi[0] || p.y < lo[1] || p.y > hi[1] || p.z < lo[2] || p.z > hi[2]) continue;
      V3 v_sum{0, 0, 0};
      double w_sum = 0.0;
      grid.for_each_neighbor(p, [&](size_t j) {
        const double w = particles[j].mass;
        v_sum += particles[j].vel * w;
        w_sum = w_sum + w;
      });
      const V3 v_f = w_sum > 0.0 ? v_sum / w_sum : V3{0, 0, 0};
      const double vol = soft_density > 0.0 ? pmass[k] / soft_density : 0.0;
      const V3 f_b = V3{-g.x, -g.y, -g.z} * (rho_f * vol);
      const V3 f_d = (v_f - pvel[k]) * (drag * pmass[k]);
      const V3 f = f_b + f_d;
      pforce[k] = f;
      double m_sum = 0.0;
      idxs.clear();
      grid.for_each_neighbor(p, [&](size_t j) {
        m_sum = m_sum + particles[j].mass;
        idxs.push_back(j);
      });
      if (m_sum > 0.0) {
        const V3 reaction = V3{-f.x, -f.y, -f.z} * dt;
        for (size_t j : idxs) {
          const double frac = particles[j].mass / m_sum;
          particles[j].vel += reaction * frac;
        }
      }
    }
  }
};

// Forward-mode derivative (JVP) of one step, for checking the product's
// adjoint: the primal is advanced by the very same step() passes (so every
// branch is the reference's), and the tangents (tx, tv) of positions and
// velocities plus the tangents dk of stiffness and dc of visc_k[0] are
// pushed through the differentiated expressions of world.rs:204-397 with the
// neighbour sets and branches of that step.
struct Jvp {
  World& W;
  explicit Jvp(World& w) : W(w) {}

  static double dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

  void step(double dt, std::vector<V3>& tx, std::vector<V3>& tv, double dk, double dc) {
    auto& P = W.particles;
    const size_t n = P.size();
    if (n == 0) return;
    const Kernels& K = W.kernels;
    const double h = W.params.h, rest = W.params.rest_density, stiff = W.params.stiffness;
    const double r_eps = 1e-4, shear_min = W.params.shear_min;
    auto wp = [&](double r) {  // d poly6 / dr
      if (r >= K.h) return 0.0;
      double q = K.h2 - r * r;
      return -6.0 * K.poly6_coeff * r * q * q;
    };
    auto gp = [&](double r) {  // d spiky_grad_mag / dr
      if (r >= K.h || r <= 0.0) return 0.0;
      return -2.0 * K.spiky_grad_coeff * (K.h - r);
    };
    auto lp = [&](double r) { return r >= K.h ? 0.0 : -K.visc_lap_coeff; };
    W.grid.build(P);
    W.compute_density_pressure();
    // Density, pressure and p / rho^2 tangents.
    std::vector<double> trho(n), tpr2(n), pr2(n);
#pragma omp parallel for schedule(static) num_threads(W.nthreads)
    for (long long ii = 0; ii < (long long)n; ++ii) {
      size_t i = (size_t)ii;
      V3 p_i = P[i].pos;
      double t = 0.0;
      W.grid.for_each_neighbor(p_i, [&](size_t j) {
        V3 d = p_i - P[j].pos;
        double r = norm(d);
        if (!(r < h) || r <= 0.0) return;
        double dr = dot(d, tx[i] - tx[j]) / r;
        t += P[j].mass * wp(r) * dr;
      });
      trho[i] = t;
      double rho = P[i].rho, over = rho - rest;
      double tp = over > 0.0 ? dk * over + stiff * t : 0.0;
      pr2[i] = P[i].p / (rho * rho);
      tpr2[i] = tp / (rho * rho) - 2.0 * P[i].p * t / (rho * rho * rho);
    }
    // Force tangents (the primal sums are recomputed alongside).
    std::vector<V3> tacc(n), txs(n);
    const std::vector<Particle> snap = P;
#pragma omp parallel for schedule(static) num_threads(W.nthreads)
    for (long long ii = 0; ii < (long long)n; ++ii) {
      size_t i = (size_t)ii;
      const Particle& a = snap[i];
      V3 fp{0, 0, 0}, fv{0, 0, 0}, tfp{0, 0, 0}, tfv{0, 0, 0}, txsph{0, 0, 0};
      double shear = 0.0, tshear = 0.0;
      double m_i = a.mass, rho_i = a.rho;
      W.grid.for_each_neighbor(a.pos, [&](size_t j) {
        if (j == i) return;
        const Particle& b = snap[j];
        V3 d = b.pos - a.pos;
        double r = norm(d);
        if (r >= h || r <= 0.0) return;
        V3 u = d / r, dd = tx[j] - tx[i];
        double dr = dot(u, dd);
        V3 du = (dd - u * dr) / r;
        double mm = m_i * b.mass;
        double G = K.spiky_grad_mag(r), L = K.visc_lap(r), Wv = K.poly6(r);
        double A = mm * (pr2[i] + pr2[j]), tA = mm * (tpr2[i] + tpr2[j]);
        fp += u * (A * G);
        tfp += du * (A * G) + u * (tA * G + A * gp(r) * dr);
        V3 dv = b.vel - a.vel, tdv = tv[j] - tv[i];
        double B = mm / b.rho, tB = -mm * trho[j] / (b.rho * b.rho);
        fv += dv * (B * L);
        tfv += tdv * (B * L) + dv * (tB * L + B * lp(r) * dr);
        double mr = b.mass / b.rho, tmr = -b.mass * trho[j] / (b.rho * b.rho);
        txsph += tdv * (mr * Wv) + dv * (tmr * Wv + mr * wp(r) * dr);
        double dvn = norm(dv), tdvn = dvn > 0.0 ? dot(dv, tdv) / dvn : 0.0;
        double re = r + r_eps;
        shear += dvn / re * mr;
        tshear += tdvn / re * mr - dvn * dr / (re * re) * mr + dvn / re * tmr;
      });
      uint64_t m_idx = a.material < W.params.n_visc_k ? a.material : 0;
      double kc = W.params.visc_k[m_idx], nn = W.params.visc_n[m_idx];
      double ex = nn - 1.0;
      double sreg = shear > shear_min ? shear : shear_min;
      double fac = std::pow(sreg, ex);
      double tkc = m_idx == 0 ? dc : 0.0;
      double tmu = tkc * fac + ((ex != 0.0 && shear > shear_min) ? kc * ex * std::pow(sreg, ex - 1.0) * tshear : 0.0);
      double mu = kc * fac;
      V3 acc = (fp + fv * mu) / rho_i;
      tacc[i] = (tfp + tfv * mu + fv * tmu) / rho_i - acc * (trho[i] / rho_i);
      txs[i] = txsph;
    }
    W.compute_forces();
    // Integration and walls: the primal's decisions, recomputed in its order.
    V3 g{W.params.gravity[0], W.params.gravity[1], W.params.gravity[2]};
    const double eps = W.params.xsph_eps, damp = W.params.boundary_damp;
    for (size_t i = 0; i < n; ++i) {
      const Particle& pt = P[i];
      V3 a = pt.acc + g + pt.body_acc;
      V3 v = pt.vel + a * dt;
      v = v + pt.xsph * eps;
      V3 x = pt.pos + v * dt;
      V3 tv2 = tv[i] + tacc[i] * dt + txs[i] * eps;
      V3 tx1 = tx[i] + tv2 * dt;
      double xs[3] = {x.x, x.y, x.z};
      double t_x[3] = {tx1.x, tx1.y, tx1.z}, t_v[3] = {tv2.x, tv2.y, tv2.z};
      for (int k = 0; k < 3; ++k) {
        if (xs[k] < W.params.bounds_min[k] || xs[k] > W.params.bounds_max[k]) {
          t_x[k] = 0.0;
          t_v[k] = -damp * t_v[k];
        }
      }
      tx[i] = {t_x[0], t_x[1], t_x[2]};
      tv[i] = {t_v[0], t_v[1], t_v[2]};
    }
    W.integrate(dt);
    W.enforce_bounds();
  }
};

enum Field : int {
  F_POS = 0, F_VEL = 1, F_ACC = 2, F_BODY_ACC = 3, F_RHO = 4, F_P = 5,
  F_MASS = 6, F_MU_EFF = 7, F_XSPH = 8, F_MATERIAL = 9
};

V3* vec_field(Particle& p, int f) {
  switch (f) {
    case F_POS: return &p.pos;
    case F_VEL: return &p.vel;
    case F_ACC: return &p.acc;
    case F_BODY_ACC: return &p.body_acc;
    case F_XSPH: return &p.xsph;
    default: return nullptr;
  }
}
double* scalar_field(Particle& p, int f) {
  switch (f) {
    case F_RHO: return &p.rho;
    case F_P: return &p.p;
    case F_MASS: return &p.mass;
    case F_MU_EFF: return &p.mu_eff;
    default: return nullptr;
  }
}

}  // namespace

extern "C" {

void* orc_new(const OrcParams* p) { return new World(*p); }
void orc_free(void* w) { delete static_cast<World*>(w); }
uint64_t orc_len(void* w) { return static_cast<World*>(w)->particles.size(); }
void orc_set_threads(void* w, int n) { static_cast<World*>(w)->nthreads = n < 1 ? 1 : n; }
int orc_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// Live parameter update: kernels and grid keep the h captured at construction
// (world.rs:94-102), exactly like mutating `FluidWorld::params` in Rust.
void orc_set_params(void* w, const OrcParams* p) { static_cast<World*>(w)->params = *p; }
void orc_get_params(void* w, OrcParams* p) { *p = static_cast<World*>(w)->params; }

void orc_fill_box(void* w, const double* mn, const double* mx, double spacing, double margin) {
  static_cast<World*>(w)->fill_box({mn[0], mn[1], mn[2]}, {mx[0], mx[1], mx[2]}, spacing, margin);
}
double orc_lattice_mass(void* w, double s) { return static_cast<World*>(w)->lattice_mass(s); }

// Appends n particles built like Particle::with_material (particle.rs:50-71);
// vel may be null (zero velocity).
void orc_add(void* w, uint64_t n, const double* pos, const double* vel, const double* mass,
             const uint64_t* material) {
  World* W = static_cast<World*>(w);
  for (uint64_t i = 0; i < n; ++i) {
    Particle pt;
    pt.pos = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    if (vel) pt.vel = {vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
    pt.mass = mass[i];
    pt.material = material ? material[i] : 0;
    W->particles.push_back(pt);
  }
}

// Field access in insertion order: vector fields are xyz-interleaved.
int orc_get(void* w, int field, double* out) {
  World* W = static_cast<World*>(w);
  size_t n = W->particles.size();
  for (size_t i = 0; i < n; ++i) {
    Particle& p = W->particles[i];
    if (field == F_MATERIAL) {
      out[i] = (double)p.material;
    } else if (V3* v = vec_field(p, field)) {
      out[3 * i] = v->x;
      out[3 * i + 1] = v->y;
      out[3 * i + 2] = v->z;
    } else if (double* s = scalar_field(p, field)) {
      out[i] = *s;
    } else {
      return -1;
    }
  }
  return 0;
}
int orc_set(void* w, int field, const double* in) {
  World* W = static_cast<World*>(w);
  size_t n = W->particles.size();
  for (size_t i = 0; i < n; ++i) {
    Particle& p = W->particles[i];
    if (field == F_MATERIAL) {
      p.material = (uint64_t)in[i];
    } else if (V3* v = vec_field(p, field)) {
      *v = {in[3 * i], in[3 * i + 1], in[3 * i + 2]};
    } else if (double* s = scalar_field(p, field)) {
      *s = in[i];
    } else {
      return -1;
    }
  }
  return 0;
}

void orc_step(void* w, double dt) { static_cast<World*>(w)->step(dt); }
void orc_step_n(void* w, double dt, int n) {
  for (int i = 0; i < n; ++i) static_cast<World*>(w)->step(dt);
}

// n steps with forward-mode tangents: tx, tv (3n doubles, xyz interleaved,
// insertion order) hold the tangents of positions and velocities on entry
// and at the end; dk, dc are the tangents of stiffness and visc_k[0].
void orc_jvp(void* w, double dt, int n, double* tx, double* tv, double dk, double dc) {
  World* W = static_cast<World*>(w);
  const size_t m = W->particles.size();
  std::vector<V3> x(m), v(m);
  for (size_t i = 0; i < m; ++i) {
    x[i] = {tx[3 * i], tx[3 * i + 1], tx[3 * i + 2]};
    v[i] = {tv[3 * i], tv[3 * i + 1], tv[3 * i + 2]};
  }
  Jvp J(*W);
  for (int k = 0; k < n; ++k) J.step(dt, x, v, dk, dc);
  for (size_t i = 0; i < m; ++i) {
    tx[3 * i] = x[i].x;
    tx[3 * i + 1] = x[i].y;
    tx[3 * i + 2] = x[i].z;
    tv[3 * i] = v[i].x;
    tv[3 * i + 1] = v[i].y;
    tv[3 * i + 2] = v[i].z;
  }
}

// Grid::key_of for every particle (int64 xyz-interleaved), used to pin the
// device cell keys bit-exactly.
void orc_cell_keys(void* w, int64_t* out) {
  World* W = static_cast<World*>(w);
  for (size_t i = 0; i < W->particles.size(); ++i) {
    Key k = W->grid.key_of(W->particles[i].pos);
    out[3 * i] = k.i;
    out[3 * i + 1] = k.j;
    out[3 * i + 2] = k.k;
  }
}

// Neighbour list of particle i in the reference's visit order
// (for_each_neighbor over a grid built from the current positions).
// Returns the number of candidates; writes up to cap indices.
uint64_t orc_neighbors(void* w, uint64_t i, uint64_t* out, uint64_t cap) {
  World* W = static_cast<World*>(w);
  W->grid.build(W->particles);
  uint64_t cnt = 0;
  W->grid.for_each_neighbor(W->particles[i].pos, [&](size_t j) {
    if (cnt < cap) out[cnt] = j;
    ++cnt;
  });
  return cnt;
}

// FluidWorld::couple_points (world.rs:691-752) on np points: pos, vel,
// force are 3*np doubles (xyz interleaved), mass np doubles; force is written
// for the points inside the bounds only.
void orc_couple_points(void* w, uint64_t np, const double* pos, const double* vel, const double* mass,
                       double* force, double dt, double drag, double soft_density) {
  World* W = static_cast<World*>(w);
  std::vector<V3> p(np), v(np), f(np);
  for (uint64_t k = 0; k < np; ++k) {
    p[k] = {pos[3 * k], pos[3 * k + 1], pos[3 * k + 2]};
    v[k] = {vel[3 * k], vel[3 * k + 1], vel[3 * k + 2]};
    f[k] = {force[3 * k], force[3 * k + 1], force[3 * k + 2]};
  }
  W->couple_points((size_t)np, p.data(), v.data(), mass, f.data(), dt, drag, soft_density);
  for (uint64_t k = 0; k < np; ++k) {
    force[3 * k] = f[k].x;
    force[3 * k + 1] = f[k].y;
    force[3 * k + 2] = f[k].z;
  }
}

// Same layout as PhyCoupleBody in include/phy_fluid.h.
struct OrcBody {
  int32_t shape;
  uint32_t data_first, data_count, face_first, face_count, reserved;
  double size[3], pos[3], rot[4], vel[3], inv_mass;
};

// Convex vertices / heightfield heights of a shape from the shared arrays.
static void shape_data(World::Body& b, uint32_t data_first, uint32_t data_count, uint32_t face_first,
                       uint32_t face_count, const double* data, const uint32_t* faces) {
  if (b.shape == 3) {
    for (uint32_t v = 0; v < data_count; ++v) {
      const double* d = data + data_first + 3 * v;
      b.verts.push_back({d[0], d[1], d[2]});
    }
    b.faces.assign(faces + 3 * (size_t)face_first, faces + 3 * ((size_t)face_first + face_count));
  } else if (b.shape == 4) {
    b.heights.assign(data + data_first, data + data_first + data_count);
  }
}

// FluidWorld::couple_bodies (world.rs:414-503); the bodies' velocities are
// updated in place.  Convex vertices are data_count xyz triples from
// data[data_first]; faces are face_count index triples from
// faces[3 * face_first]; heightfield heights are data_count values; a
// compound body's data_count sub shapes are 16-double records from
// data[data_first]: shape, size[3], offset[3], quaternion (i, j, k, w),
// data_first, data_count, face_first, face_count, unused.
void orc_couple_bodies(void* w, OrcBody* bodies, uint32_t nb, const double* data, const uint32_t* faces, double dt) {
  std::vector<World::Body> bs(nb);
  for (uint32_t k = 0; k < nb; ++k) {
    const OrcBody& o = bodies[k];
    World::Body& b = bs[k];
    b.shape = o.shape;
    for (int a = 0; a < 3; ++a) b.size[a] = o.size[a];
    b.pos = {o.pos[0], o.pos[1], o.pos[2]};
    for (int a = 0; a < 4; ++a) b.rot[a] = o.rot[a];
    b.vel = {o.vel[0], o.vel[1], o.vel[2]};
    b.inv_mass = o.inv_mass;
    shape_data(b, o.data_first, o.data_count, o.face_first, o.face_count, data, faces);
    if (o.shape == 5) {
      for (uint32_t q = 0; q < o.data_count; ++q) {
        const double* r = data + o.data_first + 16 * (size_t)q;
        World::Body sub;
        sub.shape = (int)r[0];
        for (int a = 0; a < 3; ++a) sub.size[a] = r[1 + a];
        sub.pos = {r[4], r[5], r[6]};
        for (int a = 0; a < 4; ++a) sub.rot[a] = r[7 + a];
        shape_data(sub, (uint32_t)r[11], (uint32_t)r[12], (uint32_t)r[13], (uint32_t)r[14], data, faces);
        b.subs.push_back(sub);
      }
    }
  }
  static_cast<World*>(w)->couple_bodies(bs, dt);
  for (uint32_t k = 0; k < nb; ++k) {
    bodies[k].vel[0] = bs[k].vel.x;
    bodies[k].vel[1] = bs[k].vel.y;
    bodies[k].vel[2] = bs[k].vel.z;
  }
}

// FluidWorld::couple_heat (world.rs:555-678) against a heat grid of
// dims3[0..2] cells (x fastest), origin3 and cell size `cell`: u holds the
// temperatures, src the sources (updated in place).
void orc_couple_heat(void* w, const uint64_t* dims3, const double* origin3, double cell, const double* u, double* src,
                     double dt, double t_ref, double beta, double heat_gain) {
  World::HeatGrid g{dims3[0], dims3[1], dims3[2], V3{origin3[0], origin3[1], origin3[2]}, cell, u, src};
  static_cast<World*>(w)->couple_heat(g, dt, t_ref, beta, heat_gain);
}

// for_each_neighbor of an arbitrary point (xyz) over a grid of the current
// positions: the particles couple_points visits for it, in visit order.
uint64_t orc_point_neighbors(void* w, const double* p3, uint64_t* out, uint64_t cap) {
  World* W = static_cast<World*>(w);
  W->grid.build(W->particles);
  uint64_t cnt = 0;
  W->grid.for_each_neighbor(V3{p3[0], p3[1], p3[2]}, [&](size_t j) {
    if (cnt < cap) out[cnt] = j;
    ++cnt;
  });
  return cnt;
}

// Diagnostics of FluidSubsystem (subsystem.rs:149-163): momentum xyz, KE.
void orc_diagnostics(void* w, double* out4) {
  World* W = static_cast<World*>(w);
  V3 p{0, 0, 0};
  for (auto& pt : W->particles) p += pt.vel * pt.mass;
  double e = 0.0;
  for (auto& pt : W->particles) e = e + (norm_squared(pt.vel) * pt.mass) / (1.0 + 1.0);
  out4[0] = p.x;
  out4[1] = p.y;
  out4[2] = p.z;
  out4[3] = e;
}

// Candidates visited and in-range pairs counted by the density passes since
// the last reset (roofline accounting).
void orc_counters(void* w, uint64_t* out2, int reset) {
  World* W = static_cast<World*>(w);
  out2[0] = W->counters.candidates;
  out2[1] = W->counters.pairs;
  if (reset) W->counters = Counters{};
}

}  // extern "C"
