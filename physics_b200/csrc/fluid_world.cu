// Host-side FluidWorld / FluidSubsystem / World of the B200 build.
#include "fluid_world.h"

#include "adjoint.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <climits>
#include <limits>

namespace phy {

namespace {

constexpr double kPi = 3.14159265358979323846;  // std::f64::consts::PI
constexpr long long kMaxCells = 1ll << 27;       // grid box cap (512 MiB of cell starts)
constexpr int kThreads = 256;

int grid_for(size_t n) { return (int)std::max<size_t>(1, (n + kThreads - 1) / kThreads); }

__global__ void k_set_scalar_by_id(int n, const uint32_t* __restrict__ id, const double* __restrict__ src,
                                   double* __restrict__ dst) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) dst[s] = src[id[s]];
}
__global__ void k_set_u32_by_id(int n, const uint32_t* __restrict__ id, const double* __restrict__ src,
                                uint32_t* __restrict__ dst) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) {
    double v = src[id[s]];
    dst[s] = v >= 4294967295.0 ? 0xffffffffu : (v > 0.0 ? (uint32_t)v : 0u);
  }
}
__global__ void k_set_vec_by_id(int n, const uint32_t* __restrict__ id, const double* __restrict__ src,
                                double* __restrict__ x, double* __restrict__ y, double* __restrict__ z) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) {
    size_t o = 3 * (size_t)id[s];
    x[s] = src[o];
    y[s] = src[o + 1];
    z[s] = src[o + 2];
  }
}
__global__ void k_get_scalar_by_id(int n, const uint32_t* __restrict__ id, const double* __restrict__ src,
                                   double* __restrict__ dst) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) dst[id[s]] = src[s];
}
__global__ void k_get_vec_by_id(int n, const uint32_t* __restrict__ id, const double* __restrict__ x,
                                const double* __restrict__ y, const double* __restrict__ z,
                                double* __restrict__ dst) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) {
    size_t o = 3 * (size_t)id[s];
    dst[o] = x[s];
    dst[o + 1] = y[s];
    dst[o + 2] = z[s];
  }
}
__global__ void k_get_vec_f32_by_id(int n, const uint32_t* __restrict__ id, const double* __restrict__ x,
                                    const double* __restrict__ y, const double* __restrict__ z,
                                    float* __restrict__ dst) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) {
    size_t o = 3 * (size_t)id[s];
    dst[o] = (float)x[s];
    dst[o + 1] = (float)y[s];
    dst[o + 2] = (float)z[s];
  }
}
// Appends m particles (insertion-order staging: pos 3m, vel 3m, mass m,
// material m) at slots [n0, n0+m).
__global__ void k_append(int n0, int m, const double* __restrict__ st, double* px, double* py, double* pz,
                         double* vx, double* vy, double* vz, double* mass, uint32_t* mat, uint32_t* id) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const double* pos = st;
  const double* vel = st + 3 * (size_t)m;
  const double* ms = st + 6 * (size_t)m;
  const double* mt = st + 7 * (size_t)m;
  int s = n0 + k;
  px[s] = pos[3 * (size_t)k];
  py[s] = pos[3 * (size_t)k + 1];
  pz[s] = pos[3 * (size_t)k + 2];
  vx[s] = vel[3 * (size_t)k];
  vy[s] = vel[3 * (size_t)k + 1];
  vz[s] = vel[3 * (size_t)k + 2];
  mass[s] = ms[k];
  double v = mt[k];
  mat[s] = v >= 4294967295.0 ? 0xffffffffu : (v > 0.0 ? (uint32_t)v : 0u);
  id[s] = (uint32_t)s;
}

// Cell-key bounding box of n interleaved positions: out[0..2] min, out[3..5]
// max over finite coordinates, out[6] = 1 when a coordinate is not finite.
// out must be preset to (LLONG_MAX x3, LLONG_MIN x3, 0).
__global__ void k_key_bbox(int n, const double* __restrict__ pos3, double inv, long long* out) {
  long long mn[3] = {LLONG_MAX, LLONG_MAX, LLONG_MAX}, mx[3] = {LLONG_MIN, LLONG_MIN, LLONG_MIN};
  int bad = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double x = pos3[3 * (size_t)i + a];
      if (!isfinite(x)) {
        bad = 1;
        continue;
      }
      long long k = key_axis(x, inv);
      mn[a] = k < mn[a] ? k : mn[a];
      mx[a] = k > mx[a] ? k : mx[a];
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    for (int o = 16; o > 0; o >>= 1) {
      long long y = __shfl_xor_sync(0xffffffffu, mn[a], o);
      long long z = __shfl_xor_sync(0xffffffffu, mx[a], o);
      mn[a] = y < mn[a] ? y : mn[a];
      mx[a] = z > mx[a] ? z : mx[a];
    }
  }
  bad = __any_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0) {
    for (int a = 0; a < 3; ++a) {
      if (mn[a] != LLONG_MAX) atomicMin(&out[a], mn[a]);
      if (mx[a] != LLONG_MIN) atomicMax(&out[3 + a], mx[a]);
    }
    if (bad) atomicMax(&out[6], 1ll);
  }
}

// Scene of every slot from its insertion index: the scene whose insertion
// range [pbase[s], pbase[s+1]) holds it.
__global__ void k_scene_of_id(int n, const uint32_t* __restrict__ id, const uint32_t* __restrict__ pbase,
                              int n_scenes, uint16_t* __restrict__ scene) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t i = id[s];
  int lo = 0, hi = n_scenes - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pbase[mid] <= i) lo = mid; else hi = mid - 1;
  }
  scene[s] = (uint16_t)lo;
}

// Cell-key bounding box of each scene's finite positions (interleaved xyz,
// insertion order): one block per scene, out[7 s ..] = min xyz, max xyz,
// non-finite flag.
__global__ void __launch_bounds__(kThreads) k_scene_bbox(const double* __restrict__ pos3,
                                                         const uint32_t* __restrict__ pbase, double inv,
                                                         long long* __restrict__ out) {
  const int sc = blockIdx.x;
  long long mn[3] = {LLONG_MAX, LLONG_MAX, LLONG_MAX}, mx[3] = {LLONG_MIN, LLONG_MIN, LLONG_MIN};
  int bad = 0;
  for (uint32_t i = pbase[sc] + threadIdx.x; i < pbase[sc + 1]; i += kThreads) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double x = pos3[3 * (size_t)i + a];
      if (!isfinite(x)) {
        bad = 1;
        continue;
      }
      const long long k = key_axis(x, inv);
      mn[a] = k < mn[a] ? k : mn[a];
      mx[a] = k > mx[a] ? k : mx[a];
    }
  }
  __shared__ long long s_mn[3][kThreads / 32], s_mx[3][kThreads / 32];
  __shared__ int s_bad[kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    for (int o = 16; o > 0; o >>= 1) {
      const long long y = __shfl_xor_sync(0xffffffffu, mn[a], o);
      const long long z = __shfl_xor_sync(0xffffffffu, mx[a], o);
      mn[a] = y < mn[a] ? y : mn[a];
      mx[a] = z > mx[a] ? z : mx[a];
    }
    if (lane == 0) {
      s_mn[a][warp] = mn[a];
      s_mx[a][warp] = mx[a];
    }
  }
  bad = __any_sync(0xffffffffu, bad);
  if (lane == 0) s_bad[warp] = bad;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long r[7] = {LLONG_MAX, LLONG_MAX, LLONG_MAX, LLONG_MIN, LLONG_MIN, LLONG_MIN, 0};
    for (int w = 0; w < kThreads / 32; ++w) {
      for (int a = 0; a < 3; ++a) {
        r[a] = s_mn[a][w] < r[a] ? s_mn[a][w] : r[a];
        r[3 + a] = s_mx[a][w] > r[3 + a] ? s_mx[a][w] : r[3 + a];
      }
      r[6] |= s_bad[w];
    }
    for (int k = 0; k < 7; ++k) out[7 * sc + k] = r[k];
  }
}

// One recorded step of the adjoint tape: every per-particle array of the
// step copied in one launch (22 f64 arrays, 2 u32 arrays).
struct TapeCopy {
  const double* src[22];
  double* dst[22];
  const uint32_t* usrc[3];  // mat, id, neighbour count
  uint32_t* udst[3];
  const uint32_t* nbr;      // column-major, stride nbr_stride
  uint32_t* nbr_dst;        // column-major, stride n
  int nbr_stride;
  uint32_t* slot_of;        // nullable: insertion index -> recorded slot
};

__global__ void k_tape_copy(int n, TapeCopy t) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
#pragma unroll
  for (int k = 0; k < 22; ++k) t.dst[k][s] = t.src[k][s];
  t.udst[0][s] = t.usrc[0][s];
  const uint32_t id = t.usrc[1][s];
  t.udst[1][s] = id;
  if (t.slot_of) t.slot_of[id] = (uint32_t)s;
  const uint32_t cnt = t.usrc[2][s];
  t.udst[2][s] = cnt;
  const uint32_t m = cnt < (uint32_t)kMaxNeighbors ? cnt : (uint32_t)kMaxNeighbors;
  for (uint32_t k = 0; k < m; ++k) t.nbr_dst[(size_t)k * n + s] = t.nbr[(size_t)k * t.nbr_stride + s];
}

// Several device arrays copied in one launch (blockIdx.y = array): 16-byte
// words where both ends are 16-byte aligned, 8-byte words where they are
// 8-byte aligned, bytes for the rest.
struct ArrayCopy {
  static constexpr int kMax = 24;
  const unsigned char* src[kMax];
  unsigned char* dst[kMax];
  size_t bytes[kMax];
};

__global__ void k_copy_arrays(ArrayCopy a) {
  const int q = blockIdx.y;
  const unsigned char* s = a.src[q];
  unsigned char* d = a.dst[q];
  const size_t bytes = a.bytes[q];
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uintptr_t align = reinterpret_cast<uintptr_t>(s) | reinterpret_cast<uintptr_t>(d);
  size_t done = 0;
  if ((align & 15) == 0) {
    const size_t words = bytes / 16;
    for (size_t k = i; k < words; k += stride)
      reinterpret_cast<uint4*>(d)[k] = reinterpret_cast<const uint4*>(s)[k];
    done = words * 16;
  } else if ((align & 7) == 0) {
    const size_t words = bytes / 8;
    for (size_t k = i; k < words; k += stride)
      reinterpret_cast<unsigned long long*>(d)[k] = reinterpret_cast<const unsigned long long*>(s)[k];
    done = words * 8;
  }
  for (size_t k = done + i; k < bytes; k += stride) d[k] = s[k];
}

// The compensated step's outputs (its sorted order, slot q) written over the
// recorded f64 ones (the recorded slot of the same particle, from slot_of):
// density, pressure, p/rho^2 and m/rho from them, mu, acceleration, XSPH.
struct CompOverride {
  const uint32_t* id;  // compensated order: insertion index
  const double* mass;
  const double* rho;
  const double* p;
  const double* mu;
  const double* acc[3];
  const double* xsph[3];
  const uint32_t* slot_of;
  double* t_rho;
  double* t_p;
  double* t_pr2;
  double* t_mr;
  double* t_mu;
  double* t_acc[3];
  double* t_xsph[3];
};

__global__ void k_comp_override(int n, CompOverride o) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const uint32_t s = o.slot_of[o.id[q]];
  const double r = o.rho[q], pr = o.p[q];
  o.t_rho[s] = r;
  o.t_p[s] = pr;
  o.t_pr2[s] = __ddiv_rn(pr, __dmul_rn(r, r));
  o.t_mr[s] = __ddiv_rn(o.mass[q], r);
  o.t_mu[s] = o.mu[q];
  for (int k = 0; k < 3; ++k) {
    o.t_acc[k][s] = o.acc[k][q];
    o.t_xsph[k][s] = o.xsph[k][q];
  }
}

// num-traits ToPrimitive::to_i64 on f64 with None -> 0 (grid.rs:25-33).
long long key_axis_host(double x, double inv) {
  double f = std::floor(x * inv);
  if (f > -9223372036854775808.0 && f < 9223372036854775808.0) return (long long)f;
  return 0;
}

template <class T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

template <class T>
void dalloc(T*& p, size_t count) {
  dfree(p);
  if (count == 0) count = 1;
  cuda_check(cudaMalloc((void**)&p, count * sizeof(T)), "cudaMalloc");
}

// Grows a device array to `cap` elements, keeping the first `keep`.
template <class T>
void dgrow(T*& p, size_t keep, size_t cap, cudaStream_t s) {
  T* q = nullptr;
  cuda_check(cudaMalloc((void**)&q, std::max<size_t>(cap, 1) * sizeof(T)), "cudaMalloc");
  if (p && keep) cuda_check(cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, s), "grow copy");
  if (p) {
    cuda_check(cudaStreamSynchronize(s), "grow sync");
    cudaFree(p);
  }
  p = q;
}

}  // namespace

void cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  // The error goes to the caller; a non-sticky API error must not stay in the
  // runtime's last-error slot and fail the next, unrelated call's check.
  (void)cudaGetLastError();
  throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

// ---- SphParams -------------------------------------------------------------

SphParams SphParams::defaults() {
  SphParams p;
  p.rest_density = 1000.0;
  p.stiffness = 250.0;
  p.viscosity = 3.5;
  p.visc_k = {3.5};
  p.visc_n = {1.0};
  p.shear_min = 0.01;
  p.mass = 0.02;
  p.h = 0.2;
  p.gravity = {0.0, -9.81, 0.0};
  p.bounds_min = {-5.0, -5.0, -5.0};
  p.bounds_max = {5.0, 5.0, 5.0};
  p.boundary_damp = 0.4;
  p.xsph_eps = 0.5;
  return p;
}

PhySphParams SphParams::to_c() const {
  PhySphParams c;
  std::memset(&c, 0, sizeof(c));
  c.rest_density = rest_density;
  c.stiffness = stiffness;
  c.viscosity = viscosity;
  c.shear_min = shear_min;
  c.mass = mass;
  c.h = h;
  const Vec3* v[3] = {&gravity, &bounds_min, &bounds_max};
  double* d[3] = {c.gravity, c.bounds_min, c.bounds_max};
  for (int k = 0; k < 3; ++k) {
    d[k][0] = v[k]->x;
    d[k][1] = v[k]->y;
    d[k][2] = v[k]->z;
  }
  c.boundary_damp = boundary_damp;
  c.xsph_eps = xsph_eps;
  c.n_visc_k = (uint32_t)std::min<size_t>(visc_k.size(), PHY_MAX_MATERIALS);
  c.n_visc_n = (uint32_t)std::min<size_t>(visc_n.size(), PHY_MAX_MATERIALS);
  for (uint32_t k = 0; k < c.n_visc_k; ++k) c.visc_k[k] = visc_k[k];
  for (uint32_t k = 0; k < c.n_visc_n; ++k) c.visc_n[k] = visc_n[k];
  return c;
}

SphParams SphParams::from_c(const PhySphParams& c) {
  if (c.n_visc_k < 1 || c.n_visc_k > PHY_MAX_MATERIALS || c.n_visc_n > PHY_MAX_MATERIALS)
    throw std::invalid_argument("SphParams: n_visc_k must be 1..16 and n_visc_n at most 16");
  SphParams p;
  p.rest_density = c.rest_density;
  p.stiffness = c.stiffness;
  p.viscosity = c.viscosity;
  p.shear_min = c.shear_min;
  p.mass = c.mass;
  p.h = c.h;
  p.gravity = {c.gravity[0], c.gravity[1], c.gravity[2]};
  p.bounds_min = {c.bounds_min[0], c.bounds_min[1], c.bounds_min[2]};
  p.bounds_max = {c.bounds_max[0], c.bounds_max[1], c.bounds_max[2]};
  p.boundary_damp = c.boundary_damp;
  p.xsph_eps = c.xsph_eps;
  p.visc_k.assign(c.visc_k, c.visc_k + c.n_visc_k);
  p.visc_n.assign(c.visc_n, c.visc_n + c.n_visc_n);
  return p;
}

// ---- FluidWorld --------------------------------------------------------------

FluidWorld::FluidWorld(const SphParams& p, Precision prec) : params(p), prec_(prec), h0_(p.h) {
  cuda_check(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  stream_ = own_stream_;
  dalloc(b_.flags, 1);
  dalloc(b_.counters, 2);
  dalloc(b_.order_count, 1);
  cuda_check(cudaMemsetAsync(b_.flags, 0, sizeof(uint32_t), stream_), "memset");
  cuda_check(cudaMemsetAsync(b_.counters, 0, 2 * sizeof(unsigned long long), stream_), "memset");
}

FluidWorld::~FluidWorld() {
  if (stream_) cudaStreamSynchronize(stream_);
  drop_graphs();
  free_all();
  dfree(d_bbox_);
  dfree(d_couple_);
  couple_scratch_.release();
  dfree(d_heat_);
  dfree(d_bodies_);
  dfree(d_pbase_);
  dfree(d_scene_bbox_);
  release_snapshot();
  tape_clear();
  for (auto& set : ev_pool_)
    for (auto& e : set) cudaEventDestroy(e);
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

void FluidWorld::free_all() {
  for (int k = 0; k < 6; ++k) {
    dfree(b_.pv0[k]);
    dfree(b_.pv1[k]);
  }
  for (int q = 0; q < 2; ++q) {
    dfree(b_.pc[q].mass);
    dfree(b_.pc[q].mat);
    dfree(b_.pc[q].id);
    dfree(b_.pc[q].scene);
    for (int k = 0; k < 3; ++k) dfree(b_.pc[q].ba[k]);
  }
  dfree(b_.rho);
  dfree(b_.p);
  dfree(b_.pr2);
  dfree(b_.mr);
  for (int k = 0; k < 3; ++k) {
    dfree(b_.acc[k]);
    dfree(b_.xsph[k]);
  }
  dfree(b_.mu);
  dfree(b_.cpos);
  dfree(b_.cvel);
  dfree(b_.cmr);
  dfree(b_.nbr);
  dfree(b_.nbr_count);
  dfree(b_.nbr16);
  dfree(b_.sorted_cell);
  dfree(b_.tile_head);
  b_.tile_scan_entries = 0;
  dfree(b_.tile_of);
  dfree(b_.large_cells);
  dfree(b_.tile_slot);
  dfree(b_.num_tiles);
  dfree(b_.boxes);
  dfree(b_.queue);
  dfree(b_.tile_crowd);
  dfree(b_.dense_q0);
  dfree(b_.task_mbase);
  dfree(b_.task_mcount);
  dfree(b_.mask_hdr);
  dfree(b_.mask_bits);
  dfree(b_.mask_ctl);
  b_.mask_cap = 0;
  mask_tried_ = 0;
  if (b_.mask_demand) cudaFreeHost(b_.mask_demand);
  b_.mask_demand = nullptr;
  dfree(b_.okey);
  dfree(b_.cell_of);
  dfree(b_.rank);
  dfree(b_.tmp);
  dfree(b_.perm);
  dfree(b_.cell_start);
  dfree(b_.block_sums);
  dfree(b_.stage);
  dfree(b_.flags);
  dfree(b_.counters);
  dfree(b_.order_count);
}

void FluidWorld::set_stream(cudaStream_t s) {
  cuda_check(cudaStreamSynchronize(stream_), "stream switch");
  stream_ = s ? s : own_stream_;
}

void FluidWorld::synchronize() { cuda_check(cudaStreamSynchronize(stream_), "synchronize"); }

// Grows every per-particle array to hold n particles (geometric growth),
// keeping the current n_ particles.
void FluidWorld::ensure_capacity(size_t n) {
  if (n >= (1ull << (32 - kCodeBits)))
    throw std::invalid_argument("FluidWorld: more than 2^27 particles in one subsystem");
  if ((int)n <= b_.capacity) return;
  size_t cap = std::max<size_t>(n, (size_t)b_.capacity + b_.capacity / 2);
  cudaStream_t s = stream_;
  for (int k = 0; k < 6; ++k) {
    dgrow(b_.pv0[k], 0, cap, s);
    dgrow(b_.pv1[k], n_, cap, s);
  }
  // The current per-particle constants live in pc[cur]; the other set is
  // scratch for the next sort.
  for (int q = 0; q < 2; ++q) {
    size_t keep = q == b_.cur ? n_ : 0;
    dgrow(b_.pc[q].mass, keep, cap, s);
    dgrow(b_.pc[q].mat, keep, cap, s);
    dgrow(b_.pc[q].id, keep, cap, s);
    if (b_.has_ba)
      for (int k = 0; k < 3; ++k) dgrow(b_.pc[q].ba[k], keep, cap, s);
    if (b_.pc[q].scene) dgrow(b_.pc[q].scene, keep, cap, s);
  }
  dgrow(b_.rho, n_, cap, s);
  dgrow(b_.p, n_, cap, s);
  dgrow(b_.pr2, 0, cap, s);
  dgrow(b_.mr, 0, cap, s);
  for (int k = 0; k < 3; ++k) {
    dgrow(b_.acc[k], n_, cap, s);
    dgrow(b_.xsph[k], n_, cap, s);
  }
  dgrow(b_.mu, n_, cap, s);
  if (prec_ == Precision::F32Comp) {
    dgrow(b_.cpos, 0, cap, s);
    dgrow(b_.cvel, 0, cap, s);
    dgrow(b_.cmr, 0, cap, s);
  }
  dgrow(b_.nbr_count, 0, cap, s);
  dfree(b_.nbr);
  dfree(b_.nbr16);
  dfree(b_.sorted_cell);
  dfree(b_.tile_of);
  dfree(b_.large_cells);
  dfree(b_.tile_slot);
  dfree(b_.tile_crowd);
  dfree(b_.dense_q0);
  dfree(b_.task_mbase);
  dfree(b_.task_mcount);
  dfree(b_.okey);
  dgrow(b_.cell_of, 0, cap, s);
  dgrow(b_.rank, 0, cap, s);
  dgrow(b_.tmp, 0, cap, s);
  dgrow(b_.perm, 0, cap, s);
  dgrow(b_.stage, 0, 8 * cap, s);
  b_.capacity = (int)cap;
  ++alloc_gen_;
  ensure_mode_buffers();
}

// Buffers that depend on the kernel form: 32-bit neighbour lists for the
// x-major passes, 16-bit staged-slot lists and the tile list for tiles.
void FluidWorld::ensure_mode_buffers() {
  const size_t cap = (size_t)b_.capacity;
  if (cap == 0) return;
  const bool tiled = prec_ == Precision::F32Comp && comp_tile_ > 0;
  if (!tiled && !b_.nbr) dalloc(b_.nbr, (size_t)kMaxNeighbors * cap);
  if (tiled) {
    if (!b_.nbr16) dalloc(b_.nbr16, (size_t)kMaxNeighbors * cap);
    if (!b_.sorted_cell) dalloc(b_.sorted_cell, cap);
    if (!b_.tile_of) dalloc(b_.tile_of, cap + 1);
    if (!b_.large_cells) dalloc(b_.large_cells, cap / 64 + 64);  // cells of more than 64 particles
    if (!b_.tile_slot) dalloc(b_.tile_slot, cap + 1);
    if (!b_.tile_crowd) dalloc(b_.tile_crowd, cap + 1);
    if (!b_.num_tiles) dalloc(b_.num_tiles, 1);
    if (!b_.queue) dalloc(b_.queue, 5);
    // Dense-cell tasks: at most one per 32 particles plus one per occupied cell.
    if (!b_.dense_q0) dalloc(b_.dense_q0, cap + cap / 32 + 64);
    if (!b_.task_mbase) dalloc(b_.task_mbase, cap + cap / 32 + 64);
    if (!b_.task_mcount) dalloc(b_.task_mcount, cap + cap / 32 + 64);
    if (!b_.mask_ctl) dalloc(b_.mask_ctl, 1);
    if (!b_.mask_demand) {
      cuda_check(cudaMallocHost((void**)&b_.mask_demand, sizeof(unsigned long long)), "cudaMallocHost");
      *b_.mask_demand = 0;
    }
    if (!b_.okey) dalloc(b_.okey, cap);
  }
  ++alloc_gen_;
}

void FluidWorld::set_comp_tile(int t) {
  if (t != 0 && t != 2 && t != 4)
    throw std::invalid_argument("comp tile must be 0 (x-major runs), 2 or 4 (cells per tile edge)");
  if (t == 0 && !scenes_.empty()) throw std::invalid_argument("batched scenes need the tiled form (comp tile 4)");
  comp_tile_ = t;
  ensure_mode_buffers();
}

void FluidWorld::grow_box_with_bounds() {
  const double inv = 1.0 / h0_;  // grid.rs:27, cell = h captured at construction
  const double lo[3] = {params.bounds_min.x, params.bounds_min.y, params.bounds_min.z};
  const double hi[3] = {params.bounds_max.x, params.bounds_max.y, params.bounds_max.z};
  for (int a = 0; a < 3; ++a) {
    long long k0 = key_axis_host(lo[a], inv), k1 = key_axis_host(hi[a], inv);
    long long mn = std::min(k0, k1), mx = std::max(k0, k1);
    if (!box_valid_) {
      kmin_[a] = mn;
      kmax_[a] = mx;
    } else {
      kmin_[a] = std::min(kmin_[a], mn);
      kmax_[a] = std::max(kmax_[a], mx);
    }
  }
  box_valid_ = true;
}

// Widens the box with the keys of host positions.  Keys of non-finite
// coordinates (0 on that axis, as in the reference) are included only when
// the box stays within the cell cap; otherwise such particles are reported
// through the out-of-box flag at run time.
void FluidWorld::grow_box_with_positions(size_t n, const double* pos3) {
  const double inv = 1.0 / h0_;
  long long mn[3] = {LLONG_MAX, LLONG_MAX, LLONG_MAX}, mx[3] = {LLONG_MIN, LLONG_MIN, LLONG_MIN};
  bool any_nonfinite = false;
  for (size_t i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) {
      double x = pos3[3 * i + a];
      if (!std::isfinite(x)) {
        any_nonfinite = true;
        continue;
      }
      long long k = key_axis_host(x, inv);
      mn[a] = std::min(mn[a], k);
      mx[a] = std::max(mx[a], k);
    }
  }
  merge_box(mn, mx, any_nonfinite);
}

// Same as grow_box_with_positions for positions already on the device
// (interleaved xyz), through a reduction kernel and one small readback.
void FluidWorld::grow_box_with_device_positions(size_t n, const double* d_pos3) {
  if (n == 0) return;
  if (!d_bbox_) dalloc(d_bbox_, 7);
  long long init[7] = {LLONG_MAX, LLONG_MAX, LLONG_MAX, LLONG_MIN, LLONG_MIN, LLONG_MIN, 0};
  long long res[7];
  cuda_check(cudaMemcpyAsync(d_bbox_, init, sizeof(init), cudaMemcpyHostToDevice, stream_), "bbox init");
  int blocks = (int)std::min<size_t>(148 * 8, (n + kThreads - 1) / kThreads);
  k_key_bbox<<<std::max(blocks, 1), kThreads, 0, stream_>>>((int)n, d_pos3, 1.0 / h0_, d_bbox_);
  cuda_check(cudaGetLastError(), "bbox kernel");
  cuda_check(cudaMemcpyAsync(res, d_bbox_, sizeof(res), cudaMemcpyDeviceToHost, stream_), "bbox read");
  cuda_check(cudaStreamSynchronize(stream_), "bbox sync");
  merge_box(res, res + 3, res[6] != 0);
}

// Merges a key range into the box (throws, leaving the box unchanged, when
// the result would exceed the cell cap).
void FluidWorld::merge_box(const long long* pmn, const long long* pmx, bool any_nonfinite) {
  if (!box_valid_) grow_box_with_bounds();
  long long mn[3], mx[3];
  for (int a = 0; a < 3; ++a) {
    mn[a] = std::min(kmin_[a], pmn[a]);
    mx[a] = std::max(kmax_[a], pmx[a]);
  }
  auto cells = [](const long long* a, const long long* b) {
    long double c = 1;
    for (int q = 0; q < 3; ++q) c *= (long double)(b[q] - a[q] + 3);
    return c;
  };
  if (cells(mn, mx) > (long double)kMaxCells)
    throw std::invalid_argument("FluidWorld: particle positions span more grid cells than the 2^27-cell box");
  if (any_nonfinite) {
    long long mn0[3], mx0[3];
    for (int a = 0; a < 3; ++a) {
      mn0[a] = std::min(mn[a], 0ll);
      mx0[a] = std::max(mx[a], 0ll);
    }
    if (cells(mn0, mx0) <= (long double)kMaxCells)
      for (int a = 0; a < 3; ++a) {
        mn[a] = mn0[a];
        mx[a] = mx0[a];
      }
  }
  for (int a = 0; a < 3; ++a) {
    kmin_[a] = mn[a];
    kmax_[a] = mx[a];
  }
}

// (Re)builds the dense box: keys [kmin-1, kmax+1] per axis, so that every
// cell inside [kmin, kmax] has its 26 neighbours in the box.  The tiled form
// rounds each axis up to whole tiles and keeps a device table of scene boxes
// (one box for a single world, one per scene of a batch, numbered
// consecutively).
void FluidWorld::ensure_cells() {
  tile_ = (prec_ == Precision::F32Comp) ? comp_tile_ : 0;
  auto box_dims = [&](const long long* kmin, const long long* kmax, int* nc) {
    long long total = 1;
    for (int a = 0; a < 3; ++a) {
      long long d = kmax[a] - kmin[a] + 3;
      if (tile_) d = (d + tile_ - 1) / tile_ * tile_;
      if (d > kMaxCells) throw std::invalid_argument("FluidWorld: grid box exceeds 2^27 cells");
      nc[a] = (int)d;
      total *= d;
      if (total > kMaxCells)
        throw std::invalid_argument("FluidWorld: bounds span more than 2^27 grid cells of size h");
    }
    return total;
  };
  std::vector<SceneBox> boxes;
  long long total = 0;
  if (scenes_.empty()) {
    grow_box_with_bounds();
    int nc[3];
    total = box_dims(kmin_, kmax_, nc);
    for (int a = 0; a < 3; ++a) {
      nc_[a] = nc[a];
      bx0_[a] = kmin_[a] - 1;
    }
    if (tile_) {
      SceneBox bx;
      std::memset(&bx, 0, sizeof(bx));
      const double lo[3] = {params.bounds_min.x, params.bounds_min.y, params.bounds_min.z};
      const double hi[3] = {params.bounds_max.x, params.bounds_max.y, params.bounds_max.z};
      for (int a = 0; a < 3; ++a) {
        bx.b0[a] = bx0_[a];
        bx.nc[a] = nc[a];
        bx.nt[a] = nc[a] / tile_;
        bx.lo[a] = lo[a];
        bx.hi[a] = hi[a];
      }
      boxes.push_back(bx);
    }
  } else {
    for (const Scene& sc : scenes_) {
      SceneBox bx;
      std::memset(&bx, 0, sizeof(bx));
      int nc[3];
      const long long cells = box_dims(sc.kmin, sc.kmax, nc);
      const double lo[3] = {sc.lo.x, sc.lo.y, sc.lo.z}, hi[3] = {sc.hi.x, sc.hi.y, sc.hi.z};
      for (int a = 0; a < 3; ++a) {
        bx.b0[a] = sc.kmin[a] - 1;
        bx.nc[a] = nc[a];
        bx.nt[a] = nc[a] / tile_;
        bx.lo[a] = lo[a];
        bx.hi[a] = hi[a];
      }
      bx.cell_base = (int)total;
      total += cells;
      if (total > kMaxCells) throw std::invalid_argument("FluidWorld: the scenes' boxes exceed 2^27 cells");
      boxes.push_back(bx);
    }
  }
  ncells_ = (int)total;
  if (!boxes.empty() &&
      (boxes.size() != host_boxes_.size() ||
       std::memcmp(boxes.data(), host_boxes_.data(), boxes.size() * sizeof(SceneBox)) != 0)) {
    if ((int)boxes.size() > boxes_capacity_) {
      cuda_check(cudaStreamSynchronize(stream_), "boxes sync");
      dalloc(b_.boxes, boxes.size());
      boxes_capacity_ = (int)boxes.size();
      ++alloc_gen_;
    }
    host_boxes_ = boxes;
    cuda_check(cudaMemcpyAsync(b_.boxes, host_boxes_.data(), host_boxes_.size() * sizeof(SceneBox),
                               cudaMemcpyHostToDevice, stream_),
               "boxes upload");
    cuda_check(cudaStreamSynchronize(stream_), "boxes upload sync");
  }
  if (ncells_ > b_.cell_capacity) {
    int cap = (int)std::min<long long>(kMaxCells, std::max<long long>(ncells_, (long long)b_.cell_capacity * 3 / 2));
    size_t scan_len = scan_block_sums_needed(cap) * 4096;
    cuda_check(cudaStreamSynchronize(stream_), "cells sync");
    dalloc(b_.cell_start, scan_len);
    b_.cell_capacity = cap;
    ++alloc_gen_;
  }
  // The tiled sort's tile counts.
  if (tile_ && tile_scan_length(b_.cell_capacity) > b_.tile_scan_entries) {
    const size_t len = tile_scan_length(b_.cell_capacity);
    cuda_check(cudaStreamSynchronize(stream_), "tile scan sync");
    dalloc(b_.tile_head, len);
    b_.tile_scan_entries = len;
    ++alloc_gen_;
  }
  // The scan's tile sums serve the cell scan and the tile scan alike.
  const int sums = (int)std::max(scan_block_sums_needed(b_.cell_capacity), tile_scan_sums_needed(b_.cell_capacity));
  if (sums > b_.block_sums_capacity) {
    cuda_check(cudaStreamSynchronize(stream_), "sums sync");
    dalloc(b_.block_sums, (size_t)sums);
    b_.block_sums_capacity = sums;
    ++alloc_gen_;
  }
}

StepConsts FluidWorld::make_consts(double dt) const {
  StepConsts c;
  std::memset(&c, 0, sizeof(c));
  // Kernels::new(h0) (kernels.rs:22-35), evaluated in the same order.
  const double h = h0_;
  const double h2 = h * h, h3 = h2 * h, h6 = h3 * h3, h9 = h6 * h3;
  c.h0 = h;
  c.h0sq = h2;
  c.poly6_c = 315.0 / (64.0 * kPi * h9);
  c.spiky_c = (-45.0) / (kPi * h6);
  c.lap_c = 45.0 / (kPi * h6);
  c.inv_cell = 1.0 / h;
  c.h = params.h;
  c.r2_guard = std::nextafter(params.h * params.h, std::numeric_limits<double>::infinity());
  if (std::isnan(c.r2_guard)) c.r2_guard = std::numeric_limits<double>::quiet_NaN();
  c.rest = params.rest_density;
  c.stiff = params.stiffness;
  c.shear_min = params.shear_min;
  c.damp = params.boundary_damp;
  c.xsph_eps = params.xsph_eps;
  c.dt = dt;
  const Vec3* v[3] = {&params.gravity, &params.bounds_min, &params.bounds_max};
  double* d[3] = {c.g, c.lo, c.hi};
  for (int k = 0; k < 3; ++k) {
    d[k][0] = v[k]->x;
    d[k][1] = v[k]->y;
    d[k][2] = v[k]->z;
  }
  c.n_visc_k = (int)params.visc_k.size();
  for (size_t k = 0; k < params.visc_k.size() && k < (size_t)kMaxMaterials; ++k) c.visc_k[k] = params.visc_k[k];
  for (size_t k = 0; k < params.visc_n.size() && k < (size_t)kMaxMaterials; ++k) c.visc_n[k] = params.visc_n[k];
  c.shear_live = 0;
  for (int k = 0; k < c.n_visc_k && k < kMaxMaterials; ++k)
    if (!(c.visc_n[k] == 1.0)) c.shear_live = 1;  // NaN exponents keep it live too
  c.n = (int)n_;
  c.bx0 = bx0_[0];
  c.by0 = bx0_[1];
  c.bz0 = bx0_[2];
  c.ncx = nc_[0];
  c.ncy = nc_[1];
  c.ncz = nc_[2];
  c.ncells = ncells_;
  c.tile = tile_;
  c.tile_log2 = tile_ == 4 ? 2 : (tile_ == 2 ? 1 : 0);
  c.halo_cap = halo_cap_;
  c.dense_mean = dense_mean_;
  c.boxes = tile_ ? b_.boxes : nullptr;
  c.n_scenes = scenes_.empty() ? 1 : (int)scenes_.size();
  if (tile_) {
    c.ntx = nc_[0] / tile_;
    c.nty = nc_[1] / tile_;
    c.ntz = nc_[2] / tile_;
  }
  c.h0f = (float)h;
  c.h0sqf = (float)h2;
  c.poly6_cf = (float)c.poly6_c;
  c.spiky_cf = (float)c.spiky_c;
  c.lap_cf = (float)c.lap_c;
  c.hf = (float)params.h;
  c.h2f = (float)(params.h * params.h);
  return c;
}

double FluidWorld::lattice_mass(double s) const {
  // world.rs:148-169: uses the live params.h and the captured kernels.
  const double h = params.h;
  const double hh = h0_;
  const double h2 = hh * hh, h3 = h2 * hh, h6 = h3 * h3, h9 = h6 * h3;
  const double poly6_c = 315.0 / (64.0 * kPi * h9);
  auto poly6 = [&](double r) {
    if (r >= hh) return 0.0;
    double diff = h2 - r * r;
    return poly6_c * diff * diff * diff;
  };
  int n_shell = (int)std::ceil(h / s) + 1;
  double sum_w = 0.0;
  for (int i = -n_shell; i <= n_shell; ++i)
    for (int j = -n_shell; j <= n_shell; ++j)
      for (int l = -n_shell; l <= n_shell; ++l) {
        double rr = std::sqrt((double)(i * i + j * j + l * l));
        double r = s * rr;
        if (r < h) sum_w = sum_w + poly6(r);
      }
  return sum_w > 0.0 ? params.rest_density / sum_w : params.mass;
}

void FluidWorld::fill_box(Vec3 mn, Vec3 mx, double spacing, double margin) {
  // world.rs:124-144: float-accumulated lattice, z innermost.
  const double lo[3] = {mn.x + margin, mn.y + margin, mn.z + margin};
  const double hi[3] = {mx.x - margin, mx.y - margin, mx.z - margin};
  const double d = spacing;
  const double mass = lattice_mass(d);
  std::vector<double> pos;
  for (double x = lo[0]; x <= hi[0]; x = x + d)
    for (double y = lo[1]; y <= hi[1]; y = y + d)
      for (double z = lo[2]; z <= hi[2]; z = z + d) {
        pos.push_back(x);
        pos.push_back(y);
        pos.push_back(z);
      }
  size_t m = pos.size() / 3;
  std::vector<double> ms(m, mass);
  add_particles(m, pos.data(), nullptr, ms.data(), nullptr);
}

void FluidWorld::add_particles(size_t m, const double* pos, const double* vel, const double* mass,
                               const uint32_t* material) {
  if (m == 0) return;
  if (!pos || !mass) throw std::invalid_argument("add_particles: pos and mass are required");
  if (!scenes_.empty())
    throw std::invalid_argument("add_particles: the world holds batched scenes (clear_scenes first)");
  ensure_capacity(n_ + m);
  // Staging layout: pos 3m | vel 3m | mass m | material m (as doubles).
  std::vector<double> st(8 * m, 0.0);
  std::memcpy(st.data(), pos, 3 * m * sizeof(double));
  if (vel) std::memcpy(st.data() + 3 * m, vel, 3 * m * sizeof(double));
  std::memcpy(st.data() + 6 * m, mass, m * sizeof(double));
  if (material)
    for (size_t k = 0; k < m; ++k) st[7 * m + k] = (double)material[k];
  // stage holds 8 * capacity doubles.
  cuda_check(cudaMemcpyAsync(b_.stage, st.data(), st.size() * sizeof(double), cudaMemcpyHostToDevice, stream_),
             "append upload");
  grow_box_with_device_positions(m, b_.stage);
  ParticleConsts& pc = b_.pc[b_.cur];
  k_append<<<grid_for(m), kThreads, 0, stream_>>>((int)n_, (int)m, b_.stage, b_.pv1[0], b_.pv1[1], b_.pv1[2],
                                                  b_.pv1[3], b_.pv1[4], b_.pv1[5], pc.mass, pc.mat, pc.id);
  // Particle::new: acc, rho, p, mu_eff, xsph start at zero (particle.rs:50-63).
  size_t bytes = m * sizeof(double);
  cuda_check(cudaMemsetAsync(b_.rho + n_, 0, bytes, stream_), "memset");
  cuda_check(cudaMemsetAsync(b_.p + n_, 0, bytes, stream_), "memset");
  cuda_check(cudaMemsetAsync(b_.mu + n_, 0, bytes, stream_), "memset");
  for (int k = 0; k < 3; ++k) {
    cuda_check(cudaMemsetAsync(b_.acc[k] + n_, 0, bytes, stream_), "memset");
    cuda_check(cudaMemsetAsync(b_.xsph[k] + n_, 0, bytes, stream_), "memset");
    if (b_.has_ba) cuda_check(cudaMemsetAsync(pc.ba[k] + n_, 0, bytes, stream_), "memset");
  }
  cuda_check(cudaGetLastError(), "append kernel");
  n_ += m;
  // The staging vector must outlive the copy.
  cuda_check(cudaStreamSynchronize(stream_), "append sync");
}

// Device-side twin of k_append for set_particles_device: material as u32.
__global__ void k_load_dev(int m, const double* __restrict__ pos, const double* __restrict__ vel,
                           const double* __restrict__ mass, const uint32_t* __restrict__ material, double* px,
                           double* py, double* pz, double* vx, double* vy, double* vz, double* ms, uint32_t* mat,
                           uint32_t* id) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  px[k] = pos[3 * (size_t)k];
  py[k] = pos[3 * (size_t)k + 1];
  pz[k] = pos[3 * (size_t)k + 2];
  vx[k] = vel ? vel[3 * (size_t)k] : 0.0;
  vy[k] = vel ? vel[3 * (size_t)k + 1] : 0.0;
  vz[k] = vel ? vel[3 * (size_t)k + 2] : 0.0;
  ms[k] = mass[k];
  mat[k] = material ? material[k] : 0u;
  id[k] = (uint32_t)k;
}

void FluidWorld::set_particles_device(size_t m, const double* pos, const double* vel, const double* mass,
                                      const uint32_t* material) {
  if (m > 0 && (!pos || !mass)) throw std::invalid_argument("set_particles_device: pos and mass are required");
  if (!scenes_.empty()) throw std::invalid_argument("set_particles_device: the world holds batched scenes");
  if (tape_.on) throw std::invalid_argument("set_particles_device: the adjoint tape is recording");
  if (m > (size_t)INT32_MAX) throw std::invalid_argument("set_particles_device: too many particles");
  n_ = 0;
  if (m == 0) return;
  ensure_capacity(m);
  // The positions, read from the caller's device buffer, may widen the grid box.
  cuda_check(cudaMemcpyAsync(b_.stage, pos, 3 * m * sizeof(double), cudaMemcpyDeviceToDevice, stream_),
             "set_particles_device positions");
  grow_box_with_device_positions(m, b_.stage);
  ParticleConsts& pc = b_.pc[b_.cur];
  k_load_dev<<<grid_for(m), kThreads, 0, stream_>>>((int)m, pos, vel, mass, material, b_.pv1[0], b_.pv1[1],
                                                    b_.pv1[2], b_.pv1[3], b_.pv1[4], b_.pv1[5], pc.mass, pc.mat,
                                                    pc.id);
  // Particle::new: acc, rho, p, mu_eff, xsph, body_acc start at zero (particle.rs:50-63).
  const size_t bytes = m * sizeof(double);
  cuda_check(cudaMemsetAsync(b_.rho, 0, bytes, stream_), "memset");
  cuda_check(cudaMemsetAsync(b_.p, 0, bytes, stream_), "memset");
  cuda_check(cudaMemsetAsync(b_.mu, 0, bytes, stream_), "memset");
  for (int k = 0; k < 3; ++k) {
    cuda_check(cudaMemsetAsync(b_.acc[k], 0, bytes, stream_), "memset");
    cuda_check(cudaMemsetAsync(b_.xsph[k], 0, bytes, stream_), "memset");
    if (b_.has_ba) cuda_check(cudaMemsetAsync(pc.ba[k], 0, bytes, stream_), "memset");
  }
  cuda_check(cudaGetLastError(), "set_particles_device kernel");
  n_ = m;
  cuda_check(cudaStreamSynchronize(stream_), "set_particles_device sync");
}

void FluidWorld::get_field_device(int field, double* out) {
  if (components(field) == 0) throw std::invalid_argument("get_field_device: unknown field");
  if (n_ == 0) return;
  if (!out) throw std::invalid_argument("get_field_device: null output");
  stage_field(field, out);
  cuda_check(cudaGetLastError(), "get_field_device kernel");
  cuda_check(cudaStreamSynchronize(stream_), "get_field_device sync");
}

int FluidWorld::components(int field) {
  switch (field) {
    case PHY_FIELD_POS:
    case PHY_FIELD_VEL:
    case PHY_FIELD_ACC:
    case PHY_FIELD_BODY_ACC:
    case PHY_FIELD_XSPH:
      return 3;
    case PHY_FIELD_RHO:
    case PHY_FIELD_P:
    case PHY_FIELD_MASS:
    case PHY_FIELD_MU_EFF:
    case PHY_FIELD_MATERIAL:
      return 1;
    default:
      return 0;
  }
}

// Field `field` of every particle in insertion order into device memory `st`
// (3n or n doubles), on the world's stream.
void FluidWorld::stage_field(int field, double* st) {
  const int n = (int)n_;
  const ParticleConsts& pc = b_.pc[b_.cur];
  switch (field) {
    case PHY_FIELD_POS:
      k_get_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, b_.pv1[0], b_.pv1[1], b_.pv1[2], st);
      break;
    case PHY_FIELD_VEL:
      k_get_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, b_.pv1[3], b_.pv1[4], b_.pv1[5], st);
      break;
    case PHY_FIELD_ACC:
      k_get_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, b_.acc[0], b_.acc[1], b_.acc[2], st);
      break;
    case PHY_FIELD_XSPH:
      k_get_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, b_.xsph[0], b_.xsph[1], b_.xsph[2], st);
      break;
    case PHY_FIELD_BODY_ACC:
      if (b_.has_ba)
        k_get_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, pc.ba[0], pc.ba[1], pc.ba[2], st);
      else
        cuda_check(cudaMemsetAsync(st, 0, 3 * n_ * sizeof(double), stream_), "memset");
      break;
    case PHY_FIELD_RHO:
      k_get_scalar_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, b_.rho, st);
      break;
    case PHY_FIELD_P:
      k_get_scalar_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, b_.p, st);
      break;
    case PHY_FIELD_MASS:
      k_get_scalar_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, pc.mass, st);
      break;
    case PHY_FIELD_MU_EFF:
      k_get_scalar_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, b_.mu, st);
      break;
    case PHY_FIELD_MATERIAL:
      launch_unsort_u32(b_, n, pc.mat, st, stream_);
      break;
  }
}

void FluidWorld::get_field(int field, double* out) {
  int nc = components(field);
  if (nc == 0) throw std::invalid_argument("get_field: unknown field");
  if (n_ == 0) return;
  double* st = b_.stage;
  stage_field(field, st);
  cuda_check(cudaGetLastError(), "get_field kernel");
  cuda_check(cudaMemcpyAsync(out, st, (size_t)nc * n_ * sizeof(double), cudaMemcpyDeviceToHost, stream_),
             "get_field copy");
  cuda_check(cudaStreamSynchronize(stream_), "get_field sync");
}

void FluidWorld::get_vec_f64(int field, double* out, size_t count) {
  if (field != PHY_FIELD_POS && field != PHY_FIELD_VEL) throw std::invalid_argument("get_vec_f64: pos or vel only");
  if (n_ == 0 || count == 0) return;
  if (count > n_) count = n_;
  const int n = (int)n_;
  const ParticleConsts& pc = b_.pc[b_.cur];
  double* st = b_.stage;
  const int o = field == PHY_FIELD_POS ? 0 : 3;
  k_get_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, b_.pv1[o], b_.pv1[o + 1], b_.pv1[o + 2], st);
  cuda_check(cudaGetLastError(), "get_vec_f64 kernel");
  // The stage is in insertion order, so the first `count` particles are its
  // first 3 * count values: one copy straight into the caller's buffer (a DMA
  // when the caller registered it with phy_fluid_pin_host).
  cuda_check(cudaMemcpyAsync(out, st, 3 * count * sizeof(double), cudaMemcpyDeviceToHost, stream_),
             "get_vec_f64 copy");
  cuda_check(cudaStreamSynchronize(stream_), "get_vec_f64 sync");
}

void FluidWorld::get_vec_f32(int field, float* out, size_t count) {
  if (field != PHY_FIELD_POS && field != PHY_FIELD_VEL) throw std::invalid_argument("get_vec_f32: pos or vel only");
  if (n_ == 0 || count == 0) return;
  if (count > n_) count = n_;
  const int n = (int)n_;
  const ParticleConsts& pc = b_.pc[b_.cur];
  float* st = reinterpret_cast<float*>(b_.stage);  // 3n floats fit the 8n-double stage
  const int o = field == PHY_FIELD_POS ? 0 : 3;
  k_get_vec_f32_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, b_.pv1[o], b_.pv1[o + 1], b_.pv1[o + 2], st);
  cuda_check(cudaGetLastError(), "get_vec_f32 kernel");
  cuda_check(cudaMemcpyAsync(out, st, 3 * count * sizeof(float), cudaMemcpyDeviceToHost, stream_), "get_vec_f32 copy");
  cuda_check(cudaStreamSynchronize(stream_), "get_vec_f32 sync");
}

void FluidWorld::set_field(int field, const double* in) {
  int nc = components(field);
  if (nc == 0) throw std::invalid_argument("set_field: unknown field");
  if (n_ == 0) return;
  const int n = (int)n_;
  ParticleConsts& pc = b_.pc[b_.cur];
  double* st = b_.stage;
  cuda_check(cudaMemcpyAsync(st, in, (size_t)nc * n_ * sizeof(double), cudaMemcpyHostToDevice, stream_),
             "set_field copy");
  // New positions may widen the grid box; checked before the state changes.
  if (field == PHY_FIELD_POS) {
    if (scenes_.empty())
      grow_box_with_device_positions(n_, st);
    else
      grow_scene_boxes(st);
  }
  if (field == PHY_FIELD_BODY_ACC && !b_.has_ba) {
    for (int q = 0; q < 2; ++q)
      for (int k = 0; k < 3; ++k) dgrow(b_.pc[q].ba[k], 0, (size_t)b_.capacity, stream_);
    b_.has_ba = true;
    ++alloc_gen_;
  }
  switch (field) {
    case PHY_FIELD_POS:
      k_set_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, st, b_.pv1[0], b_.pv1[1], b_.pv1[2]);
      break;
    case PHY_FIELD_VEL:
      k_set_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, st, b_.pv1[3], b_.pv1[4], b_.pv1[5]);
      break;
    case PHY_FIELD_ACC:
      k_set_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, st, b_.acc[0], b_.acc[1], b_.acc[2]);
      break;
    case PHY_FIELD_XSPH:
      k_set_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, st, b_.xsph[0], b_.xsph[1], b_.xsph[2]);
      break;
    case PHY_FIELD_BODY_ACC:
      k_set_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, st, pc.ba[0], pc.ba[1], pc.ba[2]);
      break;
    case PHY_FIELD_RHO:
      k_set_scalar_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, st, b_.rho);
      break;
    case PHY_FIELD_P:
      k_set_scalar_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, st, b_.p);
      break;
    case PHY_FIELD_MASS:
      k_set_scalar_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, st, pc.mass);
      break;
    case PHY_FIELD_MU_EFF:
      k_set_scalar_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, st, b_.mu);
      break;
    case PHY_FIELD_MATERIAL:
      k_set_u32_by_id<<<grid_for(n_), kThreads, 0, stream_>>>(n, pc.id, st, pc.mat);
      break;
  }
  cuda_check(cudaGetLastError(), "set_field kernel");
  // The caller's buffer may be reused as soon as we return.
  cuda_check(cudaStreamSynchronize(stream_), "set_field sync");
}

// Validation, grid box and launch constants of a step (host work only, no
// device synchronisation unless a buffer grows).
StepConsts FluidWorld::prepare_step(double dt) {
  if (params.visc_k.empty() || params.visc_k.size() > (size_t)kMaxMaterials)
    throw std::invalid_argument("step: visc_k must hold 1..16 entries");
  if (params.visc_n.size() < params.visc_k.size())
    throw std::invalid_argument("step: visc_n shorter than visc_k (the reference would index out of bounds)");
  if (!scenes_.empty() && !(prec_ == Precision::F32Comp && comp_tile_ > 0))
    throw std::invalid_argument("step: batched scenes need the tiled compensated form");
  ensure_cells();
  if (prec_ == Precision::F32Comp && comp_tile_ > 0) ensure_masks();
  return make_consts(dt);
}

// Grows the dense-cell mask buffer ahead of the entries the dense-cell tasks
// reserve.  The host reads the demand of a recent step from its pinned copy,
// which lags by the steps still in flight (hundreds when a caller enqueues a
// long run), and a collapsing fluid's demand keeps rising meanwhile; so once
// the demand passes three quarters of the buffer it is re-read after a wait
// and the buffer grows to three times it, and at least to 12 entries per
// particle (a fluid collapsed to a thousand particles per cell reserves about
// 8) and 2^20 entries, within a quarter of the free device memory and 16 GiB.  Tasks that find no room
// filter again in the force pass, so the size never changes a result.  A
// failed allocation leaves the buffer empty and is not retried below the
// demand that failed.
void FluidWorld::ensure_masks() {
  if (!tuning_.dense_masks || !b_.mask_ctl || !b_.mask_demand) return;
  const volatile unsigned long long* demand = b_.mask_demand;
  const unsigned long long seen = *demand;
  if (seen == 0 || 4 * seen <= 3 * b_.mask_cap || seen <= mask_tried_) return;
  mask_tried_ = seen;
  constexpr unsigned long long kEntryBytes = 33 * sizeof(uint32_t);
  cuda_check(cudaStreamSynchronize(stream_), "mask buffer sync");
  const unsigned long long want = std::max(seen, (unsigned long long)*demand);  // current after the wait
  size_t free_b = 0, total_b = 0;
  cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
  const unsigned long long limit = std::min<unsigned long long>(
      std::min<unsigned long long>(free_b / 4 + b_.mask_cap * kEntryBytes, 16ull << 30) / kEntryBytes,
      0xfffffffeull);
  const unsigned long long cap = std::min(std::max({3 * want, 12ull * n_, 1ull << 20}), limit);
  if (cap <= b_.mask_cap) return;
  dfree(b_.mask_hdr);
  dfree(b_.mask_bits);
  b_.mask_cap = 0;
  ++alloc_gen_;
  if (cudaMalloc((void**)&b_.mask_hdr, cap * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc((void**)&b_.mask_bits, cap * 32 * sizeof(uint32_t)) != cudaSuccess) {
    (void)cudaGetLastError();
    dfree(b_.mask_hdr);
    dfree(b_.mask_bits);
    return;
  }
  b_.mask_cap = cap;
}

// The device work of one step on the world's stream.
void FluidWorld::enqueue_step(const StepConsts& c, const PassEvents& pe, const cudaEvent_t* ev) {
  cuda_check(cudaMemsetAsync(b_.flags, 0, sizeof(uint32_t), stream_), "flags reset");
  if (counting_) cuda_check(cudaMemsetAsync(b_.counters, 0, 2 * sizeof(unsigned long long), stream_), "memset");
  unsigned long long* saved = b_.counters;
  if (!counting_) b_.counters = nullptr;
  if (ev) cuda_check(cudaEventRecord(ev[0], stream_), "event");
  launch_sort(c, b_, stream_, tuning_.sort_block);
  if (ev) cuda_check(cudaEventRecord(ev[1], stream_), "event");
  if (prec_ == Precision::F64Plain)
    launch_plain_passes(c, b_, stream_, pe);
  else if (tile_)
    launch_comp_tiled(c, b_, stream_, pe, tuning_);
  else
    launch_comp_passes(c, b_, stream_, pe);
  b_.counters = saved;
  cuda_check(cudaGetLastError(), "step launch");
}

void FluidWorld::step(double dt) {
  if (n_ == 0) return;  // world.rs:184-186
  step_impl(dt);
}

// One step; returns the launch constants it ran with.
StepConsts FluidWorld::step_impl(double dt) {
  if (tape_.on && !recomputing_) {
    const PhySphParams now = params.to_c();
    if (std::memcmp(&now, &tape_.params, sizeof(now)) != 0)
      throw std::invalid_argument("step: parameters changed while the adjoint tape is recording");
    if (b_.has_ba) throw std::invalid_argument("step: body accelerations are not recorded by the adjoint tape");
    if (!tape_.dts.empty() && tape_.dts.size() % (size_t)tape_.every == 0) save_checkpoint();
    tape_.dts.push_back(dt);
  }
  StepConsts c = prepare_step(dt);
  PassEvents pe;
  cudaEvent_t* ev = nullptr;
  if (timing_) {
    if (ev_used_ == 4096) collect_phase_times();  // bounds the pool
    if (ev_used_ == ev_pool_.size()) {
      std::array<cudaEvent_t, 5> set;
      for (auto& e : set) cuda_check(cudaEventCreate(&e), "cudaEventCreate");
      ev_pool_.push_back(set);
    }
    ev = ev_pool_[ev_used_++].data();
    pe.after_prep = ev[2];
    pe.after_density = ev[3];
  }
  enqueue_step(c, pe, ev);
  if (ev) cuda_check(cudaEventRecord(ev[4], stream_), "event");
  return c;
}

void FluidWorld::step_n(double dt, int n) {
  if (n_ == 0 || n <= 0) return;
  if (graph_chunk_ > 0 && !timing_ && !tape_.on)
    for (; n >= graph_chunk_; n -= graph_chunk_) run_graph(dt, graph_chunk_);
  for (; n > 0; --n) step(dt);
}

void FluidWorld::drop_graphs() {
  for (auto& g : graphs_) cudaGraphExecDestroy(g.exec);
  graphs_.clear();
}

// k steps as one CUDA graph.  The key holds every value a captured launch
// bakes in: the launch constants (parameters, dt, box, particle count), the
// buffer generation, the double-buffer parity, counting, body_acc, the
// launch knobs and the stream.
void FluidWorld::run_graph(double dt, int k) {
  const StepConsts c = prepare_step(dt);
  if (tile_) (void)tiled_max_ctas_per_sm();  // one-time attribute setup, outside the capture
  std::vector<unsigned char> key(sizeof(StepConsts) + 64, 0);
  std::memcpy(key.data(), &c, sizeof(StepConsts));
  long long extra[8] = {k, (long long)alloc_gen_, b_.cur, counting_ ? 1 : 0, b_.has_ba ? 1 : 0,
                        tuning_.ctas_per_sm + 1000ll * tuning_.queue + 10000ll * tuning_.dense_masks,
                        tuning_.sort_block,
                        (long long)(uintptr_t)stream_};
  std::memcpy(key.data() + sizeof(StepConsts), extra, sizeof(extra));
  const int cur0 = b_.cur;
  cudaGraphExec_t exec = nullptr;
  for (auto& g : graphs_)
    if (g.key == key) exec = g.exec;
  if (!exec) {
    cudaGraph_t graph = nullptr;
    cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "graph capture");
    try {
      PassEvents none;
      for (int q = 0; q < k; ++q) enqueue_step(c, none, nullptr);
    } catch (...) {
      cudaStreamEndCapture(stream_, &graph);
      if (graph) cudaGraphDestroy(graph);
      b_.cur = cur0;
      throw;
    }
    cuda_check(cudaStreamEndCapture(stream_, &graph), "graph capture end");
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    cuda_check(e, "graph instantiate");
    if (graphs_.size() >= 4) {
      cudaGraphExecDestroy(graphs_.front().exec);
      graphs_.erase(graphs_.begin());
    }
    graphs_.push_back({key, exec});
  }
  b_.cur = cur0;
  cuda_check(cudaGraphLaunch(exec, stream_), "graph launch");
  b_.cur = cur0 ^ (k & 1);
}

// ---- Batched scenes ---------------------------------------------------------

void FluidWorld::set_scenes(const std::vector<uint64_t>& counts, const std::vector<Vec3>& lo,
                            const std::vector<Vec3>& hi) {
  if (prec_ != Precision::F32Comp || comp_tile_ == 0)
    throw std::invalid_argument("set_scenes: batched scenes need the tiled compensated form");
  if (counts.empty() || counts.size() > 65535 || lo.size() != counts.size() || hi.size() != counts.size())
    throw std::invalid_argument("set_scenes: 1..65535 scenes, one bounds pair each");
  uint64_t sum = 0;
  for (uint64_t c : counts) sum += c;
  if (sum != n_) throw std::invalid_argument("set_scenes: scene counts must add up to the particle count");
  const double inv = 1.0 / h0_;
  std::vector<Scene> sc(counts.size());
  std::vector<uint32_t> pbase(counts.size() + 1, 0);
  uint64_t first = 0;
  for (size_t s = 0; s < counts.size(); ++s) {
    sc[s].first = first;
    sc[s].count = counts[s];
    sc[s].lo = lo[s];
    sc[s].hi = hi[s];
    const double l[3] = {lo[s].x, lo[s].y, lo[s].z}, h[3] = {hi[s].x, hi[s].y, hi[s].z};
    for (int a = 0; a < 3; ++a) {
      const long long k0 = key_axis_host(l[a], inv), k1 = key_axis_host(h[a], inv);
      sc[s].kmin[a] = std::min(k0, k1);
      sc[s].kmax[a] = std::max(k0, k1);
    }
    pbase[s] = (uint32_t)first;
    first += counts[s];
  }
  pbase[counts.size()] = (uint32_t)first;
  cuda_check(cudaStreamSynchronize(stream_), "scenes sync");
  dalloc(d_pbase_, pbase.size());
  cuda_check(cudaMemcpy(d_pbase_, pbase.data(), pbase.size() * sizeof(uint32_t), cudaMemcpyHostToDevice),
             "pbase upload");
  for (int q = 0; q < 2; ++q)
    if (!b_.pc[q].scene) dalloc(b_.pc[q].scene, (size_t)std::max(b_.capacity, 1));
  ++alloc_gen_;
  if (n_ > 0)
    k_scene_of_id<<<grid_for(n_), kThreads, 0, stream_>>>((int)n_, b_.pc[b_.cur].id, d_pbase_, (int)counts.size(),
                                                           b_.pc[b_.cur].scene);
  cuda_check(cudaGetLastError(), "scene ids");
  scenes_ = sc;
  // Positions (insertion order) widen each scene's box.
  if (n_ > 0) {
    k_get_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>((int)n_, b_.pc[b_.cur].id, b_.pv1[0], b_.pv1[1],
                                                             b_.pv1[2], b_.stage);
    grow_scene_boxes(b_.stage);
  }
  ensure_cells();
}

// Widens each scene's key range with its finite positions (interleaved xyz
// in insertion order on the device); throws, leaving the ranges unchanged,
// when the boxes would exceed the cell cap.
void FluidWorld::grow_scene_boxes(const double* d_pos3) {
  const int ns = (int)scenes_.size();
  dalloc(d_scene_bbox_, 7 * (size_t)ns);
  k_scene_bbox<<<ns, kThreads, 0, stream_>>>(d_pos3, d_pbase_, 1.0 / h0_, d_scene_bbox_);
  cuda_check(cudaGetLastError(), "scene bbox");
  std::vector<long long> r(7 * (size_t)ns);
  cuda_check(cudaMemcpyAsync(r.data(), d_scene_bbox_, r.size() * sizeof(long long), cudaMemcpyDeviceToHost, stream_),
             "scene bbox read");
  cuda_check(cudaStreamSynchronize(stream_), "scene bbox sync");
  std::vector<Scene> sc = scenes_;
  long double total = 0;
  for (int s = 0; s < ns; ++s) {
    long double cells = 1;
    for (int a = 0; a < 3; ++a) {
      if (sc[s].count > 0 && r[7 * s + a] != LLONG_MAX) {
        sc[s].kmin[a] = std::min(sc[s].kmin[a], r[7 * s + a]);
        sc[s].kmax[a] = std::max(sc[s].kmax[a], r[7 * s + 3 + a]);
      }
      cells *= (long double)(sc[s].kmax[a] - sc[s].kmin[a] + 3 + 3);
    }
    total += cells;
  }
  if (total > (long double)kMaxCells)
    throw std::invalid_argument("FluidWorld: the scenes' positions span more than 2^27 grid cells");
  scenes_ = sc;
}

void FluidWorld::clear_scenes() {
  scenes_.clear();
  host_boxes_.clear();
  for (int q = 0; q < 2; ++q) dfree(b_.pc[q].scene);
  ++alloc_gen_;
}

// ---- Autotuner ----------------------------------------------------------------

// Saves (restore = false) or restores (restore = true) the particle state a
// step reads and the outputs it leaves: pv1, the current per-particle
// constants, rho, p, acc, xsph and mu.  The saved copy is kept until
// release_snapshot().
void FluidWorld::snapshot(bool restore, int slot, bool sync) {
  if (slot < 0 || slot >= kSnapSlots) throw std::logic_error("snapshot: slot out of range");
  const size_t n = n_;
  if (restore) b_.cur = snap_cur_[slot];
  ParticleConsts& pc = b_.pc[b_.cur];
  std::vector<std::pair<void*, size_t>> arrays;
  for (int k = 0; k < 6; ++k) arrays.push_back({b_.pv1[k], n * 8});
  arrays.push_back({pc.mass, n * 8});
  arrays.push_back({pc.mat, n * 4});
  arrays.push_back({pc.id, n * 4});
  if (pc.scene) arrays.push_back({pc.scene, n * 2});
  if (b_.has_ba)
    for (int k = 0; k < 3; ++k) arrays.push_back({pc.ba[k], n * 8});
  arrays.push_back({b_.rho, n * 8});
  arrays.push_back({b_.p, n * 8});
  arrays.push_back({b_.mu, n * 8});
  for (int k = 0; k < 3; ++k) {
    arrays.push_back({b_.acc[k], n * 8});
    arrays.push_back({b_.xsph[k], n * 8});
  }
  // One arena, reused while large enough; each array at a 256-byte offset.
  std::vector<size_t> off(arrays.size());
  size_t total = 0;
  for (size_t q = 0; q < arrays.size(); ++q) {
    off[q] = total;
    total += (arrays[q].second + 255) / 256 * 256;
  }
  if (arrays.size() > (size_t)ArrayCopy::kMax) throw std::logic_error("snapshot: too many arrays");
  if (!restore) {
    if (total > snap_bytes_[slot]) {
      dfree(snap_arena_[slot]);
      snap_bytes_[slot] = 0;
      dalloc(snap_arena_[slot], total / 8);
      snap_bytes_[slot] = total;
    }
    snap_cur_[slot] = b_.cur;
    snap_count_[slot] = arrays.size();
  } else if (snap_count_[slot] != arrays.size() || !snap_arena_[slot]) {
    throw std::logic_error("snapshot: no saved state of this layout");
  }
  ArrayCopy ac{};
  size_t widest = 0;
  for (size_t q = 0; q < arrays.size(); ++q) {
    unsigned char* saved = reinterpret_cast<unsigned char*>(snap_arena_[slot]) + off[q];
    unsigned char* live = static_cast<unsigned char*>(arrays[q].first);
    ac.src[q] = restore ? saved : live;
    ac.dst[q] = restore ? live : saved;
    ac.bytes[q] = arrays[q].second;
    widest = std::max(widest, arrays[q].second);
  }
  if (widest > 0) {
    const size_t blocks = std::min<size_t>((widest / 16 + kThreads - 1) / kThreads + 1, 1184);
    k_copy_arrays<<<dim3((unsigned)blocks, (unsigned)arrays.size()), kThreads, 0, stream_>>>(ac);
    cuda_check(cudaGetLastError(), restore ? "restore" : "snapshot");
  }
  if (sync) cuda_check(cudaStreamSynchronize(stream_), "snapshot sync");
}

void FluidWorld::release_snapshot() {
  for (int q = 0; q < kSnapSlots; ++q) {
    dfree(snap_arena_[q]);
    snap_bytes_[q] = 0;
    snap_count_[q] = 0;
  }
}

double FluidWorld::time_tuning(const LaunchTuning& t, int comp_tile, double dt, int steps, int nslots,
                               cudaEvent_t e0, cudaEvent_t e1) {
  double total = 0.0;
  for (int slot = 0; slot < nslots; ++slot) {
    snapshot(true, slot);
    tuning_ = t;
    if (comp_tile != comp_tile_) set_comp_tile(comp_tile);
    step_n(dt, 1);  // warm-up (and graph capture when chunked)
    if (graph_chunk_ > 0) step_n(dt, graph_chunk_);
    cuda_check(cudaEventRecord(e0, stream_), "event");
    step_n(dt, steps);
    cuda_check(cudaEventRecord(e1, stream_), "event");
    cuda_check(cudaEventSynchronize(e1), "event sync");
    float ms = 0.f;
    cuda_check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
    total += (double)ms / steps;
  }
  return total / nslots;
}

// Candidates: sort block 128/256, static tile stride or work queue, 1..the
// occupancy limit of CTAs per SM, and (tiled worlds) 4 or 2 cells per tile
// edge.  With horizon > 0 the states the run will meet are sampled first:
// the current state, and the states after horizon/2 and horizon steps of the
// current configuration.  Every candidate runs `steps` steps from the first
// sample; the kKeep fastest then also run from the other samples, and the
// fastest mean over all samples wins (successive halving keeps the tuning
// time near one pass over the candidates).  The world returns to its
// starting state.
std::vector<TuneTrial> FluidWorld::autotune(double dt, int steps, int horizon) {
  std::vector<TuneTrial> trials;
  if (n_ == 0 || steps <= 0) return trials;
  if (timing_) throw std::invalid_argument("autotune: phase timing is on");
  if (horizon < 0) throw std::invalid_argument("autotune: negative horizon");
  const bool tiled = prec_ == Precision::F32Comp && comp_tile_ > 0;
  const int max_per_sm = tiled ? tiled_max_ctas_per_sm() : 1;
  std::vector<std::pair<LaunchTuning, int>> cands;
  const std::vector<int> tiles = tiled ? std::vector<int>{4, 2} : std::vector<int>{comp_tile_};
  for (int tile : tiles)
    for (int sort_block : {128, 256})
      for (int queue = 0; queue <= (tiled ? 1 : 0); ++queue)
        for (int per = 1; per <= max_per_sm; ++per) {
          LaunchTuning t;
          t.ctas_per_sm = tiled ? per : 0;
          t.queue = queue;
          t.sort_block = sort_block;
          cands.push_back({t, tile});
        }
  const LaunchTuning saved = tuning_;
  const int saved_tile = comp_tile_;
  snapshot(false, 0);
  int nslots = 1;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cuda_check(cudaEventCreate(&e0), "event");
  cuda_check(cudaEventCreate(&e1), "event");
  auto restore_start = [&]() {
    tuning_ = saved;
    if (comp_tile_ != saved_tile) set_comp_tile(saved_tile);
    snapshot(true, 0);
  };
  try {
    if (horizon > 0) {
      step_n(dt, horizon / 2);
      snapshot(false, 1);
      step_n(dt, horizon - horizon / 2);
      snapshot(false, 2);
      nslots = 3;
    }
    for (const auto& cand : cands)
      trials.push_back({cand.first, cand.second, time_tuning(cand.first, cand.second, dt, steps, 1, e0, e1), 1});
    if (nslots > 1) {
      constexpr size_t kKeep = 6;
      std::vector<size_t> order(trials.size());
      for (size_t q = 0; q < order.size(); ++q) order[q] = q;
      std::stable_sort(order.begin(), order.end(),
                       [&](size_t x, size_t y) { return trials[x].ms_per_step < trials[y].ms_per_step; });
      for (size_t r = 0; r < std::min(kKeep, order.size()); ++r) {
        TuneTrial& tr = trials[order[r]];
        tr.ms_per_step = time_tuning(tr.tuning, tr.comp_tile, dt, steps, nslots, e0, e1);
        tr.samples = nslots;
      }
    }
    restore_start();
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    try {
      restore_start();
    } catch (...) {
    }
    release_snapshot();
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  release_snapshot();
  // The fastest among the trials that ran on every sample.
  size_t best = trials.size();
  for (size_t q = 0; q < trials.size(); ++q)
    if (trials[q].samples == nslots && (best == trials.size() || trials[q].ms_per_step < trials[best].ms_per_step))
      best = q;
  tuning_ = trials[best].tuning;
  if (trials[best].comp_tile != comp_tile_) set_comp_tile(trials[best].comp_tile);
  return trials;
}

void FluidWorld::set_timing(bool on) { timing_ = on; }

// Waits for the last timed step and adds every recorded step's phases.
void FluidWorld::collect_phase_times() {
  if (ev_used_ == 0) return;
  cuda_check(cudaEventSynchronize(ev_pool_[ev_used_ - 1][4]), "event sync");
  for (size_t q = 0; q < ev_used_; ++q)
    for (int k = 0; k < 4; ++k) {
      float ms = 0.f;
      cuda_check(cudaEventElapsedTime(&ms, ev_pool_[q][k], ev_pool_[q][k + 1]), "elapsed");
      phase_ms_[k] += ms;
    }
  timed_steps_ += (double)ev_used_;
  ev_used_ = 0;
}

void FluidWorld::phase_times(double* out5, bool reset) {
  collect_phase_times();
  for (int k = 0; k < 4; ++k) out5[k] = phase_ms_[k];
  out5[4] = timed_steps_;
  if (reset) {
    for (auto& v : phase_ms_) v = 0;
    timed_steps_ = 0;
  }
}

uint32_t FluidWorld::last_step_flags() {
  uint32_t f = 0;
  cuda_check(cudaMemcpyAsync(&f, b_.flags, sizeof(f), cudaMemcpyDeviceToHost, stream_), "flags");
  cuda_check(cudaStreamSynchronize(stream_), "flags sync");
  return f;
}

void FluidWorld::dense_mask_info(uint64_t* out3) {
  cuda_check(cudaStreamSynchronize(stream_), "mask info sync");
  out3[0] = b_.mask_cap;
  out3[1] = b_.mask_demand ? *reinterpret_cast<volatile unsigned long long*>(b_.mask_demand) : 0;
  out3[2] = (last_step_flags() & kFlagMaskTable) ? 1 : 0;
}

void FluidWorld::last_step_counters(uint64_t* out2) {
  unsigned long long v[2];
  cuda_check(cudaMemcpyAsync(v, b_.counters, sizeof(v), cudaMemcpyDeviceToHost, stream_), "counters");
  cuda_check(cudaStreamSynchronize(stream_), "counters sync");
  out2[0] = v[0];
  out2[1] = v[1];
}

void FluidWorld::diagnostics(double* out4) {
  // Serial f64 sums in insertion order, like the reference's loops.
  std::vector<double> vel(3 * n_), mass(n_);
  get_field(PHY_FIELD_VEL, vel.data());
  get_field(PHY_FIELD_MASS, mass.data());
  double px = 0, py = 0, pz = 0, e = 0;
  for (size_t i = 0; i < n_; ++i) {
    double vx = vel[3 * i], vy = vel[3 * i + 1], vz = vel[3 * i + 2], m = mass[i];
    px = px + vx * m;
    py = py + vy * m;
    pz = pz + vz * m;
  }
  for (size_t i = 0; i < n_; ++i) {
    double vx = vel[3 * i], vy = vel[3 * i + 1], vz = vel[3 * i + 2];
    double n2 = (vx * vx + vy * vy) + vz * vz;
    e = e + (n2 * mass[i]) / (1.0 + 1.0);
  }
  out4[0] = px;
  out4[1] = py;
  out4[2] = pz;
  out4[3] = e;
}

// world.rs:691-752 (kernel and semantics in couple.cu).  The cell index of the
// current positions is built without moving the state, so the step's sorted
// arrays and outputs stay as they were; only fluid velocities change.
void FluidWorld::couple_points(size_t np, const double* pos, const double* vel, const double* mass, double* force,
                               double dt, double drag, double soft_density) {
  if (np == 0 || n_ == 0) return;  // world.rs:692-694
  if (!pos || !vel || !mass || !force) throw std::invalid_argument("couple_points: null array");
  if (!scenes_.empty()) throw std::invalid_argument("couple_points: not available for batched scenes");
  if (tape_.on) throw std::invalid_argument("couple_points: the adjoint tape does not record coupling");
  if (np > ((size_t)1 << 24)) throw std::invalid_argument("couple_points: more than 2^24 points");
  ensure_cells();
  StepConsts c = make_consts(dt);
  c.tile = 0;  // x-major cells for the index
  c.tile_log2 = 0;
  const size_t need = 10 * np + 1;
  if (couple_cap_ < need) {
    dalloc(d_couple_, need);
    couple_cap_ = need;
  }
  std::vector<double> h(10 * np);
  for (size_t k = 0; k < np; ++k) {
    double* r = h.data() + 10 * k;
    for (int a = 0; a < 3; ++a) {
      r[a] = pos[3 * k + a];
      r[3 + a] = vel[3 * k + a];
      r[7 + a] = force[3 * k + a];
    }
    r[6] = mass[k];
  }
  const size_t bytes = h.size() * sizeof(double);
  cuda_check(cudaMemcpyAsync(d_couple_, h.data(), bytes, cudaMemcpyHostToDevice, stream_), "couple upload");
  launch_cell_index(c, b_, reinterpret_cast<uint32_t*>(d_couple_ + 10 * np), stream_);
  launch_couple_points(c, b_, d_couple_, (int)np, dt, drag, soft_density, stream_, couple_scratch_);
  cuda_check(cudaGetLastError(), "couple launch");
  cuda_check(cudaMemcpyAsync(h.data(), d_couple_, bytes, cudaMemcpyDeviceToHost, stream_), "couple download");
  cuda_check(cudaStreamSynchronize(stream_), "couple sync");
  for (size_t k = 0; k < np; ++k)
    for (int a = 0; a < 3; ++a) force[3 * k + a] = h[10 * k + 7 + a];
}

// world.rs:555-678 (kernels and semantics in couple.cu).  The velocity
// sampler the reference installs into the field at this point is the field's
// own business: it captures the particles' positions and velocities, which
// get_field returns.
void FluidWorld::couple_heat(const uint64_t* dims3, const double* origin3, double cell, const double* temp,
                             double* src, double dt, double t_ref, double beta, double heat_gain) {
  if (n_ == 0) return;  // world.rs:563-565
  if (!dims3 || !origin3 || !temp) throw std::invalid_argument("couple_heat: null array");
  const bool deposit = heat_gain > 0.0;
  if (deposit && !src) throw std::invalid_argument("couple_heat: null source array");
  if (!scenes_.empty()) throw std::invalid_argument("couple_heat: not available for batched scenes");
  if (tape_.on) throw std::invalid_argument("couple_heat: the adjoint tape does not record coupling");
  uint64_t cells = 1;
  for (int a = 0; a < 3; ++a) {
    if (dims3[a] == 0 || dims3[a] >= ((uint64_t)1 << 31)) throw std::invalid_argument("couple_heat: bad grid dims");
    cells *= dims3[a];
    if (cells >= ((uint64_t)1 << 31)) throw std::invalid_argument("couple_heat: more than 2^31 grid cells");
  }
  if (!b_.has_ba) {
    for (int q = 0; q < 2; ++q)
      for (int k = 0; k < 3; ++k) dgrow(b_.pc[q].ba[k], 0, (size_t)b_.capacity, stream_);
    for (int k = 0; k < 3; ++k)
      cuda_check(cudaMemsetAsync(b_.pc[b_.cur].ba[k], 0, n_ * sizeof(double), stream_), "memset");
    b_.has_ba = true;
    ++alloc_gen_;
  }
  ensure_cells();
  const StepConsts c = make_consts(dt);
  const size_t need = couple_heat_scratch_bytes((int)n_, cells);
  if (heat_cap_ < need) {
    dalloc(d_heat_, need);
    heat_cap_ = need;
  }
  const size_t gbytes = cells * sizeof(double);
  cuda_check(cudaMemcpyAsync(d_heat_, temp, gbytes, cudaMemcpyHostToDevice, stream_), "couple_heat upload");
  if (deposit)
    cuda_check(cudaMemcpyAsync(d_heat_ + gbytes, src, gbytes, cudaMemcpyHostToDevice, stream_), "couple_heat upload");
  HeatGrid g;
  g.nx = dims3[0];
  g.ny = dims3[1];
  g.nz = dims3[2];
  for (int a = 0; a < 3; ++a) g.origin[a] = origin3[a];
  g.cell = cell;
  g.t_ref = t_ref;
  g.beta = beta;
  g.heat_gain = heat_gain;
  launch_couple_heat(c, b_, g, d_heat_, stream_);
  cuda_check(cudaGetLastError(), "couple_heat launch");
  if (deposit)
    cuda_check(cudaMemcpyAsync(src, d_heat_ + gbytes, gbytes, cudaMemcpyDeviceToHost, stream_), "couple_heat download");
  cuda_check(cudaStreamSynchronize(stream_), "couple_heat sync");
}

// world.rs:414-503 (kernels and semantics in couple.cu).
void FluidWorld::couple_bodies(PhyCoupleBody* bodies, uint32_t nb, const double* data, uint64_t n_data,
                               const uint32_t* faces, uint64_t n_faces, double dt) {
  if (n_ == 0 || nb == 0) return;  // world.rs:415-417
  if (!bodies) throw std::invalid_argument("couple_bodies: null bodies");
  if (!scenes_.empty()) throw std::invalid_argument("couple_bodies: not available for batched scenes");
  if (tape_.on) throw std::invalid_argument("couple_bodies: the adjoint tape does not record coupling");
  if (nb > (1u << 20)) throw std::invalid_argument("couple_bodies: more than 2^20 bodies");
  // A leaf shape's data ranges (convex vertices and faces, heightfield heights).
  auto check_leaf = [&](int shape, uint64_t data_first, uint64_t data_count, uint64_t face_first,
                        uint64_t face_count) {
    if (shape < PHY_SHAPE_SPHERE || shape > PHY_SHAPE_HEIGHTFIELD)
      throw std::invalid_argument("couple_bodies: unsupported shape (compound shapes cannot nest)");
    if (shape == PHY_SHAPE_CONVEX) {
      if (data_count == 0 || !data || data_first + 3ull * data_count > n_data)
        throw std::invalid_argument("couple_bodies: convex vertices out of range");
      if ((face_count && !faces) || 3ull * (face_first + face_count) > n_faces)
        throw std::invalid_argument("couple_bodies: convex faces out of range");
      for (uint64_t f = 3ull * face_first; f < 3ull * (face_first + face_count); ++f)
        if (faces[f] >= data_count) throw std::invalid_argument("couple_bodies: face index out of range");
    } else if (shape == PHY_SHAPE_HEIGHTFIELD) {
      if ((data_count && !data) || data_first + data_count > n_data)
        throw std::invalid_argument("couple_bodies: heights out of range");
    }
  };
  for (uint32_t k = 0; k < nb; ++k) {
    const PhyCoupleBody& b = bodies[k];
    if (b.shape != PHY_SHAPE_COMPOUND) {
      check_leaf(b.shape, b.data_first, b.data_count, b.face_first, b.face_count);
      continue;
    }
    // Shape::Compound: at least one sub shape (support_local reads the
    // first, shape.rs:240), each a 16-double record of a leaf shape.
    if (b.data_count == 0 || !data || (uint64_t)b.data_first + 16ull * b.data_count > n_data)
      throw std::invalid_argument("couple_bodies: compound sub shapes out of range");
    for (uint32_t q = 0; q < b.data_count; ++q) {
      const double* r = data + b.data_first + 16ull * q;
      for (int f = 11; f < 15; ++f)
        if (!(r[f] >= 0.0 && r[f] < 4294967296.0 && r[f] == std::floor(r[f])))
          throw std::invalid_argument("couple_bodies: compound sub shape with an invalid data range");
      if (!(r[0] >= 0.0 && r[0] <= 4.0 && r[0] == std::floor(r[0])))
        throw std::invalid_argument("couple_bodies: unsupported shape (compound shapes cannot nest)");
      check_leaf((int)r[0], (uint64_t)r[11], (uint64_t)r[12], (uint64_t)r[13], (uint64_t)r[14]);
    }
  }
  ensure_cells();
  const StepConsts c = make_consts(dt);
  const size_t need = couple_bodies_scratch_bytes((int)n_, (int)nb, n_data, n_faces);
  if (bodies_cap_ < need) {
    dalloc(d_bodies_, need);
    bodies_cap_ = need;
  }
  CoupleBodiesLaunch l;
  l.scratch = d_bodies_;
  l.bodies = bodies;
  l.nb = (int)nb;
  l.data = data;
  l.n_data = data ? n_data : 0;
  l.faces = faces;
  l.n_faces = faces ? n_faces : 0;
  l.particle_vol = params.mass / params.rest_density;
  if (launch_couple_bodies(c, b_, l, stream_) != 0) {
    const cudaError_t e = cudaGetLastError();
    cuda_check(e == cudaSuccess ? cudaErrorUnknown : e, "couple_bodies");
  }
}

// ---- FluidSubsystem / World ------------------------------------------------

int FluidSubsystem::validate() {
  if (world->is_empty()) return 0;
  uint32_t f = world->last_step_flags();
  if (f & kFlagNonFinite) return 2;
  if (f & kFlagOutOfBox) return 5;
  return 0;
}

void World::step(double dt) {
  for (auto& s : subs) s->world->step(dt);
  // Coupling stage (subsystem.rs:92-143) needs a HeatField or a
  // RigidSubsystem; worlds of this library hold fluid subsystems only, so it
  // has nothing to couple.
  t += dt;
}

int World::step_checked(double dt) {
  step(dt);
  for (auto& s : subs) {
    int rc = s->validate();
    if (rc) return rc;
  }
  return 0;
}

size_t World::fluid_count() const {
  size_t n = 0;
  for (auto& s : subs) n += s->world->len();
  return n;
}

}  // namespace phy

namespace phy {

// ---- Adjoint ---------------------------------------------------------------------

void FluidWorld::save_checkpoint() {
  const size_t k = tape_.nckpt;
  if (k >= tape_.ckpt.size()) {
    tape_.ckpt.push_back(nullptr);
    dalloc(tape_.ckpt.back(), 6 * n_);
  }
  double* ck = tape_.ckpt[k];
  const ParticleConsts& pc = b_.pc[b_.cur];
  k_get_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>((int)n_, pc.id, b_.pv1[0], b_.pv1[1], b_.pv1[2], ck);
  k_get_vec_by_id<<<grid_for(n_), kThreads, 0, stream_>>>((int)n_, pc.id, b_.pv1[3], b_.pv1[4], b_.pv1[5],
                                                           ck + 3 * n_);
  cuda_check(cudaGetLastError(), "checkpoint");
  ++tape_.nckpt;
}

void FluidWorld::tape_clear() {
  for (auto& p : tape_.ckpt) dfree(p);
  tape_.ckpt.clear();
  tape_.nckpt = 0;
  tape_.dts.clear();
  tape_.on = false;
  tape_.n = 0;
  dfree(adj_work_);
  dfree(comp_rec_);
  comp_rec_cap_ = 0;
  for (auto& p : adj_slot_f_) dfree(p);
  for (auto& p : adj_slot_u_) dfree(p);
  adj_slot_f_.clear();
  adj_slot_u_.clear();
  adj_slot_ucount_.clear();
  release_snapshot();
}

void FluidWorld::tape_begin(int every) {
  if (prec_ == Precision::F32Comp && comp_tile_ == 0)
    throw std::invalid_argument("tape_begin: the compensated form's adjoint needs the tiled passes");
  if (!scenes_.empty()) throw std::invalid_argument("tape_begin: batched scenes are not recorded");
  if (b_.has_ba) throw std::invalid_argument("tape_begin: body accelerations are not recorded");
  if (every < 1) throw std::invalid_argument("tape_begin: checkpoint interval must be >= 1");
  if (n_ == 0) throw std::invalid_argument("tape_begin: empty world");
  // Checkpoint and sweep buffers are kept for the next tape of the same size.
  if (tape_.n != n_) tape_clear();
  tape_.n = n_;
  tape_.nckpt = 0;
  tape_.dts.clear();
  tape_.every = every;
  tape_.params = params.to_c();
  save_checkpoint();
  tape_.on = true;
}

namespace {

// Device arrays of one recorded step (sorted order) plus its launch constants.
struct TapeSlot {
  double* f = nullptr;       // 22 arrays of n doubles
  uint32_t* u = nullptr;     // mat, id, nbr_count (n each), nbr (96 n), cell_start
  StepConsts c;
  AdjTape view(size_t n) const {
    AdjTape t;
    double* q = f;
    auto take = [&]() {
      double* r = q;
      q += n;
      return r;
    };
    for (int k = 0; k < 3; ++k) t.x[k] = take();
    for (int k = 0; k < 3; ++k) t.v[k] = take();
    t.mass = take();
    t.rho = take();
    t.p = take();
    t.pr2 = take();
    t.mr = take();
    for (int k = 0; k < 3; ++k) t.acc[k] = take();
    for (int k = 0; k < 3; ++k) t.xsph[k] = take();
    t.mu = take();
    for (int k = 0; k < 3; ++k) t.fv[k] = take();
    t.shear = take();
    t.mat = u;
    t.id = u + n;
    t.nbr_count = u + 2 * n;
    t.nbr = u + 3 * n;
    t.cell_start = u + (3 + (size_t)kMaxNeighbors) * n;
    return t;
  }
};

}  // namespace

void FluidWorld::step_backward(const double* gx, const double* gv, double* gx0, double* gv0, double* gparams) {
  const size_t n = n_;
  const int T = (int)tape_.dts.size();
  if (!tape_.on) throw std::invalid_argument("step_backward: no adjoint tape (call tape_begin before stepping)");
  if (n == 0) return;
  cudaStream_t s = stream_;
  // Work arrays: gx_ins, gv_ins, gx, gv, P, Q, Y (3 each), sig, rbar,
  // rbar_tot, cc, kk, the tape's fv and shear outputs (4): 30 arrays of n,
  // then the two parameter accumulators.
  constexpr size_t kWorkArrays = 30;
  if (!adj_work_) dalloc(adj_work_, kWorkArrays * n + 2);
  double* work = adj_work_;
  AdjWork w;
  {
    double* q = work;
    size_t taken = 0;
    auto take = [&]() {
      if (++taken > kWorkArrays) throw std::logic_error("step_backward: work partition exceeds its allocation");
      double* r = q;
      q += n;
      return r;
    };
    for (int k = 0; k < 3; ++k) w.gx_ins[k] = take();
    for (int k = 0; k < 3; ++k) w.gv_ins[k] = take();
    for (int k = 0; k < 3; ++k) w.gx[k] = take();
    for (int k = 0; k < 3; ++k) w.gv[k] = take();
    for (int k = 0; k < 3; ++k) w.P[k] = take();
    for (int k = 0; k < 3; ++k) w.Q[k] = take();
    for (int k = 0; k < 3; ++k) w.Y[k] = take();
    w.sig = take();
    w.rbar = take();
    w.rbar_tot = take();
    w.cc = take();
    w.kk = take();
    for (int k = 0; k < 3; ++k) b_.tape_fv[k] = take();
    b_.tape_shear = take();
    w.param_acc = q;
  }
  const int nslots = std::min(tape_.every, std::max(T, 1));
  std::vector<TapeSlot> slots(nslots);
  if ((int)adj_slot_f_.size() < nslots) {
    adj_slot_f_.resize(nslots, nullptr);
    adj_slot_u_.resize(nslots, nullptr);
    adj_slot_ucount_.resize(nslots, 0);
  }
  // A compensated world is differentiated along its own trajectory: each
  // re-run step first takes an f64 plain recording step from the same state
  // (the records of the exact step map at that state), then returns to the
  // state and takes the compensated step to the next one, whose density,
  // pressure, viscosity, acceleration and XSPH outputs replace the recorded
  // f64 values.
  const Precision form = prec_;
  const bool comp = form == Precision::F32Comp;
  uint32_t* slot_of = nullptr;  // compensated: insertion index -> recorded slot of the step being re-run
  if (comp) {
    if (comp_rec_cap_ < n) {
      dalloc(comp_rec_, n);
      comp_rec_cap_ = n;
    }
    slot_of = comp_rec_;
  }
  auto cleanup = [&]() {
    for (int k = 0; k < 3; ++k) b_.tape_fv[k] = nullptr;
    b_.tape_shear = nullptr;
    recomputing_ = false;
    prec_ = form;
  };
  try {
    snapshot(false);  // the world returns to x_T, v_T afterwards
    // Seeds (insertion order): dL/dx_T, dL/dv_T.
    cuda_check(cudaMemsetAsync(work, 0, (6 * n + 0) * sizeof(double), s), "seed clear");
    cuda_check(cudaMemsetAsync(w.param_acc, 0, 2 * sizeof(double), s), "param clear");
    if (gx) {
      cuda_check(cudaMemcpyAsync(b_.stage, gx, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s), "seed upload");
      launch_deinterleave3(b_.stage, w.gx_ins[0], w.gx_ins[1], w.gx_ins[2], (int)n, s);
    }
    if (gv) {
      cuda_check(cudaMemcpyAsync(b_.stage + 3 * n, gv, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s),
                 "seed upload");
      launch_deinterleave3(b_.stage + 3 * n, w.gv_ins[0], w.gv_ins[1], w.gv_ins[2], (int)n, s);
    }
    cuda_check(cudaStreamSynchronize(s), "seed sync");
    recomputing_ = true;
    const int every = tape_.every;
    const int nseg = (T + every - 1) / every;
    for (int seg = nseg - 1; seg >= 0; --seg) {
      const int t0 = seg * every, t1 = std::min(T, t0 + every);
      // Restore checkpoint `seg` and re-run its steps, recording each.
      const ParticleConsts& pc = b_.pc[b_.cur];
      const double* ck = tape_.ckpt[seg];
      k_set_vec_by_id<<<grid_for(n), kThreads, 0, s>>>((int)n, pc.id, ck, b_.pv1[0], b_.pv1[1], b_.pv1[2]);
      k_set_vec_by_id<<<grid_for(n), kThreads, 0, s>>>((int)n, pc.id, ck + 3 * n, b_.pv1[3], b_.pv1[4],
                                                       b_.pv1[5]);
      for (int t = t0; t < t1; ++t) {
        TapeSlot& sl = slots[t - t0];
        const int si = t - t0;
        if (comp) {
          // The f64 recording step from state t first.
          prec_ = Precision::F64Plain;
          ensure_mode_buffers();  // f64 neighbour lists, kept for later sweeps
        }
        const StepConsts c = step_impl(tape_.dts[t]);
        const size_t ncs = (size_t)c.ncells + 2;
        const size_t ucount = (3 + (size_t)kMaxNeighbors) * n + ncs;
        if (!adj_slot_f_[si]) dalloc(adj_slot_f_[si], 22 * n);
        if (adj_slot_ucount_[si] < ucount) {
          dalloc(adj_slot_u_[si], ucount);
          adj_slot_ucount_[si] = ucount;
        }
        sl.f = adj_slot_f_[si];
        sl.u = adj_slot_u_[si];
        sl.c = c;
        const AdjTape v = sl.view(n);
        const ParticleConsts& q = b_.pc[b_.cur];
        TapeCopy tc;
        int k = 0;
        auto add = [&](const double* dst, const double* src) {
          tc.dst[k] = const_cast<double*>(dst);
          tc.src[k] = src;
          ++k;
        };
        for (int a = 0; a < 3; ++a) add(v.x[a], b_.pv0[a]);
        for (int a = 0; a < 3; ++a) add(v.v[a], b_.pv0[3 + a]);
        add(v.mass, q.mass);
        add(v.rho, b_.rho);
        add(v.p, b_.p);
        add(v.pr2, b_.pr2);
        add(v.mr, b_.mr);
        for (int a = 0; a < 3; ++a) add(v.acc[a], b_.acc[a]);
        for (int a = 0; a < 3; ++a) add(v.xsph[a], b_.xsph[a]);
        add(v.mu, b_.mu);
        for (int a = 0; a < 3; ++a) add(v.fv[a], b_.tape_fv[a]);
        add(v.shear, b_.tape_shear);
        if (k != 22) throw std::logic_error("step_backward: tape layout");
        tc.usrc[0] = q.mat;
        tc.udst[0] = const_cast<uint32_t*>(v.mat);
        tc.usrc[1] = q.id;
        tc.udst[1] = const_cast<uint32_t*>(v.id);
        tc.usrc[2] = b_.nbr_count;
        tc.udst[2] = const_cast<uint32_t*>(v.nbr_count);
        tc.nbr = b_.nbr;
        tc.nbr_dst = const_cast<uint32_t*>(v.nbr);
        tc.nbr_stride = b_.capacity;
        tc.slot_of = slot_of;
        k_tape_copy<<<grid_for(n), kThreads, 0, s>>>((int)n, tc);
        cuda_check(cudaMemcpyAsync(const_cast<uint32_t*>(v.cell_start), b_.cell_start, ncs * 4,
                                   cudaMemcpyDeviceToDevice, s),
                   "tape copy");
        if (comp) {
          // Back to state t for the compensated step to state t+1: the
          // recording step left state t, sorted, in pv0 with the constants of
          // that order current, and a step's result does not depend on the
          // order of its input.  Its outputs replace the recorded f64 ones
          // (matched through the particles' insertion indices).
          ArrayCopy back{};
          for (int k = 0; k < 6; ++k) {
            back.src[k] = reinterpret_cast<const unsigned char*>(b_.pv0[k]);
            back.dst[k] = reinterpret_cast<unsigned char*>(b_.pv1[k]);
            back.bytes[k] = n * sizeof(double);
          }
          const size_t blocks = std::min<size_t>((n * sizeof(double) / 16 + kThreads - 1) / kThreads + 1, 1184);
          k_copy_arrays<<<dim3((unsigned)blocks, 6), kThreads, 0, s>>>(back);
          prec_ = Precision::F32Comp;
          step_impl(tape_.dts[t]);
          const ParticleConsts& cq = b_.pc[b_.cur];
          CompOverride co;
          co.id = cq.id;
          co.mass = cq.mass;
          co.rho = b_.rho;
          co.p = b_.p;
          co.mu = b_.mu;
          co.slot_of = slot_of;
          co.t_rho = const_cast<double*>(v.rho);
          co.t_p = const_cast<double*>(v.p);
          co.t_pr2 = const_cast<double*>(v.pr2);
          co.t_mr = const_cast<double*>(v.mr);
          co.t_mu = const_cast<double*>(v.mu);
          for (int a = 0; a < 3; ++a) {
            co.acc[a] = b_.acc[a];
            co.xsph[a] = b_.xsph[a];
            co.t_acc[a] = const_cast<double*>(v.acc[a]);
            co.t_xsph[a] = const_cast<double*>(v.xsph[a]);
          }
          k_comp_override<<<grid_for(n), kThreads, 0, s>>>((int)n, co);
          cuda_check(cudaGetLastError(), "tape override");
        }
      }
      for (int t = t1 - 1; t >= t0; --t) launch_adjoint_step(slots[t - t0].c, slots[t - t0].view(n), w, s);
      cuda_check(cudaGetLastError(), "adjoint step");
    }
    recomputing_ = false;
    std::vector<double> host(6 * n);
    launch_interleave3(w.gx_ins[0], w.gx_ins[1], w.gx_ins[2], b_.stage, (int)n, s);
    launch_interleave3(w.gv_ins[0], w.gv_ins[1], w.gv_ins[2], b_.stage + 3 * n, (int)n, s);
    double pa[2] = {0.0, 0.0};
    cuda_check(cudaMemcpyAsync(host.data(), b_.stage, 6 * n * sizeof(double), cudaMemcpyDeviceToHost, s),
               "gradient read");
    cuda_check(cudaMemcpyAsync(pa, w.param_acc, sizeof(pa), cudaMemcpyDeviceToHost, s), "gradient read");
    cuda_check(cudaStreamSynchronize(s), "gradient sync");
    if (gx0) std::memcpy(gx0, host.data(), 3 * n * sizeof(double));
    if (gv0) std::memcpy(gv0, host.data() + 3 * n, 3 * n * sizeof(double));
    if (gparams) {
      gparams[0] = pa[0];
      gparams[1] = pa[1];
    }
    snapshot(true);
  } catch (...) {
    cleanup();
    if (snap_count_[0]) snapshot(true);
    throw;
  }
  cleanup();
}

void pin_host(void* ptr, size_t bytes) {
  cuda_check(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault), "cudaHostRegister");
}

void unpin_host(void* ptr) { cuda_check(cudaHostUnregister(ptr), "cudaHostUnregister"); }

}  // namespace phy
