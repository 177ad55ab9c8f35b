// Density and pressure without any device allocation.
//
// Some callers of this library cannot allocate device memory when they need
// a density evaluation: a game or simulation engine that reserves the whole
// device up front and hands plugins only the buffers it owns, a host process
// whose allocator policy forbids foreign cudaMalloc/cudaFree calls, or a
// latency-critical loop that must not enter the driver's allocator (which can
// synchronise the device).  phy_fluid_density_noalloc() serves them: the
// caller passes its own device buffers for the inputs and outputs, and all
// scratch memory (the cell-key bounding box, the counting sort and the sorted
// copy of the particles) lives in one file-scope __device__ array of
// kScratchBytes bytes, which every GPU that loads the library holds until the
// process exits.  The call allocates nothing and calls no allocating routine.
//
// The arithmetic is that of the f64 plain step's density pass
// (FluidWorld<f64>::compute_density_pressure, crates/phy-fluid/src/sph/
// world.rs:204-246): the same cell keys, visit order, explicit round-to-nearest
// operations, so rho and p are bit-identical to what FluidWorld::step writes.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/phy_fluid.h"
#include "sph_common.cuh"

namespace phy {

namespace {

constexpr int kMaxN = PHY_NOALLOC_MAX_PARTICLES;
constexpr int kMaxCells = PHY_NOALLOC_MAX_CELLS;
constexpr int kThreads = 256;
constexpr int kScanThreads = 1024;
constexpr double kPi = 3.14159265358979323846;

// Scratch layout (byte offsets, each 256-byte aligned).
constexpr size_t align256(size_t v) { return (v + 255) / 256 * 256; }
constexpr size_t kCellStartBytes = align256((size_t)(kMaxCells + 2) * 4);
constexpr size_t kOffCellStart = 0;
constexpr size_t kOffBbox = kOffCellStart + kCellStartBytes;               // 8 x int64
constexpr size_t kOffCellOf = kOffBbox + 256;                               // u32 per particle
constexpr size_t kOffRank = kOffCellOf + align256((size_t)kMaxN * 4);
constexpr size_t kOffTmp = kOffRank + align256((size_t)kMaxN * 4);
constexpr size_t kOffPerm = kOffTmp + align256((size_t)kMaxN * 4);
constexpr size_t kOffSorted = kOffPerm + align256((size_t)kMaxN * 4);       // x, y, z, mass (f64 SoA)
constexpr size_t kScratchBytes = kOffSorted + 4 * align256((size_t)kMaxN * 8);

// The scratch array.  In host code this name is only a stand-in for the
// symbol; the kernels receive its device address from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct Scratch {
  uint32_t* cell_start;
  long long* bbox;
  uint32_t* cell_of;
  uint32_t* rank;
  uint32_t* tmp;
  uint32_t* perm;
  double* sx;
  double* sy;
  double* sz;
  double* sm;
};

Scratch carve(unsigned char* base) {
  Scratch s;
  s.cell_start = reinterpret_cast<uint32_t*>(base + kOffCellStart);
  s.bbox = reinterpret_cast<long long*>(base + kOffBbox);
  s.cell_of = reinterpret_cast<uint32_t*>(base + kOffCellOf);
  s.rank = reinterpret_cast<uint32_t*>(base + kOffRank);
  s.tmp = reinterpret_cast<uint32_t*>(base + kOffTmp);
  s.perm = reinterpret_cast<uint32_t*>(base + kOffPerm);
  const size_t col = align256((size_t)kMaxN * 8);
  s.sx = reinterpret_cast<double*>(base + kOffSorted);
  s.sy = reinterpret_cast<double*>(base + kOffSorted + col);
  s.sz = reinterpret_cast<double*>(base + kOffSorted + 2 * col);
  s.sm = reinterpret_cast<double*>(base + kOffSorted + 3 * col);
  return s;
}

__global__ void k_na_bbox_init(long long* bbox) {
  if (threadIdx.x < 3) {
    bbox[threadIdx.x] = LLONG_MAX;
    bbox[3 + threadIdx.x] = LLONG_MIN;
  }
}

// Cell keys of every coordinate (non-finite -> 0, as Grid::key_of does).
__global__ void k_na_bbox(int n, const double* __restrict__ pos3, double inv, long long* bbox) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int a = 0; a < 3; ++a) {
    const long long k = key_axis(pos3[3 * (size_t)i + a], inv);
    atomicMin(&bbox[a], k);
    atomicMax(&bbox[3 + a], k);
  }
}

__global__ void k_na_hist(StepConsts c, const double* __restrict__ pos3, Scratch s) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.n) return;
  const long long kx = key_axis(pos3[3 * (size_t)i], c.inv_cell);
  const long long ky = key_axis(pos3[3 * (size_t)i + 1], c.inv_cell);
  const long long kz = key_axis(pos3[3 * (size_t)i + 2], c.inv_cell);
  const uint32_t cell = (uint32_t)cell_linear(c, kx, ky, kz);  // inside the box by construction
  s.cell_of[i] = cell;
  s.rank[i] = atomicAdd(&s.cell_start[cell], 1u);
}

// Exclusive scan of len counts in one block: contiguous chunks per thread,
// then a scan of the chunk sums.
__global__ void __launch_bounds__(kScanThreads) k_na_scan(uint32_t* v, int len) {
  __shared__ uint32_t sums[kScanThreads];
  const int per = (len + kScanThreads - 1) / kScanThreads;
  const int b = threadIdx.x * per, e = min(b + per, len);
  uint32_t t = 0;
  for (int k = b; k < e; ++k) t += v[k];
  sums[threadIdx.x] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (int k = 0; k < kScanThreads; ++k) {
      const uint32_t x = sums[k];
      sums[k] = run;
      run += x;
    }
  }
  __syncthreads();
  uint32_t run = sums[threadIdx.x];
  for (int k = b; k < e; ++k) {
    const uint32_t x = v[k];
    v[k] = run;
    run += x;
  }
}

__global__ void k_na_scatter(int n, Scratch s) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) s.tmp[s.cell_start[s.cell_of[i]] + s.rank[i]] = (uint32_t)i;
}

// Stable order inside a cell: rank by caller index (the reference's
// insertion order), then gather the sorted copy.
__global__ void k_na_order_gather(int n, const double* __restrict__ pos3, const double* __restrict__ mass,
                                  Scratch s) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const uint32_t i = s.tmp[q];
  const uint32_t cell = s.cell_of[i];
  const uint32_t cs = s.cell_start[cell], ce = s.cell_start[cell + 1];
  uint32_t r = 0;
  for (uint32_t k = cs; k < ce; ++k) r += s.tmp[k] < i ? 1u : 0u;
  const uint32_t slot = cs + r;
  s.perm[slot] = i;
  s.sx[slot] = pos3[3 * (size_t)i];
  s.sy[slot] = pos3[3 * (size_t)i + 1];
  s.sz[slot] = pos3[3 * (size_t)i + 2];
  s.sm[slot] = mass[i];
}

__device__ __forceinline__ double na_poly6(const StepConsts& c, double r) {
  if (r >= c.h0) return 0.0;
  const double diff = __dsub_rn(c.h0sq, __dmul_rn(r, r));
  return __dmul_rn(__dmul_rn(__dmul_rn(c.poly6_c, diff), diff), diff);
}

// compute_density_pressure (world.rs:204-246) in the reference's order.
__global__ void k_na_density(StepConsts c, Scratch s, double* __restrict__ rho_out, double* __restrict__ p_out) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= c.n) return;
  const double xi = s.sx[q], yi = s.sy[q], zi = s.sz[q];
  const long long kx = key_axis(xi, c.inv_cell), ky = key_axis(yi, c.inv_cell), kz = key_axis(zi, c.inv_cell);
  const int base = cell_linear(c, kx - 1, ky - 1, kz - 1);
  double rho = 0.0;
  for (int di = 0; di < 3; ++di)
    for (int dj = 0; dj < 3; ++dj) {
      const int c0 = base + (di * c.ncy + dj) * c.ncz;
      const uint32_t b = s.cell_start[c0], e = s.cell_start[c0 + 3];
      for (uint32_t j = b; j < e; ++j) {
        const double dx = __dsub_rn(xi, s.sx[j]), dy = __dsub_rn(yi, s.sy[j]), dz = __dsub_rn(zi, s.sz[j]);
        const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        if (r2 > c.r2_guard) continue;
        const double r = __dsqrt_rn(r2);
        if (r < c.h) rho = __dadd_rn(rho, __dmul_rn(s.sm[j], na_poly6(c, r)));
      }
    }
  const double over = __dsub_rn(rho, c.rest);
  const uint32_t i = s.perm[q];
  rho_out[i] = rho;
  p_out[i] = over > 0.0 ? __dmul_rn(c.stiff, over) : 0.0;
}

// Device address of the scratch array, looked up once per device.
std::mutex g_mutex;
unsigned char* g_ptr[64] = {};

unsigned char* scratch_for_current_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) throw std::runtime_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) throw std::runtime_error("device ordinal beyond 63");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_ptr[dev] = static_cast<unsigned char*>(p);
  }
  return g_ptr[dev];
}

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

// Records the message returned by phy_fluid_last_error() (ffi.cpp).
void set_last_error(const char* msg);

}  // namespace phy

extern "C" int32_t phy_fluid_density_noalloc(const PhySphParams* params, uint64_t n, const double* pos,
                                             const double* mass, double* rho, double* p, void* cuda_stream) {
  using namespace phy;
  try {
    if (!params || (n > 0 && (!pos || !mass || !rho || !p)))
      throw std::invalid_argument("phy_fluid_density_noalloc: null argument");
    if (n > (uint64_t)kMaxN)
      throw std::invalid_argument("phy_fluid_density_noalloc: " + std::to_string(n) + " particles exceed the " +
                                  std::to_string(kMaxN) + "-particle scratch capacity");
    if (n == 0) return 0;
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    Scratch s = carve(scratch_for_current_device());
    // Kernels::new / Grid::new from params->h (kernels.rs:22-35, grid.rs:27).
    const double h = params->h;
    const double h2 = h * h, h3 = h2 * h, h6 = h3 * h3, h9 = h6 * h3;
    StepConsts c;
    std::memset(&c, 0, sizeof(c));
    c.h0 = h;
    c.h0sq = h2;
    c.poly6_c = 315.0 / (64.0 * kPi * h9);
    c.inv_cell = 1.0 / h;
    c.h = h;
    c.r2_guard = std::nextafter(h * h, std::numeric_limits<double>::infinity());
    c.rest = params->rest_density;
    c.stiff = params->stiffness;
    c.n = (int)n;
    const int blocks = (int)((n + kThreads - 1) / kThreads);
    // Cell-key bounding box (read back to size the grid: the call waits for
    // the stream here).
    k_na_bbox_init<<<1, 32, 0, st>>>(s.bbox);
    k_na_bbox<<<blocks, kThreads, 0, st>>>((int)n, pos, c.inv_cell, s.bbox);
    check(cudaGetLastError(), "bbox kernel");
    long long bb[6];
    check(cudaMemcpyAsync(bb, s.bbox, sizeof(bb), cudaMemcpyDeviceToHost, st), "bbox readback");
    check(cudaStreamSynchronize(st), "bbox sync");
    long long cells = 1;
    int nc[3];
    for (int a = 0; a < 3; ++a) {
      // Every particle has a key (non-finite coordinates map to 0), so
      // min <= max and the span is exact in unsigned 64-bit arithmetic even
      // when the keys sit near opposite ends of the int64 range.
      const unsigned long long span = (unsigned long long)bb[3 + a] - (unsigned long long)bb[a];
      // The padding cell below the box must have an int64 key too.
      if (bb[3 + a] < bb[a] || bb[a] == LLONG_MIN || bb[3 + a] == LLONG_MAX || span > (unsigned long long)kMaxCells ||
          (cells *= (long long)span + 3) > kMaxCells)  // one empty cell of padding on each side
        throw std::invalid_argument("phy_fluid_density_noalloc: the particles span more than " +
                                    std::to_string(kMaxCells) + " grid cells (padded bounding box)");
      nc[a] = (int)span + 3;
    }
    c.bx0 = bb[0] - 1;
    c.by0 = bb[1] - 1;
    c.bz0 = bb[2] - 1;
    c.ncx = nc[0];
    c.ncy = nc[1];
    c.ncz = nc[2];
    c.ncells = (int)cells;
    // The counts must start at zero: the previous call left its cell starts.
    check(cudaMemsetAsync(s.cell_start, 0, (size_t)(c.ncells + 1) * 4, st), "clear counts");
    k_na_hist<<<blocks, kThreads, 0, st>>>(c, pos, s);
    k_na_scan<<<1, kScanThreads, 0, st>>>(s.cell_start, c.ncells + 1);
    k_na_scatter<<<blocks, kThreads, 0, st>>>((int)n, s);
    k_na_order_gather<<<blocks, kThreads, 0, st>>>((int)n, pos, mass, s);
    k_na_density<<<blocks, kThreads, 0, st>>>(c, s, rho, p);
    check(cudaGetLastError(), "density kernels");
    check(cudaStreamSynchronize(st), "density sync");
    return 0;
  } catch (const std::exception& e) {
    phy::set_last_error(e.what());
  } catch (...) {
    phy::set_last_error("unknown error");
  }
  return -1;
}
