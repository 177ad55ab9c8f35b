// Host-side mirror of the reference's fluid API (crates/phy-fluid):
//   SphParams<T>      src/sph/params.rs:12-86
//   FluidWorld<T>     src/sph/world.rs:21-197
//   FluidSubsystem<T> src/subsystem.rs:26-164
//   World<T>          crates/phy-core/src/world.rs:78-294 (fluid subsystems only)
//
// The device holds the particle state; nothing is mirrored on the host.  Host
// reads and writes of a particle field go through permutation kernels so that
// callers always see insertion order, as with the reference's `particles` Vec.
#pragma once

#include <array>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/phy_fluid.h"
#include "sph_buffers.h"

namespace phy {

struct Vec3 {
  double x, y, z;
};

struct SphParams {
  double rest_density, stiffness, viscosity;
  std::vector<double> visc_k, visc_n;
  double shear_min, mass, h;
  Vec3 gravity, bounds_min, bounds_max;
  double boundary_damp, xsph_eps;

  static SphParams defaults();  // params.rs:55-85
  PhySphParams to_c() const;
  static SphParams from_c(const PhySphParams& c);
};

enum class Precision : int { F64Plain = 0, F32Comp = 1 };

class CudaError : public std::runtime_error {
 public:
  using std::runtime_error::runtime_error;
};

void cuda_check(cudaError_t e, const char* what);

// One configuration of the launch knobs and its measured step time.
struct TuneTrial {
  LaunchTuning tuning;
  int comp_tile;       // cells per tile edge of the trial (0: not a tiled world)
  double ms_per_step;  // mean over the sampled states the trial ran on
  int samples;         // sampled states it ran on
};

class FluidWorld {
 public:
  FluidWorld(const SphParams& params, Precision prec);
  ~FluidWorld();
  FluidWorld(const FluidWorld&) = delete;
  FluidWorld& operator=(const FluidWorld&) = delete;

  // Public, live parameters (the reference's `pub params`).  The smoothing
  // length of the kernel coefficients and of the grid cell was captured at
  // construction (world.rs:94-102).
  SphParams params;

  size_t len() const { return n_; }
  bool is_empty() const { return n_ == 0; }
  Precision precision() const { return prec_; }
  double captured_h() const { return h0_; }

  double lattice_mass(double s) const;                                  // world.rs:148-169
  void fill_box(Vec3 mn, Vec3 mx, double spacing, double margin);       // world.rs:124-144
  void add_particles(size_t n, const double* pos, const double* vel, const double* mass,
                     const uint32_t* material);                         // world.rs:171-174
  void step(double dt);                                                 // world.rs:183-192
  // n steps; with a graph chunk set, runs of `chunk` steps are captured once
  // into a CUDA graph and replayed (re-captured when a parameter, dt, the
  // particle count or a buffer changes).
  void step_n(double dt, int n);
  void set_graph_chunk(int steps) { graph_chunk_ = steps < 0 ? 0 : steps; }
  int graph_chunk() const { return graph_chunk_; }

  // Batched scenes: partitions the particles (insertion order) into
  // consecutive scenes of counts[s] particles, each with its own wall bounds
  // and its own grid box; a step then advances every scene through one sort
  // and one persistent launch per pass.  The scenes never interact; shared
  // parameters are the world's.  Tiled compensated form only; the particle
  // set is then fixed (add_particles throws until clear_scenes()).
  void set_scenes(const std::vector<uint64_t>& counts, const std::vector<Vec3>& lo, const std::vector<Vec3>& hi);
  void clear_scenes();
  int scene_count() const { return (int)scenes_.size(); }

  // Launch knobs of the tiled passes and the sort (results do not depend on
  // them) and the project's autotuner over them: every candidate runs
  // `steps` steps from the same saved state (restored afterwards), the
  // fastest is kept.  Returns the trials in order.
  void set_launch_tuning(const LaunchTuning& t) { tuning_ = t; }
  LaunchTuning launch_tuning() const { return tuning_; }
  std::vector<TuneTrial> autotune(double dt, int steps, int horizon = 0);

  // Adjoint of the f64 plain step (world.rs:183-397).  tape_begin makes the
  // current state checkpoint 0 and records every following step's dt, with a
  // state checkpoint every `every` steps; parameters must not change and
  // body accelerations must not be set while recording.  step_backward runs
  // the reverse sweep over the recorded steps, re-running each segment
  // forward from its checkpoint: given dL/dx_T and dL/dv_T (insertion order,
  // xyz interleaved; null = zero) it returns dL/dx_0, dL/dv_0 and
  // {dL/d stiffness, dL/d visc_k[0]} (outputs may be null) and leaves the
  // world in its state x_T, v_T.  The tape is kept for further sweeps.
  void tape_begin(int every);
  void tape_clear();
  int tape_steps() const { return (int)tape_.dts.size(); }
  void step_backward(const double* gx, const double* gv, double* gx0, double* gv0, double* gparams);

  // Insertion-order field access (particle.rs:17-46).
  static int components(int field);
  void get_field(int field, double* out);
  // Device-memory forms (no host copy): replace the whole particle set from
  // device arrays (pos/vel 3m interleaved, mass m, material m u32; vel and
  // material may be null), and read a field in insertion order into a
  // device buffer.
  void set_particles_device(size_t m, const double* pos, const double* vel, const double* mass,
                            const uint32_t* material);
  void get_field_device(int field, double* out);
  // Position or velocity as f32 (an exact `as f32` cast of each f64 value,
  // made on the device so half the bytes cross to the host): the first
  // `count` particles in insertion order, xyz interleaved.
  // The first `count` particles' xyz (pos or vel) in insertion order, copied
  // straight into `out` (no host bounce).
  void get_vec_f64(int field, double* out, size_t count);
  void get_vec_f32(int field, float* out, size_t count);
  void set_field(int field, const double* in);

  void set_stream(cudaStream_t s);
  cudaStream_t stream() const { return stream_; }
  void synchronize();
  // Error bits of the last step (synchronises).
  uint32_t last_step_flags();
  // Candidates / pairs of the last step (synchronises); counting is enabled
  // by set_counting(true) and costs one atomic per warp.
  void set_counting(bool on) { counting_ = on; }
  void last_step_counters(uint64_t* out2);
  // Dense-cell mask buffer: entries allocated, entries the last step's tasks
  // reserved, 1 when the last step found a task's masks outside the buffer
  // (waits for the stream).
  void dense_mask_info(uint64_t* out3);
  int grid_cells() const { return ncells_; }

  // FluidWorld::couple_points (world.rs:691-752) on the device, bit-exact:
  // np point masses (pos, vel: xyz interleaved; mass) coupled one after
  // another; force (xyz interleaved) is written for the points inside the
  // bounds and the fluid velocities take the reactions.  Not available for
  // batched scenes or while the adjoint tape records.
  void couple_points(size_t np, const double* pos, const double* vel, const double* mass, double* force,
                     double dt, double drag, double soft_density);

  // FluidWorld::couple_heat (world.rs:555-678) on the device, bit-exact:
  // against a heat grid of dims3 cells (x fastest), origin3 and cell size
  // `cell` with temperatures `temp`: body_acc += -g beta (T - t_ref) for the
  // particles inside the bounds, and with heat_gain > 0 the sources `src`
  // (dims product doubles, updated in place) take heat_gain |v| dt per
  // particle, added in insertion order.  Not available for batched scenes or
  // while the adjoint tape records.
  void couple_heat(const uint64_t* dims3, const double* origin3, double cell, const double* temp, double* src,
                   double dt, double t_ref, double beta, double heat_gain);

  // FluidWorld::couple_bodies (world.rs:414-503) on the device, bit-exact:
  // `bodies` (velocities updated in place) with their vertex / height data
  // and face indices as described for PhyCoupleBody.  Not available for
  // batched scenes or while the adjoint tape records.
  void couple_bodies(PhyCoupleBody* bodies, uint32_t nb, const double* data, uint64_t n_data, const uint32_t* faces,
                     uint64_t n_faces, double dt);

  // Total momentum and kinetic energy (subsystem.rs:149-163), f64, insertion order.
  void diagnostics(double* out4);

  // Per-phase device timing with CUDA events on the world's stream: while
  // enabled, every step records events around the sort, the per-particle
  // preparation, the density pass and the force pass without waiting for
  // them; phase_times waits for the last recorded step and accumulates the
  // durations (ms).  out = {sort, prep, density, force, steps}.
  void set_timing(bool on);
  void phase_times(double* out5, bool reset);

  // Kernel configuration of the compensated form: tile edge in cells
  // (0 = x-major runs, 4 = staged 4x4x4 tiles, the default).
  void set_comp_tile(int t);
  int comp_tile() const { return comp_tile_; }
  // Staging capacity (particles per tile halo) below the kernels' maximum;
  // smaller values route more tiles through the global-memory path.
  void set_halo_cap(int v) { halo_cap_ = v < 0 ? 0 : v; }
  int halo_cap() const { return halo_cap_; }
  void set_dense_mean(int v) { dense_mean_ = v < 1 ? 1 : v; }
  int dense_mean() const { return dense_mean_; }

  // Device state access for in-library consumers (sorted order).
  DevBuffers& buffers() { return b_; }
  StepConsts make_consts(double dt) const;

 private:
  void ensure_capacity(size_t n);
  void ensure_mode_buffers();
  void ensure_masks();
  void ensure_cells();
  void grow_box_with_bounds();
  void grow_box_with_positions(size_t n, const double* pos3);
  void merge_box(const long long* mn, const long long* mx, bool any_nonfinite);
  void grow_box_with_device_positions(size_t n, const double* d_pos3);
  void grow_scene_boxes(const double* d_pos3);
  void free_all();
  StepConsts prepare_step(double dt);
  StepConsts step_impl(double dt);
  void save_checkpoint();
  void enqueue_step(const StepConsts& c, const PassEvents& pe, const cudaEvent_t* ev);
  void run_graph(double dt, int k);
  void drop_graphs();
  void stage_field(int field, double* st);
  // Saves (or restores) the per-particle state in slot `slot` with one copy
  // launch on the world's stream; `sync` waits for it.
  void snapshot(bool restore, int slot = 0, bool sync = true);
  void release_snapshot();
  // Mean ms per step of `steps` steps from each saved slot 0..nslots-1 under
  // tuning t (warm-up and graph capture first).
  double time_tuning(const LaunchTuning& t, int comp_tile, double dt, int steps, int nslots, cudaEvent_t e0,
                     cudaEvent_t e1);

  Precision prec_;
  double h0_;
  size_t n_ = 0;
  DevBuffers b_;
  cudaStream_t stream_ = nullptr;
  cudaStream_t own_stream_ = nullptr;
  // Grid box: inclusive key range of occupied-or-possible cells (unpadded).
  bool box_valid_ = false;
  long long kmin_[3] = {0, 0, 0}, kmax_[3] = {0, 0, 0};
  int ncells_ = 0;
  long long bx0_[3] = {0, 0, 0};
  int nc_[3] = {0, 0, 0};
  bool counting_ = false;
  int comp_tile_ = 4;
  int halo_cap_ = 1 << 30;
  int dense_mean_ = (int)kDenseMean;
  int tile_ = 0;  // linearisation of the current box (0 = x-major)
  bool timing_ = false;
  // One set of 5 events per timed step, recycled after phase_times reads them.
  std::vector<std::array<cudaEvent_t, 5>> ev_pool_;
  size_t ev_used_ = 0;
  void collect_phase_times();
  double phase_ms_[4] = {0, 0, 0, 0};
  double timed_steps_ = 0;
  long long* d_bbox_ = nullptr;  // 7 values: min xyz, max xyz, non-finite flag
  // Point records of couple_points (10 doubles each) plus one word of flags.
  double* d_couple_ = nullptr;
  CouplePointsScratch couple_scratch_;
  size_t couple_cap_ = 0;
  // Scratch arena of couple_heat (grid, sources, sort keys).
  unsigned char* d_heat_ = nullptr;
  size_t heat_cap_ = 0;
  // Scratch arena of couple_bodies.
  unsigned char* d_bodies_ = nullptr;
  size_t bodies_cap_ = 0;

  // Batched scenes.
  struct Scene {
    uint64_t first, count;
    Vec3 lo, hi;
    long long kmin[3], kmax[3];
  };
  std::vector<Scene> scenes_;
  std::vector<SceneBox> host_boxes_;  // last uploaded box table
  int boxes_capacity_ = 0;
  uint32_t* d_pbase_ = nullptr;
  long long* d_scene_bbox_ = nullptr;
  LaunchTuning tuning_;
  // CUDA graphs of step chunks, keyed by everything a captured launch bakes in.
  struct GraphEntry {
    std::vector<unsigned char> key;
    cudaGraphExec_t exec;
  };
  std::vector<GraphEntry> graphs_;
  int graph_chunk_ = 0;
  unsigned long long alloc_gen_ = 0;  // bumped on every (re)allocation
  // Adjoint tape: per-step dt and device checkpoints (6n doubles each: pos
  // and vel, xyz interleaved, insertion order) every `every` steps.
  struct Tape {
    bool on = false;
    int every = 1;
    size_t n = 0;        // particle count the buffers are sized for
    std::vector<double> dts;
    std::vector<double*> ckpt;  // pool; the first nckpt are this tape's
    size_t nckpt = 0;
    PhySphParams params;
  } tape_;
  // Reverse-sweep buffers kept between sweeps (freed by tape_clear).
  double* adj_work_ = nullptr;
  uint32_t* comp_rec_ = nullptr;  // compensated adjoint: insertion index -> recorded slot
  size_t comp_rec_cap_ = 0;
  std::vector<double*> adj_slot_f_;
  std::vector<uint32_t*> adj_slot_u_;
  std::vector<size_t> adj_slot_ucount_;
  bool recomputing_ = false;
  // Saved states (autotuner, reverse sweep): per slot one arena reused while
  // large enough.
  unsigned long long mask_tried_ = 0;  // the last mask demand the buffer was grown for
  static constexpr int kSnapSlots = 3;
  double* snap_arena_[kSnapSlots] = {};
  size_t snap_bytes_[kSnapSlots] = {};
  size_t snap_count_[kSnapSlots] = {};
  int snap_cur_[kSnapSlots] = {};
};

// FluidSubsystem<T> (subsystem.rs:26-55): the world plus coupling coefficients.
struct FluidSubsystem {
  std::unique_ptr<FluidWorld> world;
  double thermal_expansion = 0.0, heat_gain = 0.0, t_ref = 0.0, drag = 1.0, friction = 0.1;
  explicit FluidSubsystem(std::unique_ptr<FluidWorld> w) : world(std::move(w)) {}
  // Subsystem::validate (subsystem.rs:74-90): 0 ok, 2 non-finite, 5 grid box.
  int validate();
};

// World<T> restricted to fluid subsystems (phy-core/src/world.rs:224-293).
class World {
 public:
  std::vector<std::unique_ptr<FluidSubsystem>> subs;
  double t = 0.0;
  void step(double dt);            // world.rs:265-267
  int step_checked(double dt);     // world.rs:282-293
  size_t fluid_count() const;
};

// cudaHostRegister / cudaHostUnregister of a caller's buffer (throws on error).
void pin_host(void* ptr, size_t bytes);
void unpin_host(void* ptr);

}  // namespace phy
