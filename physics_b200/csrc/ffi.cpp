// extern "C" boundary of libphysph.so: the reference's phy-ffi symbols
// (crates/phy-ffi/src/lib.rs) and the phy_fluid_* additions of ABI 3.
//
// Every entry catches all C++ exceptions (the counterpart of the reference's
// catch_unwind guard, lib.rs:71-75) and maps them to its failure value, with
// the message kept for phy_fluid_last_error().
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/phy_ffi.h"
#include "../../include/phy_fluid.h"
#include "checkpoint.h"
#include "fluid_world.h"

using phy::FluidSubsystem;
using phy::FluidWorld;
using phy::Precision;
using phy::SphParams;
using phy::LaunchTuning;
using phy::TuneTrial;
using phy::Vec3;
using phy::World;

namespace {

thread_local std::string g_last_error;

template <class R, class F>
R guard(R fail, F&& f) {
  try {
    g_last_error.clear();
    return f();
  } catch (const std::exception& e) {
    g_last_error = e.what();
  } catch (...) {
    g_last_error = "unknown error";
  }
  return fail;
}

World* as_world(PhyWorldHandle* w) { return reinterpret_cast<World*>(w); }
PhyWorldHandle* box_world(World* w) { return reinterpret_cast<PhyWorldHandle*>(w); }

FluidSubsystem& sub_of(PhyWorldHandle* w, uint32_t sub) {
  World* W = as_world(w);
  if (!W) throw std::invalid_argument("null world handle");
  if (sub >= W->subs.size()) throw std::invalid_argument("fluid subsystem index out of range");
  return *W->subs[sub];
}

Precision precision_of(int32_t p) {
  if (p == PHY_PRECISION_F64_PLAIN) return Precision::F64Plain;
  if (p == PHY_PRECISION_F32_COMP) return Precision::F32Comp;
  throw std::invalid_argument("unknown precision form");
}

// build_fluid_world (phy-ffi/src/lib.rs:113-126).
World* build_fluid_world() {
  auto* W = new World();
  try {
    auto fw = std::make_unique<FluidWorld>(SphParams::defaults(), Precision::F64Plain);
    fw->fill_box({-4.0, -4.0, -1.0}, {0.0, 4.0, 1.0}, 0.18, 0.05);
    W->subs.push_back(std::make_unique<FluidSubsystem>(std::move(fw)));
  } catch (...) {
    delete W;
    throw;
  }
  return W;
}

// Interleaved xyz readback over every fluid subsystem, truncating at len/3
// particles (phy-ffi/src/lib.rs:399-460).
template <class T>
uintptr_t read_vec(PhyWorldHandle* w, T* buf, uintptr_t len, int field) {
  World* W = as_world(w);
  if (!W || !buf) return 0;
  uintptr_t written = 0;  // particles
  for (auto& s : W->subs) {
    size_t n = s->world->len();
    if (n == 0) continue;
    uintptr_t room = len / 3 - written;
    if (room == 0) break;
    size_t take = n < room ? n : (size_t)room;
    if constexpr (std::is_same<T, float>::value) {
      // The f32 channel is cast on the device (lib.rs:595-653: an `as f32` of each value).
      s->world->get_vec_f32(field, buf + 3 * written, take);
    } else {
      // One device-to-host copy of the first `take` particles into the caller's buffer.
      s->world->get_vec_f64(field, buf + 3 * written, take);
    }
    written += take;
    if (take < n) break;
  }
  return written;
}

}  // namespace

namespace phy {
void set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }
}  // namespace phy

extern "C" {

uint32_t phy_ffi_abi_version(void) { return PHY_FFI_ABI_VERSION; }

PhyWorldHandle* phy_world_create_fluid(void) {
  return guard<PhyWorldHandle*>(nullptr, [] { return box_world(build_fluid_world()); });
}

static PhyWorldHandle* not_in_build(const char* what) {
  g_last_error = std::string(what) + ": this library holds fluid subsystems only";
  return nullptr;
}
PhyWorldHandle* phy_world_create_rigid(void) { return not_in_build("rigid world"); }
PhyWorldHandle* phy_world_create_rigid_empty(void) { return not_in_build("rigid world"); }
PhyWorldHandle* phy_world_create_granular(void) { return not_in_build("granular world"); }
PhyWorldHandle* phy_world_create_coupled(void) { return not_in_build("coupled fluid+rigid world"); }
PhyWorldHandle* phy_world_create_soft_empty(void) { return not_in_build("soft world"); }
PhyWorldHandle* phy_world_create_field_empty(void) { return not_in_build("field world"); }
PhyWorldHandle* phy_world_create_optics_empty(void) { return not_in_build("optics world"); }
PhyWorldHandle* phy_world_create_solid_empty(void) { return not_in_build("solid world"); }

int32_t phy_world_step(PhyWorldHandle* w, double dt) {
  World* W = as_world(w);
  if (!W) return -1;
  return guard<int32_t>(-1, [&] {
    W->step(dt);
    return 0;
  });
}

int32_t phy_world_step_checked(PhyWorldHandle* w, double dt) {
  World* W = as_world(w);
  if (!W) return -1;
  return guard<int32_t>(-1, [&] { return (int32_t)W->step_checked(dt); });
}

double phy_world_time(PhyWorldHandle* w) {
  World* W = as_world(w);
  return W ? W->t : std::numeric_limits<double>::quiet_NaN();
}

uintptr_t phy_world_sub_count(PhyWorldHandle* w) {
  World* W = as_world(w);
  return W ? (uintptr_t)W->subs.size() : 0;
}

uintptr_t phy_world_fluid_count(PhyWorldHandle* w) {
  World* W = as_world(w);
  return W ? (uintptr_t)W->fluid_count() : 0;
}

uintptr_t phy_world_get_fluid_positions(PhyWorldHandle* w, double* buf, uintptr_t len) {
  return guard<uintptr_t>(0, [&] { return read_vec<double>(w, buf, len, PHY_FIELD_POS); });
}
uintptr_t phy_world_get_fluid_velocities(PhyWorldHandle* w, double* buf, uintptr_t len) {
  return guard<uintptr_t>(0, [&] { return read_vec<double>(w, buf, len, PHY_FIELD_VEL); });
}
uintptr_t phy_world_get_fluid_positions_f32(PhyWorldHandle* w, float* buf, uintptr_t len) {
  return guard<uintptr_t>(0, [&] { return read_vec<float>(w, buf, len, PHY_FIELD_POS); });
}
uintptr_t phy_world_get_fluid_velocities_f32(PhyWorldHandle* w, float* buf, uintptr_t len) {
  return guard<uintptr_t>(0, [&] { return read_vec<float>(w, buf, len, PHY_FIELD_VEL); });
}

uintptr_t phy_world_rigid_count(PhyWorldHandle*) { return 0; }
uintptr_t phy_world_get_rigid_transforms(PhyWorldHandle*, double*, uintptr_t) { return 0; }
uintptr_t phy_world_get_rigid_transforms_f32(PhyWorldHandle*, float*, uintptr_t) { return 0; }

int32_t phy_world_step_f32(PhyWorldHandle* w, float dt) { return phy_world_step(w, (double)dt); }

int32_t phy_world_save(PhyWorldHandle* w, const char* path) {
  World* W = as_world(w);
  if (!W || !path) return -1;
  return guard<int32_t>(-1, [&] {
    phy::save_world(*W, path);
    return 0;
  });
}

PhyWorldHandle* phy_world_load(const char* path) {
  if (!path) return nullptr;
  return guard<PhyWorldHandle*>(nullptr, [&] { return box_world(phy::load_world(path).release()); });
}

void phy_world_destroy(PhyWorldHandle* w) {
  World* W = as_world(w);
  if (!W) return;
  guard<int>(0, [&] {
    delete W;
    return 0;
  });
}

int64_t phy_world_rigid_add_body(PhyWorldHandle*, int32_t, double, const double*, const double*) {
  g_last_error = "rigid bodies: this library holds fluid subsystems only";
  return -1;
}
int32_t phy_world_rigid_apply_force(PhyWorldHandle*, int64_t, const double*, double, int32_t) { return -1; }
int32_t phy_world_rigid_apply_torque(PhyWorldHandle*, int64_t, const double*, double, int32_t) { return -1; }
int32_t phy_world_rigid_get_velocity(PhyWorldHandle*, int64_t, double*) { return -1; }
int32_t phy_world_rigid_get_angular_velocity(PhyWorldHandle*, int64_t, double*) { return -1; }

// ---- phy_fluid_* -------------------------------------------------------------

void phy_sph_params_defaults(PhySphParams* out) {
  if (out) *out = SphParams::defaults().to_c();
}

PhyWorldHandle* phy_fluid_world_create(const PhySphParams* params, int32_t precision) {
  if (!params) return nullptr;
  return guard<PhyWorldHandle*>(nullptr, [&] {
    auto fw = std::make_unique<FluidWorld>(SphParams::from_c(*params), precision_of(precision));
    auto* W = new World();
    W->subs.push_back(std::make_unique<FluidSubsystem>(std::move(fw)));
    return box_world(W);
  });
}

int32_t phy_fluid_add_subsystem(PhyWorldHandle* w, const PhySphParams* params, int32_t precision) {
  World* W = as_world(w);
  if (!W || !params) return -1;
  return guard<int32_t>(-1, [&] {
    auto fw = std::make_unique<FluidWorld>(SphParams::from_c(*params), precision_of(precision));
    W->subs.push_back(std::make_unique<FluidSubsystem>(std::move(fw)));
    return (int32_t)(W->subs.size() - 1);
  });
}

int32_t phy_fluid_fill_box(PhyWorldHandle* w, uint32_t sub, const double* mn, const double* mx, double spacing,
                           double margin) {
  if (!mn || !mx) return -1;
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->fill_box({mn[0], mn[1], mn[2]}, {mx[0], mx[1], mx[2]}, spacing, margin);
    return 0;
  });
}

double phy_fluid_lattice_mass(PhyWorldHandle* w, uint32_t sub, double spacing) {
  return guard<double>(std::numeric_limits<double>::quiet_NaN(),
                       [&] { return sub_of(w, sub).world->lattice_mass(spacing); });
}

int32_t phy_fluid_add_particles(PhyWorldHandle* w, uint32_t sub, uint64_t n, const double* pos, const double* vel,
                                const double* mass, const uint32_t* material) {
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->add_particles((size_t)n, pos, vel, mass, material);
    return 0;
  });
}

int64_t phy_fluid_len(PhyWorldHandle* w, uint32_t sub) {
  return guard<int64_t>(-1, [&] { return (int64_t)sub_of(w, sub).world->len(); });
}

int32_t phy_fluid_get_field(PhyWorldHandle* w, uint32_t sub, int32_t field, double* out, uint64_t len) {
  if (!out) return -1;
  return guard<int32_t>(-1, [&] {
    FluidWorld& fw = *sub_of(w, sub).world;
    int nc = FluidWorld::components(field);
    if (nc == 0) throw std::invalid_argument("unknown field");
    if (len < (uint64_t)nc * fw.len()) throw std::invalid_argument("output buffer too small");
    fw.get_field(field, out);
    return 0;
  });
}

int32_t phy_fluid_set_particles_device(PhyWorldHandle* w, uint32_t sub, uint64_t n, const double* pos,
                                       const double* vel, const double* mass, const uint32_t* material) {
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->set_particles_device((size_t)n, pos, vel, mass, material);
    return 0;
  });
}

int32_t phy_fluid_get_field_device(PhyWorldHandle* w, uint32_t sub, int32_t field, double* out, uint64_t len) {
  if (!out) return -1;
  return guard<int32_t>(-1, [&] {
    FluidWorld& fw = *sub_of(w, sub).world;
    int nc = FluidWorld::components(field);
    if (nc == 0) throw std::invalid_argument("unknown field");
    if (len < (uint64_t)nc * fw.len()) throw std::invalid_argument("output buffer too small");
    fw.get_field_device(field, out);
    return 0;
  });
}

int32_t phy_fluid_set_field(PhyWorldHandle* w, uint32_t sub, int32_t field, const double* in, uint64_t len) {
  if (!in) return -1;
  return guard<int32_t>(-1, [&] {
    FluidWorld& fw = *sub_of(w, sub).world;
    int nc = FluidWorld::components(field);
    if (nc == 0) throw std::invalid_argument("unknown field");
    if (len < (uint64_t)nc * fw.len()) throw std::invalid_argument("input buffer too small");
    fw.set_field(field, in);
    return 0;
  });
}

int32_t phy_fluid_get_params(PhyWorldHandle* w, uint32_t sub, PhySphParams* out) {
  if (!out) return -1;
  return guard<int32_t>(-1, [&] {
    *out = sub_of(w, sub).world->params.to_c();
    return 0;
  });
}

int32_t phy_fluid_set_params(PhyWorldHandle* w, uint32_t sub, const PhySphParams* in) {
  if (!in) return -1;
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->params = SphParams::from_c(*in);
    return 0;
  });
}

int32_t phy_fluid_step(PhyWorldHandle* w, uint32_t sub, double dt, uint32_t n) {
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->step_n(dt, (int)n);
    return 0;
  });
}

int32_t phy_fluid_diagnostics(PhyWorldHandle* w, uint32_t sub, double* out4) {
  if (!out4) return -1;
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->diagnostics(out4);
    return 0;
  });
}

int32_t phy_fluid_couple_points(PhyWorldHandle* w, uint32_t sub, uint64_t n, const double* pos, const double* vel,
                                const double* mass, double* force, double dt, double drag, double soft_density) {
  if (n > 0 && (!pos || !vel || !mass || !force)) return -1;
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->couple_points((size_t)n, pos, vel, mass, force, dt, drag, soft_density);
    return 0;
  });
}

int32_t phy_fluid_couple_heat(PhyWorldHandle* w, uint32_t sub, const uint64_t* dims3, const double* origin3,
                              double cell, const double* temp, double* src, double dt, double t_ref, double beta,
                              double heat_gain) {
  if (!dims3 || !origin3 || !temp) return -1;
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->couple_heat(dims3, origin3, cell, temp, src, dt, t_ref, beta, heat_gain);
    return 0;
  });
}

int32_t phy_fluid_couple_bodies(PhyWorldHandle* w, uint32_t sub, PhyCoupleBody* bodies, uint32_t n_bodies,
                                const double* data, uint64_t n_data, const uint32_t* faces, uint64_t n_faces,
                                double dt, double friction) {
  (void)friction;  // unused by the reference too (world.rs:755)
  if (n_bodies > 0 && !bodies) return -1;
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->couple_bodies(bodies, n_bodies, data, n_data, faces, n_faces, dt);
    return 0;
  });
}

int32_t phy_fluid_get_coupling(PhyWorldHandle* w, uint32_t sub, double* out5) {
  if (!out5) return -1;
  return guard<int32_t>(-1, [&] {
    FluidSubsystem& s = sub_of(w, sub);
    out5[0] = s.thermal_expansion;
    out5[1] = s.heat_gain;
    out5[2] = s.t_ref;
    out5[3] = s.drag;
    out5[4] = s.friction;
    return 0;
  });
}

int32_t phy_fluid_set_coupling(PhyWorldHandle* w, uint32_t sub, const double* in5) {
  if (!in5) return -1;
  return guard<int32_t>(-1, [&] {
    FluidSubsystem& s = sub_of(w, sub);
    s.thermal_expansion = in5[0];
    s.heat_gain = in5[1];
    s.t_ref = in5[2];
    s.drag = in5[3];
    s.friction = in5[4];
    return 0;
  });
}

int32_t phy_fluid_set_stream(PhyWorldHandle* w, void* cuda_stream) {
  World* W = as_world(w);
  if (!W) return -1;
  return guard<int32_t>(-1, [&] {
    for (auto& s : W->subs) s->world->set_stream((cudaStream_t)cuda_stream);
    return 0;
  });
}

int32_t phy_fluid_pin_host(void* ptr, uint64_t bytes) {
  if (!ptr || bytes == 0) {
    g_last_error = "phy_fluid_pin_host: null pointer or zero size";
    return -1;
  }
  return guard<int32_t>(-1, [&] {
    phy::pin_host(ptr, (size_t)bytes);
    return 0;
  });
}

int32_t phy_fluid_unpin_host(void* ptr) {
  if (!ptr) {
    g_last_error = "phy_fluid_unpin_host: null pointer";
    return -1;
  }
  return guard<int32_t>(-1, [&] {
    phy::unpin_host(ptr);
    return 0;
  });
}

int32_t phy_fluid_synchronize(PhyWorldHandle* w) {
  World* W = as_world(w);
  if (!W) return -1;
  return guard<int32_t>(-1, [&] {
    for (auto& s : W->subs) s->world->synchronize();
    return 0;
  });
}

int32_t phy_fluid_step_counters(PhyWorldHandle* w, uint32_t sub, uint64_t* out4) {
  if (!out4) return -1;
  return guard<int32_t>(-1, [&] {
    FluidWorld& fw = *sub_of(w, sub).world;
    fw.last_step_counters(out4);
    out4[2] = fw.len();
    out4[3] = (uint64_t)fw.grid_cells();
    return 0;
  });
}

int32_t phy_fluid_dense_mask_info(PhyWorldHandle* w, uint32_t sub, uint64_t* out3) {
  if (!out3) return -1;
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->dense_mask_info(out3);
    return 0;
  });
}

int32_t phy_fluid_set_counting(PhyWorldHandle* w, uint32_t sub, int32_t on) {
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->set_counting(on != 0);
    return 0;
  });
}

int32_t phy_fluid_set_timing(PhyWorldHandle* w, uint32_t sub, int32_t on) {
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->set_timing(on != 0);
    return 0;
  });
}

int32_t phy_fluid_phase_times(PhyWorldHandle* w, uint32_t sub, double* out5, int32_t reset) {
  if (!out5) return -1;
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->phase_times(out5, reset != 0);
    return 0;
  });
}

int32_t phy_fluid_set_tuning(PhyWorldHandle* w, uint32_t sub, int32_t param, int64_t value) {
  return guard<int32_t>(-1, [&] {
    FluidWorld& fw = *sub_of(w, sub).world;
    LaunchTuning t = fw.launch_tuning();
    auto in_range = [&](int64_t lo, int64_t hi) {
      if (value < lo || value > hi) throw std::invalid_argument("tuning value out of range");
      return (int)value;
    };
    switch (param) {
      case PHY_TUNE_COMP_TILE:
        fw.set_comp_tile((int)value);
        break;
      case PHY_TUNE_HALO_CAP:
        fw.set_halo_cap(value > (1 << 30) ? (1 << 30) : (int)value);
        break;
      case PHY_TUNE_CTAS_PER_SM:
        t.ctas_per_sm = in_range(0, 64);
        fw.set_launch_tuning(t);
        break;
      case PHY_TUNE_QUEUE:
        t.queue = in_range(0, 1);
        fw.set_launch_tuning(t);
        break;
      case PHY_TUNE_SORT_BLOCK:
        t.sort_block = in_range(32, 256) / 32 * 32;
        fw.set_launch_tuning(t);
        break;
      case PHY_TUNE_GRAPH_CHUNK:
        fw.set_graph_chunk(in_range(0, 1 << 20));
        break;
      case PHY_TUNE_DENSE_MEAN:
        fw.set_dense_mean(in_range(1, 1 << 20));
        break;
      case PHY_TUNE_DENSE_MASKS:
        t.dense_masks = in_range(0, 1);
        fw.set_launch_tuning(t);
        break;
      default:
        throw std::invalid_argument("unknown tuning parameter");
    }
    return 0;
  });
}

int32_t phy_fluid_get_tuning(PhyWorldHandle* w, uint32_t sub, int32_t param, int64_t* out) {
  if (!out) return -1;
  return guard<int32_t>(-1, [&] {
    FluidWorld& fw = *sub_of(w, sub).world;
    const LaunchTuning t = fw.launch_tuning();
    switch (param) {
      case PHY_TUNE_COMP_TILE: *out = fw.comp_tile(); break;
      case PHY_TUNE_HALO_CAP: *out = fw.halo_cap(); break;
      case PHY_TUNE_CTAS_PER_SM: *out = t.ctas_per_sm; break;
      case PHY_TUNE_QUEUE: *out = t.queue; break;
      case PHY_TUNE_SORT_BLOCK: *out = t.sort_block; break;
      case PHY_TUNE_GRAPH_CHUNK: *out = fw.graph_chunk(); break;
      case PHY_TUNE_DENSE_MEAN: *out = fw.dense_mean(); break;
      case PHY_TUNE_DENSE_MASKS: *out = t.dense_masks; break;
      default: throw std::invalid_argument("unknown tuning parameter");
    }
    return 0;
  });
}

int32_t phy_fluid_set_scenes(PhyWorldHandle* w, uint32_t sub, uint32_t n_scenes, const uint64_t* counts,
                             const double* bounds_min, const double* bounds_max) {
  if (!counts || !bounds_min || !bounds_max) return -1;
  return guard<int32_t>(-1, [&] {
    FluidWorld& fw = *sub_of(w, sub).world;
    std::vector<uint64_t> c(counts, counts + n_scenes);
    std::vector<Vec3> lo(n_scenes), hi(n_scenes);
    for (uint32_t s = 0; s < n_scenes; ++s) {
      lo[s] = {bounds_min[3 * s], bounds_min[3 * s + 1], bounds_min[3 * s + 2]};
      hi[s] = {bounds_max[3 * s], bounds_max[3 * s + 1], bounds_max[3 * s + 2]};
    }
    try {
      fw.set_scenes(c, lo, hi);
    } catch (const std::invalid_argument& e) {
      if (std::string(e.what()).find("2^27") != std::string::npos) {
        g_last_error = e.what();
        return 5;
      }
      throw;
    }
    return 0;
  });
}

int32_t phy_fluid_clear_scenes(PhyWorldHandle* w, uint32_t sub) {
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->clear_scenes();
    return 0;
  });
}

uint32_t phy_fluid_scene_count(PhyWorldHandle* w, uint32_t sub) {
  return guard<uint32_t>(0u, [&] { return (uint32_t)sub_of(w, sub).world->scene_count(); });
}

int32_t phy_fluid_tape_begin(PhyWorldHandle* w, uint32_t sub, uint32_t checkpoint_every) {
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->tape_begin((int)checkpoint_every);
    return 0;
  });
}

int32_t phy_fluid_tape_clear(PhyWorldHandle* w, uint32_t sub) {
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->tape_clear();
    return 0;
  });
}

uint32_t phy_fluid_tape_steps(PhyWorldHandle* w, uint32_t sub) {
  return guard<uint32_t>(0u, [&] { return (uint32_t)sub_of(w, sub).world->tape_steps(); });
}

int32_t phy_fluid_step_backward(PhyWorldHandle* w, uint32_t sub, const double* grad_pos, const double* grad_vel,
                                double* grad_pos0, double* grad_vel0, double* grad_params2) {
  return guard<int32_t>(-1, [&] {
    sub_of(w, sub).world->step_backward(grad_pos, grad_vel, grad_pos0, grad_vel0, grad_params2);
    return 0;
  });
}

int32_t phy_fluid_autotune_horizon(PhyWorldHandle* w, uint32_t sub, double dt, uint32_t steps, uint32_t horizon,
                                   PhyTuneTrial* out, uint32_t cap, uint32_t* n_out) {
  return guard<int32_t>(-1, [&] {
    if (horizon > (1u << 30)) throw std::invalid_argument("autotune: horizon too large");
    const std::vector<TuneTrial> trials = sub_of(w, sub).world->autotune(dt, (int)steps, (int)horizon);
    for (size_t k = 0; out && k < trials.size() && k < cap; ++k) {
      out[k].ctas_per_sm = trials[k].tuning.ctas_per_sm;
      out[k].queue = trials[k].tuning.queue;
      out[k].sort_block = trials[k].tuning.sort_block;
      out[k].comp_tile = trials[k].comp_tile;
      out[k].ms_per_step = trials[k].ms_per_step;
      out[k].samples = trials[k].samples;
      out[k].reserved = 0;
    }
    if (n_out) *n_out = (uint32_t)trials.size();
    return 0;
  });
}

int32_t phy_fluid_autotune(PhyWorldHandle* w, uint32_t sub, double dt, uint32_t steps, PhyTuneTrial* out,
                           uint32_t cap, uint32_t* n_out) {
  return phy_fluid_autotune_horizon(w, sub, dt, steps, 0, out, cap, n_out);
}

const char* phy_fluid_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"
