#ifndef PHY_FLUID_H
#define PHY_FLUID_H

/*
 * SPH fluid entry points added by the B200 build (ABI version 3).
 *
 * They expose the reference's Rust API of crates/phy-fluid to C callers:
 * SphParams<T> (src/sph/params.rs:12-86), FluidWorld<T> (src/sph/world.rs:
 * 21-197) and FluidSubsystem<T> (src/subsystem.rs:26-164).  A world handle is
 * the PhyWorldHandle of phy_ffi.h; `sub` selects a fluid subsystem by its index
 * among the world's fluid subsystems (0 for the first).
 *
 * Particle fields are read and written in insertion order, exactly like the
 * reference's `FluidWorld::particles` Vec, whatever order the device keeps
 * them in.  Vector fields are xyz-interleaved (3 doubles per particle).
 *
 * Precision forms of the step:
 *   PHY_PRECISION_F64_PLAIN  f64 everywhere, the reference's operation order,
 *                            no FMA contraction: bit-identical to
 *                            FluidWorld<f64>::step and run-to-run.
 *   PHY_PRECISION_F32_COMP   pairwise kernel math in f32 on cell-relative
 *                            coordinates with compensated (Kahan) sums of
 *                            density and force; positions, velocities,
 *                            cell keys, integration and diagnostics stay f64.
 *
 * Return codes are those of phy_ffi.h.
 */

#include <stddef.h>
#include <stdint.h>

#include "phy_ffi.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PHY_MAX_MATERIALS 16

enum {
  PHY_PRECISION_F64_PLAIN = 0,
  PHY_PRECISION_F32_COMP = 1
};

/* Particle fields (crates/phy-fluid/src/particle.rs:17-46). */
enum {
  PHY_FIELD_POS = 0,      /* 3 per particle */
  PHY_FIELD_VEL = 1,      /* 3 */
  PHY_FIELD_ACC = 2,      /* 3, written by the step */
  PHY_FIELD_BODY_ACC = 3, /* 3, coupling input, zeroed by the step */
  PHY_FIELD_RHO = 4,      /* 1, written by the step */
  PHY_FIELD_P = 5,        /* 1, written by the step */
  PHY_FIELD_MASS = 6,     /* 1 */
  PHY_FIELD_MU_EFF = 7,   /* 1, written by the step */
  PHY_FIELD_XSPH = 8,     /* 3, written by the step */
  PHY_FIELD_MATERIAL = 9  /* 1, integer value carried in a double */
};

/* SphParams<f64> (crates/phy-fluid/src/sph/params.rs:12-86).  The two
 * per-material tables are Rust Vecs there; here they hold n_visc_k and
 * n_visc_n entries (1..PHY_MAX_MATERIALS).  `viscosity` is carried but, as in
 * the reference, the step reads visc_k/visc_n only. */
typedef struct PhySphParams {
  double rest_density;
  double stiffness;
  double viscosity;
  double shear_min;
  double mass;
  double h;
  double gravity[3];
  double bounds_min[3];
  double bounds_max[3];
  double boundary_damp;
  double xsph_eps;
  uint32_t n_visc_k;
  uint32_t n_visc_n;
  double visc_k[PHY_MAX_MATERIALS];
  double visc_n[PHY_MAX_MATERIALS];
} PhySphParams;

/* SphParams::defaults() (params.rs:55-85). */
void phy_sph_params_defaults(PhySphParams *out);

/* World holding one empty FluidSubsystem::new(FluidWorld::new(params))
 * (world.rs:94-102, subsystem.rs:44-55).  The smoothing length used by the
 * kernel coefficients and the grid cell is captured here, as in the
 * reference; later changes of params->h move only the cutoff tests. */
PhyWorldHandle *phy_fluid_world_create(const PhySphParams *params, int32_t precision);

/* Appends another fluid subsystem; returns its `sub` index or -1. */
int32_t phy_fluid_add_subsystem(PhyWorldHandle *w, const PhySphParams *params, int32_t precision);

/* FluidWorld::fill_box (world.rs:124-144). */
int32_t phy_fluid_fill_box(PhyWorldHandle *w, uint32_t sub, const double *min3, const double *max3,
                           double spacing, double margin);

/* FluidWorld::lattice_mass (world.rs:148-169); NaN on error. */
double phy_fluid_lattice_mass(PhyWorldHandle *w, uint32_t sub, double spacing);

/* Appends n particles like Particle::with_material (particle.rs:50-71) with
 * the given velocity.  vel and material may be NULL (zero / material 0). */
int32_t phy_fluid_add_particles(PhyWorldHandle *w, uint32_t sub, uint64_t n, const double *pos,
                                const double *vel, const double *mass, const uint32_t *material);

/* FluidWorld::len (world.rs:105-107); -1 on error. */
int64_t phy_fluid_len(PhyWorldHandle *w, uint32_t sub);

/* Reads / writes one particle field for all particles, insertion order.
 * len is in doubles and must be at least len(sub) * components. */
int32_t phy_fluid_get_field(PhyWorldHandle *w, uint32_t sub, int32_t field, double *out, uint64_t len);
int32_t phy_fluid_set_field(PhyWorldHandle *w, uint32_t sub, int32_t field, const double *in,
                            uint64_t len);

/* Device-memory forms for callers whose particle data already lives on the
 * GPU (a multi-GPU decomposition moving slabs between devices, an engine
 * feeding its own buffers), so no host copy is made:
 *   phy_fluid_set_particles_device replaces the whole particle set of `sub`
 *   (the counterpart of assigning the reference's public `particles` Vec,
 *   world.rs:21-30) from device arrays: pos and vel 3n doubles xyz
 *   interleaved, mass n doubles, material n u32; vel and material may be
 *   NULL (zeros).  Every other particle field starts at zero, as
 *   Particle::new (particle.rs:50-63).  The positions may widen the grid box.
 *   phy_fluid_get_field_device writes one field in insertion order to a
 *   device buffer of at least len(sub) * components doubles.
 * Both return after the world's stream has finished; 0 or -1 (batched
 * scenes, an active adjoint tape, null arguments). */
int32_t phy_fluid_set_particles_device(PhyWorldHandle *w, uint32_t sub, uint64_t n, const double *pos,
                                       const double *vel, const double *mass, const uint32_t *material);
int32_t phy_fluid_get_field_device(PhyWorldHandle *w, uint32_t sub, int32_t field, double *out, uint64_t len);

/* The public `params` field: live read and write. */
int32_t phy_fluid_get_params(PhyWorldHandle *w, uint32_t sub, PhySphParams *out);
int32_t phy_fluid_set_params(PhyWorldHandle *w, uint32_t sub, const PhySphParams *in);

/* FluidWorld::step (world.rs:183-192) on one subsystem, `n` times, without
 * the World's coupling stage or time accumulation. */
int32_t phy_fluid_step(PhyWorldHandle *w, uint32_t sub, double dt, uint32_t n);

/* FluidSubsystem::total_momentum and kinetic_energy (subsystem.rs:149-163):
 * out4 = {Px, Py, Pz, KE}, summed in insertion order in f64. */
int32_t phy_fluid_diagnostics(PhyWorldHandle *w, uint32_t sub, double *out4);

/* FluidWorld::couple_points (crates/phy-fluid/src/sph/world.rs:691-752, with
 * CouplePoint of sph/couple.rs): two-way coupling of n point masses with the
 * fluid of subsystem `sub`, computed on the device and bit-identical to the
 * reference.  pos, vel: 3n doubles (xyz per point, read only); mass: n;
 * force: 3n doubles, written for the points inside the bounds (the others
 * keep their values).  Points are taken in order: each samples the
 * mass-weighted fluid velocity of its 27 grid cells and shares -force*dt
 * among those particles by mass before the next point.  Fails (-1) on a
 * world of batched scenes or while the adjoint tape records. */
int32_t phy_fluid_couple_points(PhyWorldHandle *w, uint32_t sub, uint64_t n, const double *pos, const double *vel,
                                const double *mass, double *force, double dt, double drag, double soft_density);

/* FluidWorld::couple_heat (crates/phy-fluid/src/sph/world.rs:555-678; the
 * HeatFieldLike grid of phy-field heat.rs:15-33, grid.rs:80-82, 125-130,
 * 203-208): thermal buoyancy and advective heating between the fluid of
 * subsystem `sub` and a heat grid, computed on the device and bit-identical
 * to the reference.  The grid has dims3[0] x dims3[1] x dims3[2] cells of
 * size `cell` from origin3, values x fastest.  Every particle inside the
 * bounds gets body_acc += -g * beta * (T - t_ref), T its trilinear grid
 * temperature (t_ref outside the grid); with heat_gain > 0 the sources `src`
 * (same layout, updated in place; may be NULL otherwise) take
 * heat_gain * |v| * dt per particle, added in insertion order.  The velocity
 * sampler the reference installs into the field is left to the caller (it
 * captures the positions and velocities phy_fluid_get_field returns).  Fails
 * (-1) on a world of batched scenes or while the adjoint tape records. */
int32_t phy_fluid_couple_heat(PhyWorldHandle *w, uint32_t sub, const uint64_t *dims3, const double *origin3,
                              double cell, const double *temp, double *src, double dt, double t_ref, double beta,
                              double heat_gain);

/* One rigid body for phy_fluid_couple_bodies: the parts of phy-rigid's Body
 * (crates/phy-rigid/src/shape.rs:330-372) and Shape (shape.rs:138-176) that
 * couple_bodies reads.  Shapes: sphere size {r}; capsule {half_height, r}
 * along local y; box half extents; convex: data_count vertices (xyz triples
 * from data[data_first]) and face_count index triples (from
 * faces[3 * face_first], indices into the body's vertices); heightfield
 * {nx, nz, cell} with data_count = nx * nz heights from data[data_first].
 * Compound shapes are not supported. */
#define PHY_SHAPE_SPHERE 0
#define PHY_SHAPE_CAPSULE 1
#define PHY_SHAPE_BOX 2
#define PHY_SHAPE_CONVEX 3
#define PHY_SHAPE_HEIGHTFIELD 4
/* Shape::Compound (phy-rigid shape.rs:176-192): data_count sub shapes (at
 * least one) as 16-double records from data[data_first]: shape (0..4; no
 * nested compounds), size[3], offset[3] and unit quaternion (i, j, k, w)
 * relative to the body, then data_first, data_count, face_first, face_count
 * of the sub shape's own convex / heightfield data, and one unused value. */
#define PHY_SHAPE_COMPOUND 5
typedef struct PhyCoupleBody {
  int32_t shape;
  uint32_t data_first, data_count, face_first, face_count, reserved;
  double size[3];
  double pos[3];
  double rot[4]; /* unit quaternion (i, j, k, w) */
  double vel[3]; /* linear velocity, updated by the call */
  double inv_mass; /* 0 = static */
} PhyCoupleBody;

/* FluidWorld::couple_bodies (crates/phy-fluid/src/sph/world.rs:414-503):
 * symmetric soft contact and buoyancy between the fluid of subsystem `sub`
 * and n_bodies rigid bodies, computed on the device and bit-identical to
 * the reference's loops (particles in insertion order, bodies in order).
 * Particles inside a body are pushed to its surface and lose their inward
 * normal velocity; dynamic bodies take the contact impulses and, when any
 * particle entered them, the buoyancy impulse -g rho0 V dt of their volume.
 * `friction` is unused, as in the reference.  Fails (-1) on invalid shapes
 * or ranges, on a world of batched scenes, or while the adjoint tape
 * records. */
int32_t phy_fluid_couple_bodies(PhyWorldHandle *w, uint32_t sub, PhyCoupleBody *bodies, uint32_t n_bodies,
                                const double *data, uint64_t n_data, const uint32_t *faces, uint64_t n_faces,
                                double dt, double friction);

/* FluidSubsystem coupling coefficients (subsystem.rs:26-55):
 * {thermal_expansion, heat_gain, t_ref, drag, friction}. */
int32_t phy_fluid_get_coupling(PhyWorldHandle *w, uint32_t sub, double *out5);
int32_t phy_fluid_set_coupling(PhyWorldHandle *w, uint32_t sub, const double *in5);

/* Runs all of the world's device work on the given cudaStream_t (NULL = the
 * handle's own stream).  The caller keeps the stream alive. */
int32_t phy_fluid_set_stream(PhyWorldHandle *w, void *cuda_stream);

/* Blocks until the world's device work has finished. */
int32_t phy_fluid_synchronize(PhyWorldHandle *w);

/* Page-locks a caller-owned host buffer of `bytes` bytes (cudaHostRegister)
 * so that readbacks into it (phy_world_get_fluid_positions/velocities and
 * their f32 forms, phy_fluid_get_field) are single DMA copies instead of
 * staged pageable copies: the zero-copy form of the reference's per-frame
 * readback path (phy-ffi/src/lib.rs:399-460, 595-653).  Optional; the buffer
 * stays valid for every other use.  Undo with phy_fluid_unpin_host before
 * freeing it.  0, or -1 (null, zero size, already registered, or refused by
 * the driver; phy_fluid_last_error() says why). */
int32_t phy_fluid_pin_host(void *ptr, uint64_t bytes);
int32_t phy_fluid_unpin_host(void *ptr);

/* Enables (on != 0) or disables counting of neighbour candidates and pairs
 * in the density pass of `sub` (one atomic per warp; off by default). */
int32_t phy_fluid_set_counting(PhyWorldHandle *w, uint32_t sub, int32_t on);

/* Counters of the last counted step of `sub`: out4 = {candidates visited,
 * pairs with r < h, particles, grid cells}.  Used for roofline accounting. */
int32_t phy_fluid_step_counters(PhyWorldHandle *w, uint32_t sub, uint64_t *out4);

/* The dense-cell mask buffer of `sub` (PHY_TUNE_DENSE_MASKS), after waiting
 * for its stream: out3 = {entries allocated, entries the dense-cell tasks of
 * the last step reserved, 1 when the last step's force pass found a task's
 * kept masks outside the buffer (it filtered that task again) else 0}.  An
 * entry is one chunk of 32 candidates (33 u32). */
int32_t phy_fluid_dense_mask_info(PhyWorldHandle *w, uint32_t sub, uint64_t *out3);

/* Per-phase device timing of `sub` with CUDA events on its stream.  While on,
 * every step records five events without waiting for them (steps are then
 * not captured into CUDA graphs); phy_fluid_phase_times waits for the last
 * timed step and returns the accumulated milliseconds
 * out5 = {sort, per-particle prep, density pass, force pass, steps timed}
 * and resets them when reset != 0. */
int32_t phy_fluid_set_timing(PhyWorldHandle *w, uint32_t sub, int32_t on);
int32_t phy_fluid_phase_times(PhyWorldHandle *w, uint32_t sub, double *out5, int32_t reset);

/* Kernel configuration of `sub` (no effect on the f64 plain form's results):
 *   PHY_TUNE_COMP_TILE    0 = x-major cell runs, 4 = staged 4x4x4-cell tiles
 *                         (default), 2 = staged 2x2x2-cell tiles, for the
 *                         FP32-compensated passes (cells per tile edge);
 *   PHY_TUNE_HALO_CAP     staged particles per tile halo before a tile is
 *                         computed from global memory (default: the kernels'
 *                         capacity);
 *   PHY_TUNE_DENSE_MEAN   mean particles per occupied cell above which a
 *                         tile goes to the dense-cell passes (default 32).
 * Launch knobs (results never depend on them):
 *   PHY_TUNE_CTAS_PER_SM  resident CTAs per SM of the tiled passes'
 *                         persistent grids (0 = occupancy limit, default);
 *   PHY_TUNE_QUEUE        0 = static tile stride, 1 = device work queue;
 *   PHY_TUNE_SORT_BLOCK   threads per block of the sort's per-particle
 *                         kernels (32..256, default 256);
 *   PHY_TUNE_GRAPH_CHUNK  0 = launch every step (default); k > 0 = capture
 *                         runs of k steps of phy_fluid_step into a CUDA graph
 *                         once and replay it (re-captured when parameters,
 *                         dt, the particle set or a buffer change);
 *   PHY_TUNE_DENSE_MASKS  1 = the dense-cell force pass walks the in-range
 *                         masks the density pass kept (default; the buffer
 *                         grows with the tasks' demand, within a quarter of
 *                         the free device memory and 16 GiB), 0 = it filters
 *                         the candidates again.
 * phy_fluid_get_tuning reads the same parameters. */
enum {
  PHY_TUNE_COMP_TILE = 0,
  PHY_TUNE_HALO_CAP = 1,
  PHY_TUNE_CTAS_PER_SM = 2,
  PHY_TUNE_QUEUE = 3,
  PHY_TUNE_SORT_BLOCK = 4,
  PHY_TUNE_GRAPH_CHUNK = 5,
  PHY_TUNE_DENSE_MEAN = 6,
  PHY_TUNE_DENSE_MASKS = 7
};
int32_t phy_fluid_set_tuning(PhyWorldHandle *w, uint32_t sub, int32_t param, int64_t value);
int32_t phy_fluid_get_tuning(PhyWorldHandle *w, uint32_t sub, int32_t param, int64_t *out);

/* Batched scenes (no counterpart in the reference, which steps one scene per
 * FluidWorld).  Partitions the subsystem's particles, in insertion order,
 * into n_scenes consecutive scenes of counts[s] particles with their own wall
 * bounds (bounds_min / bounds_max: 3 doubles per scene, replacing
 * SphParams::bounds_* for that scene) and their own grid box.  Every
 * phy_fluid_step then advances all scenes with one sort and one persistent
 * launch per pass; scenes never interact and share every other parameter.
 * Each scene's result is bit-identical to the same scene stepped alone in a
 * world of the same form and kernel configuration.  FP32-compensated tiled
 * form only; afterwards phy_fluid_add_particles fails until
 * phy_fluid_clear_scenes.  1 <= n_scenes <= 65535; the counts must add up to
 * the particle count.  Returns 0, -1 (bad arguments) or 5 (the boxes exceed
 * 2^27 cells). */
int32_t phy_fluid_set_scenes(PhyWorldHandle *w, uint32_t sub, uint32_t n_scenes, const uint64_t *counts,
                             const double *bounds_min, const double *bounds_max);
int32_t phy_fluid_clear_scenes(PhyWorldHandle *w, uint32_t sub);
uint32_t phy_fluid_scene_count(PhyWorldHandle *w, uint32_t sub);

/* One autotuner candidate: launch knobs and the measured device time. */
typedef struct PhyTuneTrial {
  int32_t ctas_per_sm;
  int32_t queue;
  int32_t sort_block;
  int32_t comp_tile;   /* cells per tile edge of the trial (0: not a tiled world) */
  double ms_per_step;  /* mean over the sampled states the trial ran on */
  int32_t samples;     /* sampled states it ran on */
  int32_t reserved;
} PhyTuneTrial;

/* Autotuner (no reference counterpart): times `steps` steps of dt for every
 * combination of the knobs (sort block 128/256, static stride or work
 * queue, 1..occupancy-limit CTAs per SM, and for tiled worlds 4 or 2 cells
 * per tile edge), each from the same saved state, restores that state, and
 * keeps the fastest configuration.  Writes up to `cap` trials to out (may be
 * NULL) and their number to *n_out.  No knob changes a result bit except the
 * tile edge, which changes the compensated form's summation order only. */
int32_t phy_fluid_autotune(PhyWorldHandle *w, uint32_t sub, double dt, uint32_t steps, PhyTuneTrial *out,
                           uint32_t cap, uint32_t *n_out);

/* The same over the run ahead: first steps `horizon` steps with the current
 * configuration, saving the states after horizon/2 and horizon steps; every
 * candidate runs from the starting state, the six fastest also from the two
 * later ones, and the fastest mean over the three wins (a collapsing scene
 * gets the configuration of the states it will spend its time in).  The
 * world returns to its starting state.  horizon = 0 is phy_fluid_autotune. */
int32_t phy_fluid_autotune_horizon(PhyWorldHandle *w, uint32_t sub, double dt, uint32_t steps, uint32_t horizon,
                                   PhyTuneTrial *out, uint32_t cap, uint32_t *n_out);

/* Adjoint of the SPH step, f64 plain worlds and FP32-compensated worlds on
 * the tiled passes (the default; the x-major route is rejected).
 * phy_fluid_tape_begin makes the current state checkpoint 0 and records every
 * following phy_fluid_step of `sub` (its dt), saving a state checkpoint every
 * `checkpoint_every` steps; parameters must stay unchanged and body
 * accelerations unset while recording.  phy_fluid_step_backward runs the
 * reverse sweep over all recorded steps, re-running each segment forward
 * from its checkpoint (the f64 plain step repeats bit-exactly): given
 * dL/dpos_T and dL/dvel_T (3n doubles each, insertion order, xyz
 * interleaved; NULL = zero) it writes dL/dpos_0, dL/dvel_0 (3n each) and
 * grad_params2 = {dL/d stiffness, dL/d visc_k[0]} (any output may be NULL).
 * Neighbour sets and branches (walls, max(0, .), shear_min) are held as the
 * forward took them.  A compensated world is differentiated along its own
 * trajectory: each re-run step first takes an f64 plain recording step from
 * the compensated state, so the sweep is the exact adjoint of the step map at
 * the states the compensated forward visited.  The world is left in its
 * recorded end state and the tape is kept for further sweeps until
 * phy_fluid_tape_clear or the next phy_fluid_tape_begin.  The reference has
 * no adjoint; these calls replace nothing in phy_ffi.h. */
int32_t phy_fluid_tape_begin(PhyWorldHandle *w, uint32_t sub, uint32_t checkpoint_every);
int32_t phy_fluid_tape_clear(PhyWorldHandle *w, uint32_t sub);
uint32_t phy_fluid_tape_steps(PhyWorldHandle *w, uint32_t sub);
int32_t phy_fluid_step_backward(PhyWorldHandle *w, uint32_t sub, const double *grad_pos, const double *grad_vel,
                                double *grad_pos0, double *grad_vel0, double *grad_params2);

/* Scratch capacity of phy_fluid_density_noalloc. */
#define PHY_NOALLOC_MAX_PARTICLES 65536
#define PHY_NOALLOC_MAX_CELLS 262144

/* Density and pressure of n particles in caller-owned device buffers,
 * computed without allocating any device memory.  This entry point has no
 * counterpart in the reference: it is for callers that cannot allocate on
 * the device at that moment (an engine that owns all device memory and gives
 * plugins only its own buffers, a process whose allocator policy forbids
 * foreign cudaMalloc/cudaFree, a latency-critical loop that must not enter the
 * driver's allocator).  Inputs: pos (3n doubles, xyz interleaved) and mass
 * (n); outputs: rho and p (n doubles each); all device pointers, caller
 * order.  The values are bit-identical to the density pass of the f64 plain
 * step (FluidWorld<f64>::compute_density_pressure, world.rs:204-246) with
 * kernel coefficients and grid cell taken from params->h.
 *   Limits: n <= PHY_NOALLOC_MAX_PARTICLES and a cell-key bounding box (plus
 * one cell on each side) of at most PHY_NOALLOC_MAX_CELLS cells; larger
 * inputs return -1 and phy_fluid_last_error() says why.
 *   Scratch: one fixed 4 MiB array in device memory that every GPU which
 * loads the library holds until the process exits.  All calls share it and
 * it keeps the last call's contents, so calls that overlap on the GPU (other
 * threads or streams on the same device) race; serialise them.  The first
 * call on a device looks up the array's address with that device current;
 * make that first call before any stream capture.  The call works on the
 * given cudaStream_t (NULL: the legacy default stream) and returns after that
 * stream has finished.  Returns 0 or -1. */
int32_t phy_fluid_density_noalloc(const PhySphParams *params, uint64_t n, const double *pos,
                                  const double *mass, double *rho, double *p, void *cuda_stream);

/* Message of the last failing call on this thread ("" if none). */
const char *phy_fluid_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* PHY_FLUID_H */
