#ifndef PHY_FFI_H
#define PHY_FFI_H

/*
 * Drop-in C ABI of the SPH fluid world, B200 build (libphysph.so).
 *
 * Every declaration below replaces the symbol of the same name exported by the
 * reference's Rust cdylib `phy-ffi` (crates/phy-ffi/src/lib.rs, header
 * crates/phy-ffi/phy_ffi.h).  Signatures, argument meaning, return codes and
 * null-pointer behaviour are kept; the fluid mechanics behind them run as
 * CUDA kernels on the current device.  Worlds hold only fluid subsystems in
 * this library: the rigid / granular / soft / field / optics / solid factories
 * and the rigid-body controls are exported with the reference's failure values
 * (NULL, -1, 0) so that existing binaries still link and fail cleanly.
 *
 * Return codes (phy-ffi/src/lib.rs:330-363):
 *    0  success
 *   -1  null handle, invalid argument or internal error (the reference's
 *       caught panic); phy_fluid_last_error() holds a message
 *    2  non-finite position or velocity after the step (WorldError::NonFinite)
 *    3  a subsystem did not advance (WorldError::Stalled; never produced here)
 *    4  other WorldError
 *    5  the device reported a cell key outside the neighbour grid (new code,
 *       only reachable with non-finite positions outside the grid box)
 *
 * Threading: a handle is used by one host thread at a time (the reference's
 * World is not Send).  Distinct handles may be used concurrently.
 */

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ABI version: 3 = the reference's 2 plus the phy_fluid_* symbols of
 * phy_fluid.h (phy-ffi/src/lib.rs:32-34 requires a bump on additions that
 * change the contract). */
#define PHY_FFI_ABI_VERSION 3
#define PHY_FFI_VERSION_MAJOR 0
#define PHY_FFI_VERSION_MINOR 2
#define PHY_FFI_VERSION_PATCH 0

/* Opaque handle (phy-ffi/src/lib.rs:64-67). */
typedef struct PhyWorldHandle PhyWorldHandle;

/* phy-ffi/src/lib.rs:106-109 */
uint32_t phy_ffi_abi_version(void);

/* Dam-break fluid world: SphParams::defaults(), fill_box((-4,-4,-1),(0,4,1),
 * 0.18, 0.05) in one FluidSubsystem (phy-ffi/src/lib.rs:113-126, 209-214). */
PhyWorldHandle *phy_world_create_fluid(void);

/* Non-fluid factories: not part of this library, return NULL
 * (phy-ffi/src/lib.rs:216-248, 299-328). */
PhyWorldHandle *phy_world_create_rigid(void);
PhyWorldHandle *phy_world_create_rigid_empty(void);
PhyWorldHandle *phy_world_create_granular(void);
PhyWorldHandle *phy_world_create_coupled(void);
PhyWorldHandle *phy_world_create_soft_empty(void);
PhyWorldHandle *phy_world_create_field_empty(void);
PhyWorldHandle *phy_world_create_optics_empty(void);
PhyWorldHandle *phy_world_create_solid_empty(void);

/* World::step (phy-ffi/src/lib.rs:330-338): 0 ok, -1 null/error. */
int32_t phy_world_step(PhyWorldHandle *w, double dt);

/* World::step_checked (phy-ffi/src/lib.rs:350-363): 0, -1, 2, 3, 4 (and 5). */
int32_t phy_world_step_checked(PhyWorldHandle *w, double dt);

/* phy-ffi/src/lib.rs:365-372: NaN for a null handle. */
double phy_world_time(PhyWorldHandle *w);

/* phy-ffi/src/lib.rs:374-378 */
uintptr_t phy_world_sub_count(PhyWorldHandle *w);

/* phy-ffi/src/lib.rs:380-397 */
uintptr_t phy_world_fluid_count(PhyWorldHandle *w);

/* Interleaved xyz of every fluid particle in subsystem then insertion order;
 * returns particles written, truncating at len/3 (phy-ffi/src/lib.rs:399-429). */
uintptr_t phy_world_get_fluid_positions(PhyWorldHandle *w, double *buf, uintptr_t len);

/* phy-ffi/src/lib.rs:431-460 */
uintptr_t phy_world_get_fluid_velocities(PhyWorldHandle *w, double *buf, uintptr_t len);

/* No rigid subsystems in this library: 0 (phy-ffi/src/lib.rs:462-515). */
uintptr_t phy_world_rigid_count(PhyWorldHandle *w);
uintptr_t phy_world_get_rigid_transforms(PhyWorldHandle *w, double *buf, uintptr_t len);

/* Fluid-world checkpoint to a JSON file in the reference's archive layout
 * (phy-ffi/src/lib.rs:517-542, phy-io/src/archive.rs:37-91). 0 / -1. */
int32_t phy_world_save(PhyWorldHandle *w, const char *path);
PhyWorldHandle *phy_world_load(const char *path);

/* Null-safe release (phy-ffi/src/lib.rs:544-553). */
void phy_world_destroy(PhyWorldHandle *w);

/* f32 channel (phy-ffi/src/lib.rs:573-653): dt cast to f64; readbacks are
 * exact `as f32` casts of the f64 state. */
int32_t phy_world_step_f32(PhyWorldHandle *w, float dt);
uintptr_t phy_world_get_fluid_positions_f32(PhyWorldHandle *w, float *buf, uintptr_t len);
uintptr_t phy_world_get_fluid_velocities_f32(PhyWorldHandle *w, float *buf, uintptr_t len);
uintptr_t phy_world_get_rigid_transforms_f32(PhyWorldHandle *w, float *buf, uintptr_t len);

/* Rigid-body controls: no rigid subsystem here, always -1
 * (phy-ffi/src/lib.rs:691-899). */
int64_t phy_world_rigid_add_body(PhyWorldHandle *w, int32_t shape_kind, double mass,
                                 const double *pos7, const double *inertia3);
int32_t phy_world_rigid_apply_force(PhyWorldHandle *w, int64_t id, const double *f3, double dt,
                                    int32_t mode);
int32_t phy_world_rigid_apply_torque(PhyWorldHandle *w, int64_t id, const double *t3, double dt,
                                     int32_t mode);
int32_t phy_world_rigid_get_velocity(PhyWorldHandle *w, int64_t id, double *out3);
int32_t phy_world_rigid_get_angular_velocity(PhyWorldHandle *w, int64_t id, double *out3);

#ifdef __cplusplus
}
#endif

#endif /* PHY_FFI_H */
