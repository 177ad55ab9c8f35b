// Fluid-world checkpoints in the reference's JSON archive layout
// (crates/phy-io/src/archive.rs:37-91, 150-311):
//   {"version":1, "time":F, "subsystems":[{"Fluid":{"world":{"params":{...},
//    "particles":[...]}, "thermal_expansion":F, "heat_gain":F, "t_ref":F,
//    "drag":F, "friction":F}}]}
// where every f64 scalar F is written as {"__f64": <u64 bit pattern>} and every
// Vec3 as [bits, bits, bits] (crates/phy-rigid/src/shape.rs:18-53), so a save /
// load round trip is bit-exact.  Particle fields follow Particle<T>'s serde
// layout (crates/phy-fluid/src/particle.rs:17-46): mu_eff and xsph are not
// stored and come back as zero.
#pragma once

#include <memory>
#include <string>

#include "fluid_world.h"

namespace phy {

std::string save_world_json(World& w);
std::unique_ptr<World> load_world_json(const std::string& json);
void save_world(World& w, const char* path);
std::unique_ptr<World> load_world(const char* path);

}  // namespace phy
