// Device-side data of the adjoint of the f64 plain step (adjoint.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sph_common.cuh"

namespace phy {

// What the reverse sweep reads of one forward step, in that step's sorted
// order: the state at the step's start, the per-particle constants, the
// step's intermediate values and its cell ranges.
struct AdjTape {
  const double* x[3];
  const double* v[3];
  const double* mass;
  const uint32_t* mat;
  const uint32_t* id;   // sorted slot -> insertion index
  const double* rho;
  const double* p;
  const double* pr2;    // p / rho^2
  const double* mr;     // mass / rho
  const double* acc[3];
  const double* xsph[3];
  const double* mu;
  const double* fv[3];  // raw viscous force (before mu)
  const double* shear;  // strain-rate proxy
  const uint32_t* cell_start;
  // The density pass's neighbour lists (entry k of slot i at nbr[k * n + i],
  // every j != i not excluded by r >= h, in visit order); a count above
  // kMaxNeighbors means the list overflowed and the 27 cells are rescanned.
  const uint32_t* nbr;
  const uint32_t* nbr_count;
};

// Adjoint state: gx_ins / gv_ins hold dL/dx, dL/dv in insertion order
// between steps (dL/dx', dL/dv' on entry to a reverse step, dL/dx, dL/dv on
// exit); the rest is per-step scratch in sorted order.
struct AdjWork {
  double* gx_ins[3];
  double* gv_ins[3];
  double* gx[3];
  double* gv[3];
  double* P[3];   // dL/d f_press
  double* Q[3];   // dL/d f_visc_raw
  double* Y[3];   // dL/d xsph
  double* sig;    // dL/d shear
  double* rbar;   // direct dL/d rho (through acc)
  double* rbar_tot;
  double* cc;     // per-particle dL/d visc_k[0] terms
  double* kk;     // per-particle dL/d stiffness terms
  double* param_acc;  // device {dL/d stiffness, dL/d visc_k[0]}, accumulated
};

void launch_adjoint_step(const StepConsts& c, const AdjTape& t, const AdjWork& w, cudaStream_t s);

}  // namespace phy
