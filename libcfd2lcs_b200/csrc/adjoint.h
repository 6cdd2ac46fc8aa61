// Reverse-mode derivative of a backward-FTLE objective with respect to the gridded velocity
// at every time level (adjoint.cu).  No counterpart in the reference library.
#pragma once

#include <string>

#include "engine.h"

namespace cfd2lcs {

struct AdjointProblem {
  const int *n;                      // grid points per direction
  const lcsdata_t *x, *y, *z;        // coordinates (as cfd2lcs_init), i fastest
  int integrator;                    // EULER, TRAPEZOIDAL, RK2, RK3 or RK4
  double cfl;                        // CFL number of the subcycling (cfd2lcs_set_param "CFL")
  int nlevels;                       // velocity levels, >= 2
  const lcsdata_t *const *u, *const *v, *const *w;  // device pointers, one per level, n[0]n[1]n[2] each
  const lcsdata_t *times;            // host, one per level, increasing
  const lcsdata_t *weight;           // device, n[0]n[1]n[2]: J = sum weight * FTLE
  int checkpoint_every;              // updates between stored flow maps (>= 1)
  lcsdata_t *const *gu, *const *gv, *const *gw;  // device outputs, one per level (may be null: J only)
  // tangent-linear direction, device, one per level (may be null): with it, *dJ = dJ/du . d by
  // a forward-mode sweep alongside the flow map
  const lcsdata_t *const *du = nullptr, *const *dv = nullptr, *const *dw = nullptr;
  double *dJ = nullptr;
  int interpolator = 1;              // LINEAR (1) or CUBIC (3)
  const int *flag = nullptr;         // boundary flags as cfd2lcs_init takes them (null: all LCS_INTERNAL)
};

// Runs the backward flow map over all levels (LINEAR or CUBIC interpolation), the FTLE of the final
// map and J; with gradient outputs, the adjoint sweep; with a tangent direction, the tangent-
// linear sweep in the same forward pass.  Returns false with msg on error.
bool adjoint_ftle(const AdjointProblem &p, double *J, std::string &msg);

}  // namespace cfd2lcs
