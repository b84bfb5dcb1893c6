// nb_flow.cuh — device view of a MAC case and the flow-kernel host wrappers.
#pragma once
#include "nb_internal.h"

namespace nb {

// Per-case constants + level-0 brick view (passed by value to kernels).
struct FlowView {
  LevelView L;
  double origin[3];
  double wallv[6][3];
  double inlet_speed[6];
  int profile[6];
  int inlet_axis[6];
  int per[3];        // periodic(axis): face[2*axis] is periodic (grid.hpp:68-71)
  long long nb;      // slab offset = nbrick*512
  int weno;
  int has_solid;
  double nu;
  double bf[3];
  double density, velocity_scale;
};

// One velocity boundary action (applyVelocityBC, ns_solver.cpp:221-309).
struct BcOp {
  int comp;       // 0 u, 1 v, 2 w
  int action;     // 0 set `val`, 1 copy from `src`
  long long idx;  // storage index of the face
  long long src;  // storage index of the copy source
  double val;
};

struct StepScalars {  // per-step diagnostics (device), ns_solver.cpp:797-823
  double du2, div2, divmax, fx, fy, mass, maxinv;
};

// host wrappers (nb_flow.cu)
void launch_bc(cudaStream_t s, const BcOp* ops, int n, int serial, double* u, double* v, double* w);
void launch_rhs_rk(cudaStream_t s, const FlowView& F, int stage, const double* dtp, const double* u,
                   const double* v, const double* w, const double* u0, const double* v0,
                   const double* w0, double* uo, double* vo, double* wo, int mixed, int grid_cap);
void launch_div(cudaStream_t s, const FlowView& F, const double* u, const double* v, const double* w,
                double* b);
void launch_correct(cudaStream_t s, const FlowView& F, const double* phi, const double* dtp, double* u,
                    double* v, double* w, double* p);
void launch_diag(cudaStream_t s, const FlowView& F, const double* u, const double* v,
                 const double* w, const double* u0, const double* v0, const double* w0,
                 const double* p, RedBuf rb, StepScalars* out);
// out[q] = cell-centred component `comp` (3: pressure) at point xyz[3q..3q+2].
void launch_sample(cudaStream_t s, const FlowView& F, int comp, long long n, const double* xyz, const double* u,
                   const double* v, const double* w, const double* p, double* out);
void launch_max_inv(cudaStream_t s, const FlowView& F, const double* u, const double* v,
                    const double* w, double visc, double cfl, double* dt_out, RedBuf rb,
                    StepScalars* out);
// Layout conversion between the reference's lexicographic arrays and bricks.
// comp: 0 u, 1 v, 2 w, 3 cell. dir 0: lex -> brick, 1: brick -> lex.
void launch_convert(cudaStream_t s, const FlowView& F, int comp, int dir, const double* src,
                    double* dst);
void flow_kernel_setup();
long long lex_size(const FlowView& F, int comp);
long long store_size(const FlowView& F, int comp);

}  // namespace nb
