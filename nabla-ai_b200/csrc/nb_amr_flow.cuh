// nb_amr_flow.cuh — device view and launchers of the octree-AMR MAC step.
#pragma once
#include "nb_flow.cuh"
#include "nb_internal.h"

namespace nb {

struct AmrFlowView {
  LevelView L;  // composite level (amr = 1): per-level LUTs, bcoord, blevel, type
  double origin[3];
  double h[AMR_MAXLEV][3];
  double wallv[6][3];
  double inlet_speed[6];
  int profile[6];
  int inlet_axis[6];
  int per[3];
  long long nb;          // nbrick * 512 (slab base)
  const int* slab_id;    // [nbrick][3] slab index or -1
  const int8_t* rel_lo;  // [nbrick][3] REL_*
  const int8_t* rel_hi;
  const int* nbr_lo;     // [nbrick][3] same-level neighbour brick or -1
  const int* nbr_hi;
  int weno;
  double nu;
  double bf[3];
  // Ghost map of the momentum kernel (k_ghost_map); null: the walker serves
  // every halo point that the same-level fast path does not.
  const int* gm_off;    // [nbrick + 1] entry ranges
  const uint2* gm_ent;  // entries: point | component | term count, first term
  const int2* gm_term;  // terms: array index, FP32 weight bits
};

struct AmrStepScalars {
  double du2, div2, divmax, mass, maxinv;
};

void amr_flow_setup();
void launch_amr_rhs_rk(cudaStream_t s, const AmrFlowView& F, int stage, const double* dtp, const double* u,
                       const double* v, const double* w, const double* u0, const double* v0,
                       const double* w0, double* uo, double* vo, double* wo, int mixed, int grid_cap);
// Ghost map builder: pass 1 counts entries and terms per brick into count
// [2 nbrick]; pass 2 writes them at the scanned offsets eoff [nbrick],
// toff [nbrick].
void launch_ghost_count(cudaStream_t s, const AmrFlowView& F, int* count);
void launch_ghost_fill(cudaStream_t s, const AmrFlowView& F, const int* eoff, const int* toff, uint2* ent,
                       int2* term);
void launch_amr_sync(cudaStream_t s, const long long* list, int n, double* f);
void launch_amr_div(cudaStream_t s, const AmrFlowView& F, const double* u, const double* v, const double* w,
                    double* b);
void launch_amr_correct(cudaStream_t s, const AmrFlowView& F, const double* phi, const double* dtp,
                        double* u, double* v, double* w, double* p);
void launch_amr_diag(cudaStream_t s, const AmrFlowView& F, const double* u, const double* v,
                     const double* w, const double* u0, const double* v0, const double* w0, RedBuf rb,
                     AmrStepScalars* out);
// out[q] = cell-centred component `comp` (3: pressure) of the leaf cell containing xyz[3q..3q+2].
void launch_amr_sample(cudaStream_t s, const AmrFlowView& F, int comp, long long n, const double* xyz,
                       const double* u, const double* v, const double* w, const double* p, double* out);
// out[4 b .. 4 b + 3] = max |omega|, sqrt(2 S:S), Q, |grad p| over brick b's fluid cells.
void launch_amr_sensors(cudaStream_t s, const AmrFlowView& F, const double* u, const double* v, const double* w,
                        const double* p, double* out);
// Conservative state transfer from the mesh of view S to the mesh of view D.
void launch_amr_transfer(cudaStream_t s, const AmrFlowView& D, const AmrFlowView& S, const int* const dslab[3],
                         const long long nstore[3], const double* const fsrc[3], double* const fdst[3],
                         const double* psrc, double* pdst);
void launch_amr_max_inv(cudaStream_t s, const AmrFlowView& F, const double* u, const double* v,
                        const double* w, double cfl, double* dt_out, RedBuf rb, AmrStepScalars* out);

}  // namespace nb
