// nb_maps.h — device-side octree maps and refinement used by the case API.
#pragma once
#include <cstdint>

#include "nb_internal.h"

struct nb_ctx;

namespace nb {

// Regrid refinement of a mesh on the device: leaves (4 int32 each, rank
// order, host) are split where sensors[4 r + which] > above (device array,
// rank order) and below lmax, 26-neighbour 2:1 balance is restored, and the
// new leaves are written to `out` (host) in rank order.
void refine_from_sensors(nb_ctx* ctx, cudaStream_t s, const nb_amr_geom& g, const int32_t* leaves, int n,
                         const double* d_sensors, int which, double above, int32_t* out, int64_t cap, int64_t* n_out);

}  // namespace nb
