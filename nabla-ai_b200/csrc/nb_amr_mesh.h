// nb_amr_mesh.h — the octree-AMR mesh object behind the C ABI.
#pragma once
#include <memory>

#include "nb_amr_level.h"
#include "nb_mg.cuh"

struct nb_amr_mesh {
  nb_ctx* ctx = nullptr;
  nb_amr_geom geom{};
  nb::AmrLevelHost lvl;                 // leaves, cell types, operator maps (MG level 0)
  std::unique_ptr<nb::MgSolver> mg[2];  // per precision, built on first use
};
