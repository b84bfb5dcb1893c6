// nb_noalloc.cu — the allocation-free variant of the -Laplacian launch.
//
// Who it is for: callers that cannot call cudaMalloc — hosts that own every
// byte of device memory through their own arena or admission budget (a
// serving process that has already handed its HBM to resident cases, an
// embedding application with its own pool allocator) and forbid libraries
// from allocating behind their back, or loops that must not stall on the
// allocator's implicit device synchronisation. They hold x and A x in their
// own device buffers; this entry point allocates nothing.
//
// The only scratch the kernel needs — the per-cell solid mask, which the
// caller describes with a host pointer in nb_grid_desc — lives in a
// file-scope static device array of NB_NOALLOC_MAX_CELLS bytes. The CUDA
// driver reserves it on every GPU that loads this library, until exit. All
// calls share it: each call overwrites the whole mask region it uses before
// the kernel reads it, so calls that overlap on the GPU (different streams,
// or different host threads on one device) race and must be serialised by
// the caller.
#include <mutex>

#include "nb_internal.h"

namespace {

static __device__ __align__(256) uint8_t g_noalloc_mask[NB_NOALLOC_MAX_CELLS];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
uint8_t* g_mask_ptr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_mask on the current device, looked up once per
// device (the host-side name is only a stand-in for the symbol).
cudaError_t mask_address(int device, uint8_t** out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_mask_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_mask);
    if (e != cudaSuccess) return e;
    g_mask_ptr[device] = static_cast<uint8_t*>(p);
  }
  *out = g_mask_ptr[device];
  return cudaSuccess;
}

// -Laplacian row on the lexicographic grid: same face resolution and the same
// accumulation order as the brick kernel (axis 0 side -1, +1, axis 1, axis 2),
// identity rows on solid cells (core/src/flow/poisson.cpp:18-134).
__global__ void k_apply_a_lex(int nx, int ny, int nz, int bc0, int bc1, int bc2, int bc3, int bc4,
                              int bc5, double h2x, double h2y, double h2z,
                              const uint8_t* __restrict__ solid, const double* __restrict__ x,
                              double* __restrict__ out) {
  const long long n = static_cast<long long>(nx) * ny * nz;
  const int bc[6] = {bc0, bc1, bc2, bc3, bc4, bc5};
  const double h2[3] = {h2x, h2y, h2z};
  const int dims[3] = {nx, ny, nz};
  for (long long m = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; m < n;
       m += static_cast<long long>(gridDim.x) * blockDim.x) {
    if (solid[m]) {
      out[m] = x[m];
      continue;
    }
    const int i = static_cast<int>(m % nx), j = static_cast<int>((m / nx) % ny),
              k = static_cast<int>(m / (static_cast<long long>(nx) * ny));
    double diag = 0.0, off = 0.0;
    for (int axis = 0; axis < 3; ++axis) {
      if (axis == 2 && nz == 1) continue;
      for (int side = -1; side <= 1; side += 2) {
        int c[3] = {i, j, k};
        c[axis] += side;
        if (c[axis] < 0 || c[axis] >= dims[axis]) {
          const int bt = bc[2 * axis + (side > 0 ? 1 : 0)];
          if (bt != NB_BC_PERIODIC) {
            if (bt == NB_BC_OUTLET) diag += 2.0 * h2[axis];
            continue;
          }
          c[axis] = (c[axis] + dims[axis]) % dims[axis];
        }
        const long long nn = c[0] + static_cast<long long>(nx) * (c[1] + static_cast<long long>(ny) * c[2]);
        if (solid[nn]) continue;
        diag += h2[axis];
        off += h2[axis] * x[nn];
      }
    }
    out[m] = diag * x[m] - off;
  }
}

}  // namespace

extern "C" nb_status nb_apply_laplacian_noalloc(const nb_grid_desc* grid, const double* x,
                                                double* out, void* stream) {
  if (!grid || !x || !out) return NB_ERR_BAD_ARG;
  if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || !(grid->dx > 0.0) || !(grid->dy > 0.0) ||
      !(grid->dz > 0.0))
    return NB_ERR_BAD_ARG;
  const unsigned long long n =
      static_cast<unsigned long long>(grid->nx) * grid->ny * grid->nz;
  if (n > NB_NOALLOC_MAX_CELLS) return NB_ERR_UNSUPPORTED;  // beyond the static scratch
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) {
    (void)cudaGetLastError();
    return NB_ERR_CUDA;
  }
  uint8_t* mask = nullptr;
  if (mask_address(device, &mask) != cudaSuccess) {
    (void)cudaGetLastError();
    return NB_ERR_CUDA;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The mask region is rewritten in full on every call (the array keeps the
  // previous call's contents otherwise).
  cudaError_t e = grid->solid ? cudaMemcpyAsync(mask, grid->solid, n, cudaMemcpyHostToDevice, s)
                              : cudaMemsetAsync(mask, 0, n, s);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return NB_ERR_CUDA;
  }
  const int threads = 256;
  const unsigned long long blocks = (n + threads - 1) / threads;
  const int grid_blocks = static_cast<int>(blocks < 148ull * 16 ? blocks : 148ull * 16);
  k_apply_a_lex<<<grid_blocks, threads, 0, s>>>(
      grid->nx, grid->ny, grid->nz, grid->face[0].type, grid->face[1].type, grid->face[2].type,
      grid->face[3].type, grid->face[4].type, grid->face[5].type, 1.0 / (grid->dx * grid->dx),
      1.0 / (grid->dy * grid->dy), 1.0 / (grid->dz * grid->dz), mask, x, out);
  // Peek, not get: an error the caller had not read yet stays pending for it.
  if (cudaPeekAtLastError() != cudaSuccess) return NB_ERR_CUDA;
  return NB_OK;
}
