// Kernel selection by (p, nfq, warp mapping) -- the instantiations are in
// vt_stage_component.cu and vt_stage_pair.cu -- and the tile schedule kernels
// (vt_launch.h).
#include <cuda.h>

#include <cstring>
#include <mutex>

#include "vt_launch.h"
#include "vt_schedule.cuh"

namespace vt {

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

}  // namespace

cudaError_t tensor_maps_available() { return encode_tiled() ? cudaSuccess : cudaErrorNotSupported; }

// Tensor map of one SoA state vector: [2 Np rows] x [2 Kpad doubles], a box of
// one 32-element run. No L2 promotion: a box row is 512 contiguous bytes, whole
// sectors already (promotion to 256-byte lines was 0.2% slower at 768 x 768).
cudaError_t encode_state_map(CUtensorMap* m, const void* base, long long Kpad, int Np) {
  const EncodeTiledFn fn = encode_tiled();
  if (!fn) return cudaErrorNotSupported;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(2 * Kpad), static_cast<cuuint64_t>(2 * Np)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(2 * Kpad * sizeof(double))};
  const cuuint32_t box[2] = {2 * kTileRun, static_cast<cuuint32_t>(2 * Np)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

StageKernel select_kernel(int p, int nfq, int map) {
  return map == kMapPair ? select_kernel_pair(p, nfq) : select_kernel_component(p, nfq);
}

int stage_ops_doubles(int p, int nfq) {
  const int np = np_of_p(p), ne = p + 1;
  return 2 * np * np + 3 * np * nfq + 6 * nfq * ne;
}

void fold_stage_operators(int p, int nfq, const double* minv, const double* stiff, const double* line,
                          const double* phi_plus, const double* phi_minus, double* ops) {
  const int Np = np_of_p(p), NE = p + 1;
  int o = 0;
  for (int d = 0; d < 2; ++d)
    for (int i = 0; i < Np; ++i)
      for (int j = 0; j < Np; ++j) {
        long double s = 0;
        for (int k = 0; k < Np; ++k) s += static_cast<long double>(minv[i * Np + k]) * stiff[(d * Np + k) * Np + j];
        ops[o++] = static_cast<double>(s);
      }
  for (int sd = 0; sd < 3; ++sd)
    for (int i = 0; i < Np; ++i)
      for (int q = 0; q < nfq; ++q) {
        long double s = 0;
        for (int j = 0; j < Np; ++j) s += static_cast<long double>(minv[i * Np + j]) * phi_plus[(sd * Np + j) * nfq + q];
        ops[o++] = static_cast<double>(s * line[2 * q + 1]);
      }
  for (int sd = 0; sd < 3; ++sd)
    for (int q = 0; q < nfq; ++q)
      for (int k = 0; k < NE; ++k) ops[o++] = phi_plus[(sd * Np + edge_node(p, sd, k)) * nfq + q];
  for (int sd = 0; sd < 3; ++sd)
    for (int q = 0; q < nfq; ++q)
      for (int k = 0; k < NE; ++k) ops[o++] = phi_minus[(sd * Np + edge_node(p, sd, k)) * nfq + q];
}

std::vector<int4> structured_tile_runs(int K, const int32_t* type, const int32_t* conn) {
  return structured_tiles(K, type, conn);
}

std::vector<int4> grid_tile_runs(int nx, int ny) { return grid_tiles(nx, ny); }

cudaError_t launch_contiguous_tiles(int4* tiles, int K, int ntiles, cudaStream_t st) {
  contiguous_tiles_kernel<<<(ntiles + 255) / 256, 256, 0, st>>>(tiles, K, ntiles);
  return cudaGetLastError();
}

cudaError_t launch_build_tile_items(const int4* tiles, const int4* nbr, int* items, int* count, int ntiles, int nfq,
                                    cudaStream_t st) {
  build_tile_items_kernel<<<ntiles, 256, 0, st>>>(tiles, nbr, items, count, nfq);
  return cudaGetLastError();
}

}  // namespace vt
