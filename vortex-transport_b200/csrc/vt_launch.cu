// Instantiations of the tiled stage kernel for p = 0..3 and nfq = 1..10, and
// the tile schedule kernels (vt_launch.h).
#include <cstring>

#include "vt_launch.h"
#include "vt_schedule.cuh"
#include "vt_tile.cuh"

namespace vt {
namespace {

template <int P, int NFQ>
cudaError_t configure_stage(int* blocks_per_sm) {
  using Lay = TileLayout<P, NFQ>;
  cudaError_t e = cudaFuncSetAttribute(tile_stage_kernel<P, NFQ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       Lay::kBytes);
  if (e) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, tile_stage_kernel<P, NFQ>, 4 * kTileElems,
                                                       Lay::kBytes);
}

// Persistent launch: at most `max_blocks` blocks (SMs x resident blocks), each
// walking tiles blockIdx.x, blockIdx.x + gridDim.x, ...
template <int P, int NFQ>
cudaError_t launch_stage(const StageArgs& a, const double* ops, int max_blocks, cudaStream_t st) {
  using Lay = TileLayout<P, NFQ>;
  StageOps<P, NFQ> o;
  static_assert(sizeof(StageOps<P, NFQ>) % sizeof(double) == 0, "operator block is doubles");
  std::memcpy(&o, ops, sizeof(o));
  const int grid = a.ntiles < max_blocks ? a.ntiles : max_blocks;
  tile_stage_kernel<P, NFQ><<<grid, 4 * kTileElems, Lay::kBytes, st>>>(a, o);
  return cudaGetLastError();
}

template <int P, int NFQ>
StageKernel kernel_of() {
  return StageKernel{launch_stage<P, NFQ>, configure_stage<P, NFQ>};
}

template <int P>
StageKernel kernel_for_nfq(int nfq) {
  switch (nfq) {
    case 1: return kernel_of<P, 1>();
    case 2: return kernel_of<P, 2>();
    case 3: return kernel_of<P, 3>();
    case 4: return kernel_of<P, 4>();
    case 5: return kernel_of<P, 5>();
    case 6: return kernel_of<P, 6>();
    case 7: return kernel_of<P, 7>();
    case 8: return kernel_of<P, 8>();
    case 9: return kernel_of<P, 9>();
    case 10: return kernel_of<P, 10>();
    default: return StageKernel{};
  }
}

}  // namespace

StageKernel select_kernel(int p, int nfq) {
  switch (p) {
    case 0: return kernel_for_nfq<0>(nfq);
    case 1: return kernel_for_nfq<1>(nfq);
    case 2: return kernel_for_nfq<2>(nfq);
    case 3: return kernel_for_nfq<3>(nfq);
    default: return StageKernel{};
  }
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

cudaError_t launch_build_tile_items(const int4* tiles, const int4* nbr, int* items, int* count, int ntiles,
                                    cudaStream_t st) {
  build_tile_items_kernel<<<ntiles, 256, 0, st>>>(tiles, nbr, items, count);
  return cudaGetLastError();
}

}  // namespace vt
