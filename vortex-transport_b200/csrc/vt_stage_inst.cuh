// Launch and configuration of the tiled stage kernel for one warp mapping,
// instantiated for p = 0..3 and nfq = 1..10 by vt_stage_component.cu and
// vt_stage_pair.cu (one translation unit per mapping, compiled in parallel).
#pragma once

#include <cstring>

#include "vt_launch.h"
#include "vt_tile.cuh"

namespace vt {
namespace stage_inst {

template <int P, int NFQ, int MAP>
cudaError_t configure_stage(int* blocks_per_sm) {
  using Lay = TileLayout<P, NFQ>;
  cudaError_t e = cudaFuncSetAttribute(tile_stage_kernel<P, NFQ, MAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       Lay::kBytes);
  if (e) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, tile_stage_kernel<P, NFQ, MAP>,
                                                       4 * kTileElems, Lay::kBytes);
}

// Persistent launch: at most `max_blocks` blocks (SMs x resident blocks), each
// walking tiles blockIdx.x, blockIdx.x + gridDim.x, ...
template <int P, int NFQ, int MAP>
cudaError_t launch_stage(const StageArgs& a, const double* ops, int max_blocks, cudaStream_t st) {
  using Lay = TileLayout<P, NFQ>;
  StageOps<P, NFQ> o;
  static_assert(sizeof(StageOps<P, NFQ>) % sizeof(double) == 0, "operator block is doubles");
  std::memcpy(&o, ops, sizeof(o));
  const int grid = a.ntiles < max_blocks ? a.ntiles : max_blocks;
  // the tensor maps of this launch's state vectors (host-side encoding, no allocation)
  StageArgs k = a;
  constexpr int NP = np_of_p(P);
  cudaError_t e = encode_state_map(&k.map_in, a.in, a.Kpad, NP);
  if (!e) e = encode_state_map(&k.map_acc, a.acc, a.Kpad, NP);
  if (!e) e = encode_state_map(&k.map_base, a.base, a.Kpad, NP);
  if (e) return e;
  tile_stage_kernel<P, NFQ, MAP><<<grid, 4 * kTileElems, Lay::kBytes, st>>>(k, o);
  return cudaGetLastError();
}

template <int P, int NFQ, int MAP>
StageKernel kernel_of() {
  return StageKernel{launch_stage<P, NFQ, MAP>, configure_stage<P, NFQ, MAP>, MAP};
}

template <int P, int MAP>
StageKernel kernel_for_nfq(int nfq) {
  switch (nfq) {
    case 1: return kernel_of<P, 1, MAP>();
    case 2: return kernel_of<P, 2, MAP>();
    case 3: return kernel_of<P, 3, MAP>();
    case 4: return kernel_of<P, 4, MAP>();
    case 5: return kernel_of<P, 5, MAP>();
    case 6: return kernel_of<P, 6, MAP>();
    case 7: return kernel_of<P, 7, MAP>();
    case 8: return kernel_of<P, 8, MAP>();
    case 9: return kernel_of<P, 9, MAP>();
    case 10: return kernel_of<P, 10, MAP>();
    default: return StageKernel{};
  }
}

template <int MAP>
StageKernel select_for_map(int p, int nfq) {
  switch (p) {
    case 0: return kernel_for_nfq<0, MAP>(nfq);
    case 1: return kernel_for_nfq<1, MAP>(nfq);
    case 2: return kernel_for_nfq<2, MAP>(nfq);
    case 3: return kernel_for_nfq<3, MAP>(nfq);
    default: return StageKernel{};
  }
}

}  // namespace stage_inst
}  // namespace vt
