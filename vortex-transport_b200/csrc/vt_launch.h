// Dispatch to the stage kernel instantiation for (p, nfq), and the tile
// schedule builders; one translation unit (vt_launch.cu) instantiates them.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "vt_device.cuh"

namespace vt {

using LaunchFn = cudaError_t (*)(const StageArgs&, const double*, int, cudaStream_t);
using ConfigFn = cudaError_t (*)(int*);

struct StageKernel {
  // Launches one stage with at most `max_blocks` persistent blocks.
  LaunchFn launch = nullptr;
  // Sets the dynamic shared-memory attribute on the current device and
  // reports resident blocks per SM. Call before any launch or capture.
  ConfigFn configure = nullptr;
  // Warp mapping of the instantiation (kMapComponent or kMapPair, vt_tile.cuh).
  int map = 0;
};

// The mapping a context uses unless told otherwise (the pair mapping: 8% faster
// at p = 3 on the 768 x 768 mesh).
constexpr int kDefaultMap = kMapPair;

// Empty (null members) for p outside 0..3, nfq outside 1..10.
StageKernel select_kernel(int p, int nfq, int map = kDefaultMap);
StageKernel select_kernel_component(int p, int nfq);
StageKernel select_kernel_pair(int p, int nfq);

// Number of doubles of the StageOps<P, NFQ> block for (p, nfq).
int stage_ops_doubles(int p, int nfq);

// Writes the StageOps<P, NFQ> block (stage_ops_doubles(p, nfq) doubles) into
// `ops`: M_ref^-1 folded into the volume operators (D = M_ref^-1 S_xi, S_eta)
// and the lift (M_ref^-1 phi+_s w), with long-double accumulation, and the own /
// neighbour face tables restricted to each side's p + 1 nodes. The inputs are
// the reference-space tables of vt_mesh_desc (Preevolve.cpp:15-144,
// Evolve.cpp:76-132). Host only; allocates nothing.
void fold_stage_operators(int p, int nfq, const double* minv, const double* stiff, const double* line,
                          const double* phi_plus, const double* phi_minus, double* ops);

// Two-row tiles for the reference's structured mesh, empty if `conn` is not it.
std::vector<int4> structured_tile_runs(int K, const int32_t* type, const int32_t* conn);
// The same runs from the grid size alone (empty unless nx, ny suit them).
std::vector<int4> grid_tile_runs(int nx, int ny);

// Encodes the 2-D tensor map of a state vector for the stage kernel's tensor
// copies: [2 Np rows] x [2 Kpad doubles], box of 2 Np rows x 64 doubles (one
// run of 32 elements). Host only; a pure encoding (cuTensorMapEncodeTiled,
// reached through the runtime's driver entry point), no allocation.
cudaError_t encode_state_map(CUtensorMap* map, const void* base, long long Kpad, int Np);
// cudaSuccess when the driver provides the tensor-map encoder (looked up once;
// call before any stream capture).
cudaError_t tensor_maps_available();

// Device-side: tiles of 64 consecutive elements, then the per-tile face lists.
cudaError_t launch_contiguous_tiles(int4* tiles, int K, int ntiles, cudaStream_t st);
// nfq decides where the face items that read global memory are placed (vt_schedule.cuh).
cudaError_t launch_build_tile_items(const int4* tiles, const int4* nbr, int* items, int* count, int ntiles, int nfq,
                                    cudaStream_t st);

}  // namespace vt
