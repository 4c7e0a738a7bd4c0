// The stage kernel instantiations of the component warp mapping (vt_tile.cuh).
#include "vt_stage_inst.cuh"

namespace vt {
StageKernel select_kernel_component(int p, int nfq) { return stage_inst::select_for_map<kMapComponent>(p, nfq); }
}  // namespace vt
