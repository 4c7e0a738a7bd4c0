// The stage kernel instantiations of the pair warp mapping (vt_tile.cuh).
#include "vt_stage_inst.cuh"

namespace vt {
StageKernel select_kernel_pair(int p, int nfq) { return stage_inst::select_for_map<kMapPair>(p, nfq); }
}  // namespace vt
