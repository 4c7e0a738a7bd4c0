// The solver context behind the opaque vt_ctx handle, shared by the forward
// solver (vt_solver.cu) and the discrete adjoint (vt_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/vortex_b200.h"
#include "vt_launch.h"

namespace vt {
struct AdjointState;  // vt_adjoint.cu
}

struct vt_ctx {
  std::mutex mu;
  int device = 0, p = 0, Np = 0, nfq = 0, K = 0;
  long long Kpad = 0;
  int max_blocks = 0;  // persistent grid: SMs x resident blocks per SM
  cudaStream_t stream = nullptr;
  double2 *U = nullptr, *A = nullptr, *Sa = nullptr, *Sb = nullptr, *R = nullptr;
  double2* geo = nullptr;
  int4* nbr = nullptr;
  int4* tiles = nullptr;      // tile runs
  int* tile_items = nullptr;  // per-tile face lists
  int* tile_count = nullptr;
  int ntiles = 0;
  unsigned long long* err = nullptr;
  double2* aos = nullptr;
  double *W = nullptr, *partial = nullptr, *tot = nullptr;
  std::vector<double> ops;
  std::vector<double> minv_ref;  // Np x Np, for the projected initial condition
  vt::LaunchFn launch = nullptr;
  int map = vt::kDefaultMap;  // warp mapping of the stage kernel
  double time = 0.0;
  cudaGraphExec_t rk4_graph = nullptr;
  double rk4_graph_dt = 0.0;
  vt_error_info last{};
  int pending_steps = 0;
  double pending_dt = 0.0;
  bool side_pairing = false;  // nbr(nbr(e, s), s) == e for every element and side
  // Per-tile / per-element time steps (a batch group's view; null otherwise):
  // stage and adjoint coefficients are then fractions scaled on the device.
  const double* tile_dt = nullptr;
  const double* elem_dt = nullptr;
  vt::AdjointState* adj = nullptr;
  // vt_test_bulk_wait: the stage kernels' wait bound and test flags
  unsigned test_wait_tries = 0;
  int test_flags = 0;
};

namespace vt {

std::string cuda_msg(const char* what, cudaError_t e);

// Arguments of one stage launch on this context's mesh and schedule.
StageArgs stage_args(vt_ctx* c, const double2* in, const double2* base, double2* acc, double2* out, int stage,
                     double c_acc, double c_out);
// The four stage launches of one RK4 step of U in place (A, Sa, Sb scratch).
cudaError_t enqueue_rk4_step(vt_ctx* c, double dt);
// Clears the first-error key and the step counters.
cudaError_t reset_error_words(vt_ctx* c);
// Waits for the stream, decodes the first-error key, advances the clock by
// nsteps * dt and returns the status.
int finish(vt_ctx* c, int nsteps, double dt);
// Device AoS staging buffer (K x Np x 4 doubles), allocated on first use.
int ensure_aos(vt_ctx* c);
// AoS (K x Np x 4, device memory) <-> the SoA-of-double2 state layout.
cudaError_t aos_to_soa(vt_ctx* c, const double* src, double2* dst);
cudaError_t soa_to_aos(vt_ctx* c, const double2* src, double* dst);

// Frees the adjoint's buffers (no-op without them).
void adjoint_release(vt_ctx* c);
// Drops the adjoint's captured sweep graphs (after the stage kernel changed).
void adjoint_invalidate_graphs(vt_ctx* c);

}  // namespace vt
