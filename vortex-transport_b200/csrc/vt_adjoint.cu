// Discrete adjoint of the RK4 stepper, its tangent-linear model and the
// checkpointed reverse sweep (C ABI in include/vortex_b200.h, "discrete adjoint").
//
// Forward sweep: the plain RK4 step (the stage kernel of vt_step_rk4, launched
// on explicit buffers) advances between checkpoint slots as the binomial plan
// of vt_checkpoint.h says, or, when the snapshot budget holds four states per
// step, writes every step's start and stage states to their own buffers.
// Reverse sweep, per step i = n-1 .. 0: (binomial plan) rerun step i from its
// checkpoint keeping the stage states U1, U2, U3; then four reverse stages
// (adjoint_tile_kernel each on meshes whose faces take the edge-once form,
// else a face phase + adjoint_element_kernel) turn the adjoint of U_{i+1} into
// the adjoint of U_i:
//   a4 = dt/6 lam                 g4 = R'(U3)^T a4
//   a3 = dt/3 lam + dt   g4       g3 = R'(U2)^T a3
//   a2 = dt/3 lam + dt/2 g3       g2 = R'(U1)^T a2
//   a1 = dt/6 lam + dt/2 g2       g1 = R'(U_i)^T a1
//   lam <- lam + g4 + g3 + g2 + g1
// with the coefficients the forward stages use (Timestepping.cpp:128-305).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/vortex_b200.h"
#include "vt_adjoint_kernels.cuh"
#include "vt_adjoint_tile.cuh"
#include "vt_checkpoint.h"
#include "vt_common.h"
#include "vt_ctx.h"

namespace vt {
namespace {

using FaceFn = cudaError_t (*)(const AdjArgs&, const double*, cudaStream_t);
using TileFn = cudaError_t (*)(const AdjArgs&, const double*, int, cudaStream_t);
using TileConfigFn = cudaError_t (*)(int*);
using JvpFn = cudaError_t (*)(const double2*, const double2*, double2*, const double2*, const int4*, long long,
                              int, const double*, cudaStream_t);

struct AdjKernels {
  FaceFn face = nullptr;
  FaceFn element = nullptr;
  JvpFn jvp = nullptr;
  TileFn tile = nullptr;
  TileConfigFn tile_config = nullptr;
};

template <int P, int NFQ>
cudaError_t launch_face(const AdjArgs& a, const double* ops, cudaStream_t st) {
  StageOps<P, NFQ> o;
  std::memcpy(&o, ops, sizeof(o));
  const dim3 grid((a.K + kAdjRun - 1) / kAdjRun, 3), block(kAdjRun, NFQ);
  adjoint_face_kernel<P, NFQ><<<grid, block, 0, st>>>(a, o);
  return cudaGetLastError();
}

template <int P, int NFQ>
cudaError_t launch_element(const AdjArgs& a, const double* ops, cudaStream_t st) {
  StageOps<P, NFQ> o;
  std::memcpy(&o, ops, sizeof(o));
  const dim3 grid((a.K + kAdjRun - 1) / kAdjRun), block(kAdjRun, np_of_p(P));
  adjoint_element_kernel<P, NFQ><<<grid, block, 0, st>>>(a, o);
  return cudaGetLastError();
}

// One reverse stage as one persistent launch over the stage kernel's tiles.
template <int P, int NFQ>
cudaError_t launch_tile(const AdjArgs& a, const double* ops, int max_blocks, cudaStream_t st) {
  StageOps<P, NFQ> o;
  std::memcpy(&o, ops, sizeof(o));
  const int grid = a.ntiles < max_blocks ? a.ntiles : max_blocks;
  // the tensor maps of this launch's stage state and stage adjoint (host-side encoding, no allocation)
  AdjArgs k = a;
  cudaError_t e = encode_state_map(&k.map_U, a.U, a.Kpad, np_of_p(P));
  if (!e) e = encode_state_map(&k.map_a, a.a, a.Kpad, np_of_p(P));
  if (e) return e;
  adjoint_tile_kernel<P, NFQ><<<grid, 4 * kTileElems, AdjTileLayout<P, NFQ>::kBytes, st>>>(k, o);
  return cudaGetLastError();
}

template <int P, int NFQ>
cudaError_t configure_tile(int* blocks_per_sm) {
  constexpr int bytes = AdjTileLayout<P, NFQ>::kBytes;
  cudaError_t e = cudaFuncSetAttribute(adjoint_tile_kernel<P, NFQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, adjoint_tile_kernel<P, NFQ>, 4 * kTileElems,
                                                       bytes);
}

template <int P, int NFQ>
cudaError_t launch_jvp(const double2* U, const double2* V, double2* dR, const double2* geo, const int4* nbr,
                       long long KP, int K, const double* ops, cudaStream_t st) {
  StageOps<P, NFQ> o;
  std::memcpy(&o, ops, sizeof(o));
  rhs_jvp_kernel<P, NFQ><<<(K + 127) / 128, 128, 0, st>>>(U, V, dR, geo, nbr, KP, K, o);
  return cudaGetLastError();
}

template <int P, int NFQ>
AdjKernels kernels_of() {
  return AdjKernels{launch_face<P, NFQ>, launch_element<P, NFQ>, launch_jvp<P, NFQ>, launch_tile<P, NFQ>,
                    configure_tile<P, NFQ>};
}

template <int P>
AdjKernels kernels_for_nfq(int nfq) {
  switch (nfq) {
    case 1: return kernels_of<P, 1>();
    case 2: return kernels_of<P, 2>();
    case 3: return kernels_of<P, 3>();
    case 4: return kernels_of<P, 4>();
    case 5: return kernels_of<P, 5>();
    case 6: return kernels_of<P, 6>();
    case 7: return kernels_of<P, 7>();
    case 8: return kernels_of<P, 8>();
    case 9: return kernels_of<P, 9>();
    case 10: return kernels_of<P, 10>();
    default: return AdjKernels{};
  }
}

AdjKernels select_adjoint(int p, int nfq) {
  switch (p) {
    case 0: return kernels_for_nfq<0>(nfq);
    case 1: return kernels_for_nfq<1>(nfq);
    case 2: return kernels_for_nfq<2>(nfq);
    case 3: return kernels_for_nfq<3>(nfq);
    default: return AdjKernels{};
  }
}

}  // namespace

// A sweep's launches depend only on its buffers, step count and time step, so
// a repeated sweep replays a captured CUDA graph instead of relaunching.
struct SweepGraph {
  cudaGraphExec_t exec = nullptr;
  std::vector<long long> key;
  void reset() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    key.clear();
  }
};

// The overlapped reverse sweep (run_plan_overlapped) renames the checkpoint
// slots onto the plan's slots, the work slot and kSpareSlots spare state
// buffers, and orders its two streams through a ring of kRevRing events, one
// recorded after each reverse step.
constexpr int kSpareSlots = 2;
constexpr int kRevRing = 8;

struct AdjointState {
  AdjKernels k;
  SweepGraph fwd_graph, bwd_graph;
  size_t state_elems = 0;  // double2 entries of one state vector
  // work, stage states, adjoint, accumulator, two stage adjoints, second set
  // of stage states (contiguous)
  double2* bufs = nullptr;
  double2 *work = nullptr, *s1 = nullptr, *s2 = nullptr, *s3 = nullptr;
  double2 *lam = nullptr, *acc = nullptr, *a0 = nullptr, *a1 = nullptr;
  double2 *t1 = nullptr, *t2 = nullptr, *t3 = nullptr;
  // the reverse sweep's recomputation runs on `side`, ahead of the reverse
  // steps on the context's stream (run_plan_overlapped)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_ready[2] = {nullptr, nullptr};
  cudaEvent_t ev_rev[kRevRing] = {};
  double2 *bp = nullptr, *bm = nullptr;  // face adjoints of the two-launch form (else null)
  // fused reverse stage (adjoint_tile_kernel): persistent grid size, 0 when
  // the edge-once form does not apply (the element adjacency does not
  // 2-colour) or the kernel cannot be resident
  int tile_blocks = 0;
  double2* slots = nullptr;
  long long nslots = 0;
  int plan_slots = 0;  // checkpoint slots the plan uses (the spares follow them)
  // last forward sweep
  std::vector<CkptAction> plan;
  size_t first_adjoint = 0;
  double dt = 0.0;
  int nsteps = 0;
  bool have_forward = false;
  bool all_stages = false;  // every step's start and stage states are kept in slots 4i .. 4i+3
  bool fresh = false;  // the forward sweep's checkpoints and stage states are intact
  vt_checkpoint_info info{};
};

namespace {

void release_streams(AdjointState* s) {
  cudaEvent_t evs[4] = {s->ev_fork, s->ev_join, s->ev_ready[0], s->ev_ready[1]};
  for (cudaEvent_t ev : evs)
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : s->ev_rev)
    if (ev) cudaEventDestroy(ev);
  if (s->side) cudaStreamDestroy(s->side);
  s->side = nullptr;
}

int setup(vt_ctx* c) {
  if (c->adj) return VT_OK;
  if (!c->side_pairing)
    return fail(VT_ERR_UNSUPPORTED, "adjoint: side s of some element does not face side s of its neighbour");
  const AdjKernels k = select_adjoint(c->p, c->nfq);
  if (!k.face) return fail(VT_ERR_UNSUPPORTED, "adjoint: unsupported (p, nfq)");
  // The edge-once form needs every edge to join elements whose sides face each
  // other with opposite normals; a 2-colouring of the element adjacency
  // (breadth first) tells such meshes (the reference's type-0 / type-1
  // triangles) from ones with self-neighbours or odd cycles.
  std::vector<int4> nb(static_cast<size_t>(c->K));
  cudaError_t e = cudaMemcpy(nb.data(), c->nbr, sizeof(int4) * nb.size(), cudaMemcpyDeviceToHost);
  if (e) return fail(VT_ERR_CUDA, cuda_msg("adjoint: neighbours", e));
  std::vector<signed char> col(nb.size(), -1);
  std::vector<int> queue;
  bool ok = true;
  for (int start = 0; start < c->K && ok; ++start) {
    if (col[start] >= 0) continue;
    col[start] = 0;
    queue.assign(1, start);
    for (size_t h = 0; h < queue.size() && ok; ++h) {
      const int x = queue[h];
      const int side[3] = {nb[x].x, nb[x].y, nb[x].z};
      for (int n : side) {
        if (col[n] < 0) {
          col[n] = static_cast<signed char>(1 - col[x]);
          queue.push_back(n);
        } else if (col[n] == col[x]) {
          ok = false;
        }
      }
    }
  }
  // the fused reverse stage runs on the stage kernel's tiles
  int tile_blocks = 0;
  if (ok) {
    int per_sm = 0, sms = 0;
    if (c->tiles && c->ntiles > 0 && !k.tile_config(&per_sm) &&
        !cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device) && per_sm > 0)
      tile_blocks = sms * per_sm;
    cudaGetLastError();
  }
  // eleven state vectors, plus the face adjoints of the two-launch form when
  // that form is the one used
  constexpr int kVectors = 11;
  const size_t state_elems = static_cast<size_t>(2 * c->Np) * static_cast<size_t>(c->Kpad);
  const size_t face_elems = tile_blocks > 0 ? 0 : static_cast<size_t>(6 * c->nfq) * static_cast<size_t>(c->Kpad);
  const size_t total = kVectors * state_elems + 2 * face_elems;
  double2* bufs = nullptr;
  e = cudaMalloc(reinterpret_cast<void**>(&bufs), sizeof(double2) * total);
  if (!e) e = cudaMemsetAsync(bufs, 0, sizeof(double2) * total, c->stream);
  if (e) {
    if (bufs) cudaFree(bufs);
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? VT_ERR_NO_MEMORY : VT_ERR_CUDA, cuda_msg("adjoint buffers", e));
  }
  auto* s = new AdjointState();
  e = cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking);
  cudaEvent_t* evs[4 + kRevRing] = {&s->ev_fork, &s->ev_join, &s->ev_ready[0], &s->ev_ready[1]};
  for (int i = 0; i < kRevRing; ++i) evs[4 + i] = &s->ev_rev[i];
  for (int i = 0; i < 4 + kRevRing && !e; ++i) e = cudaEventCreateWithFlags(evs[i], cudaEventDisableTiming);
  if (e) {
    cudaGetLastError();
    release_streams(s);
    delete s;
    cudaFree(bufs);
    return fail(VT_ERR_CUDA, cuda_msg("adjoint streams", e));
  }
  s->k = k;
  s->tile_blocks = tile_blocks;
  s->state_elems = state_elems;
  s->bufs = bufs;
  double2** named[kVectors] = {&s->work, &s->s1, &s->s2, &s->s3, &s->lam, &s->acc,
                                &s->a0,   &s->a1, &s->t1, &s->t2, &s->t3};
  for (int i = 0; i < kVectors; ++i) *named[i] = s->bufs + i * s->state_elems;
  if (face_elems) {
    s->bp = s->bufs + kVectors * s->state_elems;
    s->bm = s->bp + face_elems;
  }
  c->adj = s;
  return VT_OK;
}

int ensure_slots(vt_ctx* c, long long n) {
  AdjointState* s = c->adj;
  if (s->nslots >= n) return VT_OK;
  if (s->slots) cudaFree(s->slots);
  s->slots = nullptr;
  s->nslots = 0;
  const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&s->slots), sizeof(double2) * s->state_elems * n);
  if (e) {
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? VT_ERR_NO_MEMORY : VT_ERR_CUDA,
                cuda_msg(("adjoint: " + std::to_string(n) + " checkpoint states").c_str(), e));
  }
  s->nslots = n;
  return VT_OK;
}

double2* slot(vt_ctx* c, long long i) {
  return i == kWorkSlot ? c->adj->work : c->adj->slots + static_cast<size_t>(i) * c->adj->state_elems;
}

cudaError_t stage(vt_ctx* c, const double2* in, const double2* base, double2* out, int st, double ca, double co,
                  cudaStream_t stream, bool no_acc = false) {
  StageArgs a = stage_args(c, in, base, c->A, out, st, ca, co);
  a.no_acc = no_acc ? 1 : 0;
  return c->launch(a, c->ops.data(), c->max_blocks, stream);
}

// The step size the coefficients carry: dt, or 1 when the device scales them
// by each tile's / element's own time step (a batch group).
double dt_scale(const vt_ctx* c, double dt) { return c->tile_dt ? 1.0 : dt; }

// One plain RK4 step from X into Y (Y may be X), stages through Sa, Sb.
cudaError_t plain_step(vt_ctx* c, const double2* X, double2* Y, double dt0, cudaStream_t st) {
  const double dt = dt_scale(c, dt0);
  cudaError_t e;
  if ((e = stage(c, X, X, c->Sa, 0, (1.0 / 6) * dt, 0.5 * dt, st))) return e;
  if ((e = stage(c, c->Sa, X, c->Sb, 1, (1.0 / 3) * dt, 0.5 * dt, st))) return e;
  if ((e = stage(c, c->Sb, X, c->Sa, 2, (1.0 / 3) * dt, dt, st))) return e;
  return stage(c, c->Sa, X, Y, 3, 0.0, (1.0 / 6) * dt, st);
}

cudaError_t advance(vt_ctx* c, const double2* X, int k, double2* Y, double dt, cudaStream_t st) {
  cudaError_t e = plain_step(c, X, Y, dt, st);
  for (int i = 1; i < k && !e; ++i) e = plain_step(c, Y, Y, dt, st);
  return e;
}

// Step from X keeping the stage states in S1, S2, S3; the new state goes to
// `out` when given (else the last stage is not run). With no_acc (only when
// no last stage will follow on this accumulator: the reverse sweeps' reruns)
// stage 1 does not form the accumulator (stages 0 and 2 never touch it).
cudaError_t stage_step(vt_ctx* c, const double2* X, double2* S1, double2* S2, double2* S3, double dt0,
                       double2* out, cudaStream_t st, bool no_acc = false) {
  const double dt = dt_scale(c, dt0);
  cudaError_t e;
  if ((e = stage(c, X, X, S1, 0, (1.0 / 6) * dt, 0.5 * dt, st, no_acc))) return e;
  if ((e = stage(c, S1, X, S2, 1, (1.0 / 3) * dt, 0.5 * dt, st, no_acc))) return e;
  if ((e = stage(c, S2, X, S3, 2, (1.0 / 3) * dt, dt, st, no_acc))) return e;
  return out ? stage(c, S3, X, out, 3, 0.0, (1.0 / 6) * dt, st) : cudaSuccess;
}

cudaError_t stage_step(vt_ctx* c, const double2* X, double dt, double2* out, bool no_acc = false) {
  return stage_step(c, X, c->adj->s1, c->adj->s2, c->adj->s3, dt, out, c->stream, no_acc);
}

AdjArgs adj_args(vt_ctx* c) {
  AdjArgs a{};
  a.bp = c->adj->bp;
  a.bm = c->adj->bm;
  a.elem_dt = c->elem_dt;
  a.geo = c->geo;
  a.nbr = c->nbr;
  a.tiles = c->tiles;
  a.tile_items = c->tile_items;
  a.tile_count = c->tile_count;
  a.ntiles = c->ntiles;
  a.err = c->err;
  a.Kpad = c->Kpad;
  a.K = c->K;
  a.sa = 1.0;
  return a;
}

// One reverse stage: the fused tile kernel where the face phase may take the
// edge-once form, else the two-sided face phase and the element kernel (exact
// on any mesh whose sides pair up).
cudaError_t reverse_stage(vt_ctx* c, const AdjArgs& a) {
  AdjointState* s = c->adj;
  if (s->tile_blocks > 0) return s->k.tile(a, c->ops.data(), s->tile_blocks, c->stream);
  const cudaError_t e = s->k.face(a, c->ops.data(), c->stream);
  return e ? e : s->k.element(a, c->ops.data(), c->stream);
}

// lam <- adjoint of U_i given lam = adjoint of U_{i+1}; X = U_i, stage states S1..S3.
cudaError_t adjoint_step(vt_ctx* c, const double2* X, const double2* S1, const double2* S2, const double2* S3,
                         double dt0) {
  AdjointState* s = c->adj;
  const double dt = dt_scale(c, dt0);
  AdjArgs a = adj_args(c);
  cudaError_t e;
  a.U = S3, a.a = s->lam, a.sa = (1.0 / 6) * dt, a.sa_dt = 1, a.lam = s->lam, a.acc_in = nullptr, a.lam_coef = 1.0;
  a.acc_out = s->acc, a.a_out = s->a1, a.cl = (1.0 / 3) * dt, a.cg = dt;
  if ((e = reverse_stage(c, a))) return e;
  a.U = S2, a.a = s->a1, a.sa = 1.0, a.sa_dt = 0, a.acc_in = s->acc, a.lam_coef = 0.0;
  a.acc_out = s->acc, a.a_out = s->a0, a.cl = (1.0 / 3) * dt, a.cg = 0.5 * dt;
  if ((e = reverse_stage(c, a))) return e;
  a.U = S1, a.a = s->a0, a.a_out = s->a1, a.cl = (1.0 / 6) * dt, a.cg = 0.5 * dt;
  if ((e = reverse_stage(c, a))) return e;
  a.U = X, a.a = s->a1, a.lam = nullptr, a.acc_out = s->lam, a.a_out = nullptr, a.cl = 0.0, a.cg = 0.0;
  return reverse_stage(c, a);
}

// Runs plan[begin, end). `out_last` receives the new state of the plan's first
// stage step (the forward sweep's last step), or null to skip that stage.
cudaError_t run_plan(vt_ctx* c, size_t begin, size_t end, double2* out_last) {
  AdjointState* s = c->adj;
  cudaError_t e = cudaSuccess;
  for (size_t i = begin; i < end && !e; ++i) {
    const CkptAction& a = s->plan[i];
    switch (a.op) {
      case CkptOp::kAdvance: e = advance(c, slot(c, a.src), a.steps, slot(c, a.dst), s->dt, c->stream); break;
      case CkptOp::kStageStep: {
        // the forward sweep's last step runs its last stage into out_last;
        // every other rerun only keeps its stage states
        double2* out = a.step == s->nsteps - 1 ? out_last : nullptr;
        e = stage_step(c, slot(c, a.src), s->dt, out, out == nullptr);
        break;
      }
      case CkptOp::kAdjoint: e = adjoint_step(c, slot(c, a.src), s->s1, s->s2, s->s3, s->dt); break;
    }
  }
  return e;
}

// Runs plan[begin, end) of a reverse sweep with the recomputation ahead of it:
// advances and stage steps go to the side stream R, reverse steps stay on the
// context's stream M, and the stage states alternate between two sets, so that
// the recomputation of the next steps overlaps the reverse steps (at small
// sizes neither kernel fills the GPU; a tile kernel's last round of tiles
// leaves most SMs idle). Both streams run the launches of run_plan on the same
// states, so the results are identical.
//
// Write-after-read hazards: a stage step waits until the reverse step that
// read the set it overwrites is done. An advance must not overwrite a state
// that a reverse step issued before it still reads; in the binomial plan the
// next advance after a segment's reversal writes the very slot that segment's
// last reverse step reads (the slot it just released), so waiting there would
// leave M idle for the whole advance. Instead the logical slots are renamed
// onto physical buffers (the plan's slots, the work slot and kSpareSlots
// spares): an advance whose target buffer still has a reader in flight writes
// the spare read longest ago, which takes over the logical slot, and the old
// buffer becomes a spare (schedule_overlapped, vt_checkpoint.cpp, makes these
// decisions on the host; a CPU test checks them on whole plans). R waits on a
// ring of per-reverse-step events (recorded on M after each reverse step) only
// when the buffer it is about to write has a reader that R has not yet waited
// for; a ring entry recorded again by a later reverse step only makes a wait
// stronger, since M runs in order.
// Reads of the renamed slots (advances, stage steps, reverse steps) follow the
// mapping at their place in the plan, which every replay of the captured graph
// repeats from the same identity mapping (the forward part writes the
// checkpoints to the plan's own slots). Must be called inside a stream capture
// of the context's stream; set 0 (s1..s3) holds the stage states of the plan's
// first reverse step on entry.
cudaError_t run_plan_overlapped(vt_ctx* c, size_t begin, size_t end) {
  AdjointState* s = c->adj;
  cudaStream_t M = c->stream, R = s->side;
  double2* const sets[2][3] = {{s->s1, s->s2, s->s3}, {s->t1, s->t2, s->t3}};
  bool ready_rec[2] = {false, false};  // ev_ready[k] recorded in this capture
  // physical buffers: the plan's slots 0..nlog-1, the work slot (nlog), the spares
  const int nlog = s->plan_slots;
  std::vector<double2*> buf;
  for (int i = 0; i < nlog; ++i) buf.push_back(slot(c, i));
  buf.push_back(s->work);
  for (int i = 0; i < kSpareSlots; ++i) buf.push_back(slot(c, nlog + i));
  const std::vector<OverlapStep> sched = schedule_overlapped(s->plan, begin, end, nlog, kSpareSlots);
  cudaError_t e = cudaEventRecord(s->ev_fork, M);
  if (!e) e = cudaStreamWaitEvent(R, s->ev_fork, 0);
  for (size_t i = 0; i < sched.size() && !e; ++i) {
    const OverlapStep& x = sched[i];
    if (x.wait >= 0) e = cudaStreamWaitEvent(R, s->ev_rev[x.wait % kRevRing], 0);
    if (e) break;
    switch (x.op) {
      case CkptOp::kAdvance: e = advance(c, buf[x.src], x.steps, buf[x.dst], s->dt, R); break;
      case CkptOp::kStageStep:
        e = stage_step(c, buf[x.src], sets[x.set][0], sets[x.set][1], sets[x.set][2], s->dt, nullptr, R, true);
        if (!e) e = cudaEventRecord(s->ev_ready[x.set], R);
        ready_rec[x.set] = true;
        break;
      case CkptOp::kAdjoint:
        if (ready_rec[x.set]) e = cudaStreamWaitEvent(M, s->ev_ready[x.set], 0);
        if (!e) e = adjoint_step(c, buf[x.src], sets[x.set][0], sets[x.set][1], sets[x.set][2], s->dt);
        if (!e) e = cudaEventRecord(s->ev_rev[x.index % kRevRing], M);
        break;
    }
  }
  // the side stream rejoins the capture's origin stream
  const cudaError_t j = cudaEventRecord(s->ev_join, R);
  const cudaError_t k = j ? j : cudaStreamWaitEvent(M, s->ev_join, 0);
  return e ? e : k;
}

// Host or device AoS array -> SoA buffer on the context's stream.
cudaError_t load_aos(vt_ctx* c, const double* src, int device_pointers, double2* dst) {
  if (device_pointers) return aos_to_soa(c, src, dst);
  cudaError_t e = cudaMemcpyAsync(c->aos, src, sizeof(double) * 4 * static_cast<size_t>(c->K) * c->Np,
                                  cudaMemcpyHostToDevice, c->stream);
  return e ? e : aos_to_soa(c, reinterpret_cast<const double*>(c->aos), dst);
}

cudaError_t store_aos(vt_ctx* c, const double2* src, double* dst, int device_pointers) {
  if (device_pointers) return soa_to_aos(c, src, dst);
  cudaError_t e = soa_to_aos(c, src, reinterpret_cast<double*>(c->aos));
  if (!e)
    e = cudaMemcpyAsync(dst, c->aos, sizeof(double) * 4 * static_cast<size_t>(c->K) * c->Np, cudaMemcpyDeviceToHost,
                        c->stream);
  return e;
}

cudaError_t lincomb(vt_ctx* c, double2* out, const double2* x, double cx, const double2* y, double cy,
                    const double2* z = nullptr, double cz = 0.0) {
  const long long n = static_cast<long long>(c->adj->state_elems);
  lincomb_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, c->stream>>>(out, x, cx, y, cy, z, cz, n);
  return cudaGetLastError();
}

template <typename F>
cudaError_t run_captured(vt_ctx* c, SweepGraph& g, const std::vector<long long>& key, F&& enqueue) {
  if (!g.exec || g.key != key) {
    g.reset();
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    if (e) return e;
    const cudaError_t le = enqueue();
    e = cudaStreamEndCapture(c->stream, &graph);
    if (le) e = le;
    if (!e) e = cudaGraphInstantiate(&g.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e) {
      g.reset();
      return e;
    }
    g.key = key;
  }
  return cudaGraphLaunch(g.exec, c->stream);
}

std::vector<long long> sweep_key(vt_ctx* c, int kind) {
  const AdjointState* s = c->adj;
  long long dt_bits = 0;
  std::memcpy(&dt_bits, &s->dt, sizeof(dt_bits));
  return {kind, s->nsteps, dt_bits, s->all_stages, reinterpret_cast<long long>(s->slots), s->nslots,
          reinterpret_cast<long long>(c->U), reinterpret_cast<long long>(s->bufs),
          static_cast<long long>(s->first_adjoint), static_cast<long long>(s->plan.size())};
}

int prepare(vt_ctx* c) {
  int st = setup(c);
  if (!st) st = ensure_aos(c);
  return st;
}

}  // namespace

void adjoint_invalidate_graphs(vt_ctx* c) {
  if (!c || !c->adj) return;
  c->adj->fwd_graph.reset();
  c->adj->bwd_graph.reset();
}

void adjoint_release(vt_ctx* c) {
  if (!c || !c->adj) return;
  c->adj->fwd_graph.reset();
  c->adj->bwd_graph.reset();
  if (c->adj->slots) cudaFree(c->adj->slots);
  if (c->adj->bufs) cudaFree(c->adj->bufs);
  release_streams(c->adj);
  delete c->adj;
  c->adj = nullptr;
}

}  // namespace vt

using vt::fail;

extern "C" {

int vt_adjoint_forward(vt_ctx* c, double dt, int nsteps, int nsnapshots) {
  if (!c || nsteps < 1 || nsnapshots < 1) return fail(VT_ERR_INVALID, "vt_adjoint_forward: bad argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (c->pending_steps) return fail(VT_ERR_INVALID, "a previous async step is not synchronised");
  int st = vt::prepare(c);
  if (st) return st;
  vt::AdjointState* s = c->adj;
  s->have_forward = s->fresh = false;
  s->dt = dt;
  s->nsteps = nsteps;
  s->all_stages = static_cast<long long>(nsnapshots) >= 4ll * nsteps;
  if (s->all_stages) {
    // slots 4i .. 4i+3: U_i and the stage states of step i; U_n goes to U
    if ((st = vt::ensure_slots(c, 4ll * nsteps))) return st;
    s->plan.clear();
    s->info = vt_checkpoint_info{};
    s->info.stage_steps = s->info.adjoint_steps = nsteps;
    s->info.slots_used = 4 * nsteps;
    s->info.all_stages = 1;
    cudaError_t e = vt::reset_error_words(c);
    if (!e)
      e = vt::run_captured(c, s->fwd_graph, vt::sweep_key(c, 0), [&]() {
        cudaError_t x = cudaMemcpyAsync(vt::slot(c, 0), c->U, sizeof(double2) * s->state_elems,
                                        cudaMemcpyDeviceToDevice, c->stream);
        for (int i = 0; i < nsteps && !x; ++i)
          x = vt::stage_step(c, vt::slot(c, 4ll * i), vt::slot(c, 4ll * i + 1), vt::slot(c, 4ll * i + 2),
                             vt::slot(c, 4ll * i + 3), dt, i + 1 < nsteps ? vt::slot(c, 4ll * i + 4) : c->U,
                             c->stream);
        return x;
      });
    if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("adjoint forward", e));
    st = vt::finish(c, nsteps, dt);
    if (st == VT_OK) s->have_forward = s->fresh = true;
    return st;
  }
  const int S = std::min(nsnapshots, nsteps);
  s->plan = vt::plan_reversal(nsteps, S);
  s->first_adjoint = 0;
  int used = 1;
  while (s->plan[s->first_adjoint].op != vt::CkptOp::kAdjoint) ++s->first_adjoint;
  for (const vt::CkptAction& a : s->plan)
    if (a.op == vt::CkptOp::kAdvance && a.dst != vt::kWorkSlot) used = std::max(used, a.dst + 1);
  // the overlapped reverse sweep's spare buffers follow the plan's slots
  s->plan_slots = used;
  if ((st = vt::ensure_slots(c, used + vt::kSpareSlots))) return st;
  if ((st = vt_checkpoint_plan(nsteps, S, &s->info))) return st;
  cudaError_t e = vt::reset_error_words(c);
  if (!e)
    e = vt::run_captured(c, s->fwd_graph, vt::sweep_key(c, 1), [&]() {
      cudaError_t x = cudaMemcpyAsync(vt::slot(c, 0), c->U, sizeof(double2) * s->state_elems,
                                      cudaMemcpyDeviceToDevice, c->stream);
      return x ? x : vt::run_plan(c, 0, s->first_adjoint, c->U);
    });
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("adjoint forward", e));
  st = vt::finish(c, nsteps, dt);
  if (st == VT_OK) s->have_forward = s->fresh = true;
  return st;
}

int vt_adjoint_backward(vt_ctx* c, const double* dJdU_T, double* dJdU_0, int device_pointers) {
  if (!c || !dJdU_T || !dJdU_0) return fail(VT_ERR_INVALID, "vt_adjoint_backward: null argument");
  if (device_pointers && !(vt::aligned_to(dJdU_T, 16) && vt::aligned_to(dJdU_0, 16)))
    return fail(VT_ERR_INVALID, "vt_adjoint_backward: device arrays must be 16-byte aligned");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (c->pending_steps) return fail(VT_ERR_INVALID, "a previous async step is not synchronised");
  vt::AdjointState* s = c->adj;
  if (!s || !s->have_forward) return fail(VT_ERR_INVALID, "vt_adjoint_backward: no forward sweep to reverse");
  cudaError_t e = vt::reset_error_words(c);
  if (s->all_stages) {  // nothing to recompute
    if (!e) e = vt::load_aos(c, dJdU_T, device_pointers, s->lam);
    if (!e)
      e = vt::run_captured(c, s->bwd_graph, vt::sweep_key(c, 2), [&]() {
        cudaError_t x = cudaSuccess;
        for (int i = s->nsteps - 1; i >= 0 && !x; --i)
          x = vt::adjoint_step(c, vt::slot(c, 4ll * i), vt::slot(c, 4ll * i + 1), vt::slot(c, 4ll * i + 2),
                               vt::slot(c, 4ll * i + 3), s->dt);
        return x;
      });
    if (!e) e = vt::store_aos(c, s->lam, dJdU_0, device_pointers);
    if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("adjoint backward", e));
    return vt::finish(c, 0, 0.0);
  }
  // the checkpoints of the forward sweep were reused by an earlier reverse
  // sweep (or the stage states by other calls): replay the sweep from U_0
  if (!e && !s->fresh) e = vt::run_plan(c, 0, s->first_adjoint, nullptr);
  s->fresh = false;
  if (!e) e = vt::load_aos(c, dJdU_T, device_pointers, s->lam);
  if (!e)
    e = vt::run_captured(c, s->bwd_graph, vt::sweep_key(c, 3),
                         [&]() { return vt::run_plan_overlapped(c, s->first_adjoint, s->plan.size()); });
  if (!e) e = vt::store_aos(c, s->lam, dJdU_0, device_pointers);
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("adjoint backward", e));
  return vt::finish(c, 0, 0.0);
}

int vt_adjoint_rk4(vt_ctx* c, double dt, int nsteps, int nsnapshots, const double* dJdU_T, double* dJdU_0) {
  if (!c || !dJdU_T || !dJdU_0) return fail(VT_ERR_INVALID, "vt_adjoint_rk4: null argument");
  const int st = vt_adjoint_forward(c, dt, nsteps, nsnapshots);
  return st ? st : vt_adjoint_backward(c, dJdU_T, dJdU_0, 0);
}

int vt_adjoint_info(const vt_ctx* c, vt_checkpoint_info* out) {
  if (!c || !out) return fail(VT_ERR_INVALID, "vt_adjoint_info: null argument");
  if (!c->adj || !c->adj->have_forward) return fail(VT_ERR_INVALID, "vt_adjoint_info: no forward sweep");
  *out = c->adj->info;
  return VT_OK;
}

int vt_rhs_jvp(vt_ctx* c, const double* U, const double* V, double* dR, int device_pointers) {
  if (!c || !U || !V || !dR) return fail(VT_ERR_INVALID, "vt_rhs_jvp: null argument");
  if (device_pointers && !(vt::aligned_to(U, 16) && vt::aligned_to(V, 16) && vt::aligned_to(dR, 16)))
    return fail(VT_ERR_INVALID, "vt_rhs_jvp: device arrays must be 16-byte aligned");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  int st = vt::prepare(c);
  if (st) return st;
  vt::AdjointState* s = c->adj;
  s->fresh = false;
  cudaError_t e = vt::load_aos(c, U, device_pointers, s->s1);
  if (!e) e = vt::load_aos(c, V, device_pointers, s->s2);
  if (!e) e = s->k.jvp(s->s1, s->s2, s->s3, c->geo, c->nbr, c->Kpad, c->K, c->ops.data(), c->stream);
  if (!e) e = vt::store_aos(c, s->s3, dR, device_pointers);
  if (!e) e = cudaStreamSynchronize(c->stream);
  return e ? fail(VT_ERR_CUDA, vt::cuda_msg("rhs jvp", e)) : VT_OK;
}

int vt_rhs_vjp(vt_ctx* c, const double* U, const double* W, double* G, int device_pointers) {
  if (!c || !U || !W || !G) return fail(VT_ERR_INVALID, "vt_rhs_vjp: null argument");
  if (device_pointers && !(vt::aligned_to(U, 16) && vt::aligned_to(W, 16) && vt::aligned_to(G, 16)))
    return fail(VT_ERR_INVALID, "vt_rhs_vjp: device arrays must be 16-byte aligned");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  int st = vt::prepare(c);
  if (st) return st;
  vt::AdjointState* s = c->adj;
  s->fresh = false;
  cudaError_t e = vt::reset_error_words(c);
  if (!e) e = vt::load_aos(c, U, device_pointers, s->s1);
  if (!e) e = vt::load_aos(c, W, device_pointers, s->s2);
  if (!e) {
    vt::AdjArgs a = vt::adj_args(c);
    a.U = s->s1, a.a = s->s2, a.acc_out = s->s3;
    e = vt::reverse_stage(c, a);
  }
  if (!e) e = vt::store_aos(c, s->s3, G, device_pointers);
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("rhs vjp", e));
  return vt::finish(c, 0, 0.0);
}

int vt_tangent_rk4(vt_ctx* c, double dt, int nsteps, const double* dU_0, double* dU_T, int device_pointers) {
  if (!c || nsteps < 0 || !dU_0 || !dU_T) return fail(VT_ERR_INVALID, "vt_tangent_rk4: bad argument");
  if (device_pointers && !(vt::aligned_to(dU_0, 16) && vt::aligned_to(dU_T, 16)))
    return fail(VT_ERR_INVALID, "vt_tangent_rk4: device arrays must be 16-byte aligned");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (c->pending_steps) return fail(VT_ERR_INVALID, "a previous async step is not synchronised");
  int st = vt::prepare(c);
  if (st) return st;
  vt::AdjointState* s = c->adj;
  s->fresh = false;
  double2 *dX = s->a0, *dS = s->a1, *dacc = s->acc, *dk = s->lam;
  const double2* X = c->U;
  auto jvp = [&](const double2* at, const double2* v) {
    return s->k.jvp(at, v, dk, c->geo, c->nbr, c->Kpad, c->K, c->ops.data(), c->stream);
  };
  cudaError_t e = vt::load_aos(c, dU_0, device_pointers, dX);
  if (!e) e = vt::reset_error_words(c);
  for (int n = 0; n < nsteps && !e; ++n) {
    if ((e = vt::stage_step(c, X, dt, nullptr))) break;
    if ((e = jvp(X, dX)) || (e = vt::lincomb(c, dacc, dX, 1.0, dk, (1.0 / 6) * dt)) ||
        (e = vt::lincomb(c, dS, dX, 1.0, dk, 0.5 * dt)))
      break;
    if ((e = jvp(s->s1, dS)) || (e = vt::lincomb(c, dacc, dacc, 1.0, dk, (1.0 / 3) * dt)) ||
        (e = vt::lincomb(c, dS, dX, 1.0, dk, 0.5 * dt)))
      break;
    if ((e = jvp(s->s2, dS)) || (e = vt::lincomb(c, dacc, dacc, 1.0, dk, (1.0 / 3) * dt)) ||
        (e = vt::lincomb(c, dS, dX, 1.0, dk, dt)))
      break;
    if ((e = jvp(s->s3, dS)) || (e = vt::lincomb(c, dX, dacc, 1.0, dk, (1.0 / 6) * dt))) break;
    e = vt::stage(c, s->s3, X, c->U, 3, 0.0, (1.0 / 6) * dt, c->stream);
  }
  if (!e) e = vt::store_aos(c, dX, dU_T, device_pointers);
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("tangent", e));
  return vt::finish(c, nsteps, dt);
}

int vt_roe_flux(const double* uL, const double* uR, double nx, double ny, double* flux) {
  if (!uL || !uR || !flux) return fail(VT_ERR_INVALID, "vt_roe_flux: null argument");
  return vt::roe_flux_t(uL, uR, nx, ny, flux);
}

int vt_roe_flux_jvp(const double* uL, const double* uR, double nx, double ny, const double* duL, const double* duR,
                    double* dflux) {
  if (!uL || !uR || !duL || !duR || !dflux) return fail(VT_ERR_INVALID, "vt_roe_flux_jvp: null argument");
  vt::Dual<1> L[4], R[4], f[4];
  for (int c = 0; c < 4; ++c) {
    L[c] = vt::Dual<1>(uL[c]);
    L[c].d[0] = duL[c];
    R[c] = vt::Dual<1>(uR[c]);
    R[c].d[0] = duR[c];
  }
  const int code = vt::roe_flux_t(L, R, nx, ny, f);
  for (int c = 0; c < 4; ++c) dflux[c] = f[c].d[0];
  return code;
}

void vt_roe_flux_vjp(const double* uL, const double* uR, double nx, double ny, const double* bflux, double* buL,
                     double* buR) {
  if (!uL || !uR || !bflux || !buL || !buR) return;
  vt::roe_flux_vjp(uL, uR, nx, ny, bflux, buL, buR);
}

}  // extern "C"
