// Binomial checkpointing for the discrete adjoint of an n-step RK4 run.
//
// The reverse sweep needs, for each step i = n-1 .. 0, the state at the start
// of step i (and the step's stage states, recomputed from it). With S slots
// holding states (slot 0 holds U_0), the plan below reverses the run with the
// fewest plain forward steps possible (Griewank's binomial bound):
//
//     t(n, S) = r n - C(S + r, S + 1),  r the least integer with C(S + r, S) >= n,
//
// counting the plain steps advanced between checkpoints (the forward sweep's
// included); each step is also run once with its stage states kept, right
// before its adjoint.
#pragma once

#include <cstdint>
#include <vector>

namespace vt {

enum class CkptOp : int8_t {
  kAdvance,    // advance `steps` plain RK4 steps from slot `src` into slot `dst`
  kStageStep,  // run step `step` from slot `src` keeping its stage states
  kAdjoint,    // reverse step `step` (its stage states are the last kept)
};

struct CkptAction {
  CkptOp op;
  int src = 0, dst = 0;
  int steps = 0;  // kAdvance
  int step = 0;   // kStageStep, kAdjoint: the step index
};

// The work slot: one buffer that is not a checkpoint (the end of an advance
// whose result is used once, by the stage step that follows it).
constexpr int kWorkSlot = -1;

// One action of the overlapped reverse sweep (vt_adjoint.cu,
// run_plan_overlapped): a plan action on physical state buffers. Advances and
// stage steps run on a side stream R, reverse steps on the main stream M.
// Buffers 0..nlog-1 are the plan's checkpoint slots, nlog the work slot, and
// nlog+1 .. nlog+nspare spare buffers that the slots are renamed onto.
struct OverlapStep {
  CkptOp op;
  int src = 0;          // buffer read: the start state of the advance, stage step or reverse step
  int dst = 0;          // kAdvance: buffer written
  int steps = 0;        // kAdvance: plain steps
  int step = 0;         // kStageStep, kAdjoint: the step index
  int set = 0;          // kStageStep: stage-state set written; kAdjoint: set read (0 or 1)
  long long wait = -1;  // kAdvance, kStageStep: R first waits until reverse step `wait` is done, or -1
  long long index = -1; // kAdjoint: the reverse step's issue index (0, 1, ...)
};

// Schedules plan[begin, end) (the reverse part of a plan_reversal plan, whose
// first reverse step reads stage-state set 0) for two streams:
//  * a reverse step reads the stage-state set the last stage step wrote (M
//    waits for that stage step on the device);
//  * a stage step writes the other set, after the reverse step that last read
//    it is done;
//  * an advance writes the buffer its target slot maps to; if a reverse step
//    that R has not yet waited for reads that buffer, the slot is renamed onto
//    the spare read longest ago (the old buffer becomes a spare), and R waits
//    only if that spare still has such a reader.
// The schedule's reads see the states the sequential plan's reads see, under
// every order of the two streams that the waits allow.
std::vector<OverlapStep> schedule_overlapped(const std::vector<CkptAction>& plan, size_t begin, size_t end,
                                             int nlog, int nspare);

// Minimal number of plain steps t(n, S) above (S >= 1, n >= 1).
int64_t binomial_forward_steps(int64_t n, int64_t S);

// The reversal of n steps with S >= 1 slots (slot 0 holds U_0). The first
// kStageStep of the plan is step n-1; everything before the first kAdjoint is
// the forward sweep. Slots are numbered 0..S-1, plus kWorkSlot.
std::vector<CkptAction> plan_reversal(int n, int S);

}  // namespace vt
