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

// Minimal number of plain steps t(n, S) above (S >= 1, n >= 1).
int64_t binomial_forward_steps(int64_t n, int64_t S);

// The reversal of n steps with S >= 1 slots (slot 0 holds U_0). The first
// kStageStep of the plan is step n-1; everything before the first kAdjoint is
// the forward sweep. Slots are numbered 0..S-1, plus kWorkSlot.
std::vector<CkptAction> plan_reversal(int n, int S);

}  // namespace vt
