// Binomial checkpoint schedule (vt_checkpoint.h) and its C ABI query.
#include "vt_checkpoint.h"

#include <algorithm>
#include <limits>

#include "../../include/vortex_b200.h"
#include "vt_common.h"

namespace vt {
namespace {

constexpr int64_t kSat = std::numeric_limits<int64_t>::max() / 4;

// C(a, b), saturated at kSat.
int64_t binom(int64_t a, int64_t b) {
  if (b < 0 || b > a) return 0;
  b = std::min(b, a - b);
  long double r = 1;
  for (int64_t i = 1; i <= b; ++i) {
    r = r * static_cast<long double>(a - b + i) / static_cast<long double>(i);
    if (r > static_cast<long double>(kSat)) return kSat;
  }
  return static_cast<int64_t>(r + 0.5L);
}

}  // namespace

int64_t binomial_forward_steps(int64_t n, int64_t S) {
  if (n <= 1) return 0;
  int64_t r = 0;
  while (binom(S + r, S) < n) ++r;
  return r * n - binom(S + r, S + 1);
}

// Recursion (run on an explicit stack): to reverse steps [l, r) from the state
// at l held in a slot, with free slots left, advance to a split point m chosen
// to attain the bound, store it, reverse [m, r) with one slot fewer, release it
// and reverse [l, m). With no free slot, every step re-advances from l.
std::vector<CkptAction> plan_reversal(int n, int S) {
  std::vector<CkptAction> plan;
  if (n < 1 || S < 1) return plan;
  std::vector<int> free_slots;
  for (int s = S - 1; s >= 1; --s) free_slots.push_back(s);
  struct Task {
    bool release;
    int l, r, slot;
  };
  std::vector<Task> stack{{false, 0, n, 0}};
  while (!stack.empty()) {
    const Task t = stack.back();
    stack.pop_back();
    if (t.release) {
      free_slots.push_back(t.slot);
      continue;
    }
    const int len = t.r - t.l;
    if (len == 1) {
      plan.push_back({CkptOp::kStageStep, t.slot, 0, 0, t.l});
      plan.push_back({CkptOp::kAdjoint, t.slot, 0, 0, t.l});
      continue;
    }
    if (free_slots.empty()) {
      for (int i = t.r - 1; i >= t.l; --i) {
        const int src = i > t.l ? kWorkSlot : t.slot;
        if (i > t.l) plan.push_back({CkptOp::kAdvance, t.slot, kWorkSlot, i - t.l, 0});
        plan.push_back({CkptOp::kStageStep, src, 0, 0, i});
        plan.push_back({CkptOp::kAdjoint, src, 0, 0, i});
      }
      continue;
    }
    const int64_t Sc = static_cast<int64_t>(free_slots.size()) + 1;
    const int64_t best = binomial_forward_steps(len, Sc);
    int m = 1;
    for (; m < len; ++m)
      if (m + binomial_forward_steps(len - m, Sc - 1) + binomial_forward_steps(m, Sc) == best) break;
    if (m == len) m = 1;  // not reached: some split attains the bound
    const int slot_m = free_slots.back();
    free_slots.pop_back();
    plan.push_back({CkptOp::kAdvance, t.slot, slot_m, m, 0});
    stack.push_back({false, t.l, t.l + m, t.slot});
    stack.push_back({true, 0, 0, slot_m});
    stack.push_back({false, t.l + m, t.r, slot_m});
  }
  return plan;
}

}  // namespace vt

extern "C" int vt_checkpoint_plan(int nsteps, int nsnapshots, vt_checkpoint_info* out) {
  if (nsteps < 1 || nsnapshots < 1 || !out) return vt::fail(VT_ERR_INVALID, "vt_checkpoint_plan: bad argument");
  const int S = std::min(nsnapshots, nsteps);
  const std::vector<vt::CkptAction> plan = vt::plan_reversal(nsteps, S);
  vt_checkpoint_info info{};
  int next_adjoint = nsteps - 1;
  bool forward = true;
  for (const vt::CkptAction& a : plan) {
    switch (a.op) {
      case vt::CkptOp::kAdvance:
        info.advance_steps += a.steps;
        if (forward) info.forward_sweep_steps += a.steps;
        if (a.dst != vt::kWorkSlot) info.slots_used = std::max(info.slots_used, a.dst + 1);
        break;
      case vt::CkptOp::kStageStep:
        info.stage_steps += 1;
        break;
      case vt::CkptOp::kAdjoint:
        if (a.step != next_adjoint) return vt::fail(VT_ERR_INVALID, "vt_checkpoint_plan: steps out of order");
        --next_adjoint;
        forward = false;
        info.adjoint_steps += 1;
        break;
    }
  }
  info.slots_used = std::max(info.slots_used, 1);
  info.optimal_advance_steps = vt::binomial_forward_steps(nsteps, S);
  *out = info;
  return VT_OK;
}
