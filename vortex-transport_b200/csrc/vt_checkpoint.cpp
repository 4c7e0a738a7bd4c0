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

std::vector<OverlapStep> schedule_overlapped(const std::vector<CkptAction>& plan, size_t begin, size_t end,
                                             int nlog, int nspare) {
  std::vector<OverlapStep> out;
  const int nbuf = nlog + 1 + nspare;
  std::vector<int> map(static_cast<size_t>(nlog) + 1);  // logical slot (work slot = nlog) -> buffer
  for (int i = 0; i <= nlog; ++i) map[i] = i;
  std::vector<int> spares;
  for (int i = 0; i < nspare; ++i) spares.push_back(nlog + 1 + i);
  std::vector<long long> last_read(static_cast<size_t>(nbuf), -1);  // last reverse step reading each buffer
  long long set_reader[2] = {-1, -1};  // the reverse step that last read each stage-state set
  long long issued = 0;                // reverse steps scheduled
  long long synced = 0;                // R has waited for every reverse step below this index
  int cur = 0;                         // the set the last stage step wrote
  auto logical = [&](int sl) { return sl == kWorkSlot ? nlog : sl; };
  auto need = [&](long long k) -> long long {  // the wait R needs before it may overwrite what step k read
    if (k < synced) return -1;
    synced = k + 1;
    return k;
  };
  for (size_t i = begin; i < end && i < plan.size(); ++i) {
    const CkptAction& a = plan[i];
    OverlapStep x{};
    x.op = a.op;
    x.step = a.step;
    switch (a.op) {
      case CkptOp::kAdvance: {
        x.src = map[logical(a.src)];
        const int L = logical(a.dst);
        int pd = map[L];
        if (last_read[pd] >= synced && !spares.empty()) {
          size_t best = 0;
          for (size_t j = 1; j < spares.size(); ++j)
            if (last_read[spares[j]] < last_read[spares[best]]) best = j;
          const int q = spares[best];
          spares[best] = pd;
          map[L] = pd = q;
        }
        x.dst = pd;
        x.steps = a.steps;
        x.wait = need(last_read[pd]);
        break;
      }
      case CkptOp::kStageStep: {
        const int w = cur ^ 1;
        x.src = map[logical(a.src)];
        x.set = w;
        x.wait = need(set_reader[w]);
        cur = w;
        break;
      }
      case CkptOp::kAdjoint: {
        x.src = map[logical(a.src)];
        x.set = cur;
        x.index = issued;
        last_read[x.src] = issued;
        set_reader[cur] = issued;
        ++issued;
        break;
      }
    }
    out.push_back(x);
  }
  return out;
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
