// Check of the overlapped reverse sweep's schedule (schedule_overlapped,
// vortex-transport_b200/csrc/vt_checkpoint.cpp), compiled and run by
// tests/test_overlap_schedule.py on the CPU; the GPU runner
// (run_plan_overlapped, vt_adjoint.cu) executes exactly this schedule.
//
// For a plan_reversal(n, S) plan the check follows two models:
//  * the sequential plan: which step's state every logical slot holds, so that
//    each advance, stage step and reverse step has the state it must read
//    (a reverse step of step i must read U_i and the stage states of step i);
//  * the two streams: side-stream actions (advances, stage steps) in order on
//    physical buffers, reverse steps in order on the main stream. A reverse
//    step starts after the stage step that wrote its set (its event) and is
//    known done before a side-stream action only through that action's or an
//    earlier one's wait. A reverse step must read the buffer content the last
//    side-stream write before its stage step left, and no later write to that
//    buffer (or to its stage-state set) may come before a wait on it.
// Prints one line per case and exits non-zero on the first violation.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "vt_checkpoint.h"

namespace vt {
// the scheduler's translation unit reports bad arguments through this
int fail(int status, const std::string&) { return status; }
}  // namespace vt

using vt::CkptAction;
using vt::CkptOp;
using vt::OverlapStep;

namespace {

int bad(int n, int S, int nspare, size_t i, const char* what) {
  std::printf("FAIL n=%d S=%d spares=%d action %zu: %s\n", n, S, nspare, i, what);
  return 1;
}

int check(int n, int S, int nspare, long long* waits_out) {
  const std::vector<CkptAction> plan = vt::plan_reversal(n, S);
  size_t begin = 0;
  while (begin < plan.size() && plan[begin].op != CkptOp::kAdjoint) ++begin;
  if (begin == plan.size() || begin == 0) return bad(n, S, nspare, 0, "plan has no reverse part");
  int nlog = 1;  // as vt_adjoint_forward sizes the slot pool
  for (const CkptAction& a : plan)
    if (a.op == CkptOp::kAdvance && a.dst != vt::kWorkSlot) nlog = std::max(nlog, a.dst + 1);
  auto logical = [&](int sl) { return sl == vt::kWorkSlot ? nlog : sl; };

  // sequential model over the forward part: slot -> the step whose state it holds (-1: none)
  std::vector<int> held(static_cast<size_t>(nlog) + 1, -1);
  held[0] = 0;
  int last_stage = -1;  // step whose stage states the forward part kept (set 0)
  for (size_t i = 0; i < begin; ++i) {
    const CkptAction& a = plan[i];
    if (a.op == CkptOp::kAdvance) {
      if (held[logical(a.src)] < 0) return bad(n, S, nspare, i, "forward advance from an empty slot");
      held[logical(a.dst)] = held[logical(a.src)] + a.steps;
    } else if (a.op == CkptOp::kStageStep) {
      if (held[logical(a.src)] != a.step) return bad(n, S, nspare, i, "forward stage step from the wrong state");
      last_stage = a.step;
    }
  }

  const std::vector<OverlapStep> sched = vt::schedule_overlapped(plan, begin, plan.size(), nlog, nspare);
  if (sched.size() != plan.size() - begin) return bad(n, S, nspare, begin, "schedule length");
  const int nbuf = nlog + 1 + nspare;
  // side-stream model: buffer contents after each side-stream action, the
  // stage step each set holds, and how far the side stream has waited
  std::vector<int> content(static_cast<size_t>(nbuf), -1);
  for (int l = 0; l <= nlog; ++l) content[l] = held[l];  // the forward part wrote the slots in place
  int set_step[2] = {last_stage, -1};
  long long synced = 0;  // reverse steps below this index are known done on the side stream
  long long waits = 0;
  // per buffer: the reverse steps issued since its last write that read it
  std::vector<std::vector<long long>> readers(static_cast<size_t>(nbuf));
  long long set_last_reader[2] = {-1, -1};  // the last reverse step that read each set
  std::vector<int> seq_held = held;  // sequential model, continued through the reverse part
  long long next_index = 0;
  int expect_step = n - 1;
  for (size_t k = 0; k < sched.size(); ++k) {
    const size_t i = begin + k;
    const CkptAction& a = plan[i];
    const OverlapStep& x = sched[k];
    if (x.op != a.op) return bad(n, S, nspare, i, "schedule and plan differ");
    if (x.src < 0 || x.src >= nbuf || x.dst < 0 || x.dst >= nbuf) return bad(n, S, nspare, i, "buffer out of range");
    if (x.wait >= 0) {
      if (x.wait >= next_index) return bad(n, S, nspare, i, "waits for a reverse step not yet issued");
      synced = std::max(synced, x.wait + 1);
      ++waits;
    }
    switch (a.op) {
      case CkptOp::kAdvance: {
        const int want = seq_held[logical(a.src)];
        if (want < 0 || content[x.src] != want) return bad(n, S, nspare, i, "advance reads the wrong state");
        // write-after-read: every reverse step that read this buffer is done
        for (const long long r : readers[x.dst])
          if (r >= synced) return bad(n, S, nspare, i, "advance overwrites a buffer a reverse step may still read");
        readers[x.dst].clear();
        content[x.dst] = want + a.steps;
        seq_held[logical(a.dst)] = want + a.steps;
        break;
      }
      case CkptOp::kStageStep: {
        const int want = seq_held[logical(a.src)];
        if (want != a.step || content[x.src] != want) return bad(n, S, nspare, i, "stage step reads the wrong state");
        if (x.set != 0 && x.set != 1) return bad(n, S, nspare, i, "stage-state set out of range");
        if (set_last_reader[x.set] >= synced)
          return bad(n, S, nspare, i, "stage step overwrites a set a reverse step may still read");
        set_step[x.set] = a.step;
        break;
      }
      case CkptOp::kAdjoint: {
        if (a.step != expect_step--) return bad(n, S, nspare, i, "reverse steps out of order");
        if (x.index != next_index) return bad(n, S, nspare, i, "reverse step index");
        // read-after-write: the reverse step starts after the stage step that
        // wrote its set, i.e. after every side-stream action issued so far
        if (set_step[x.set] != a.step) return bad(n, S, nspare, i, "reverse step reads another step's stage states");
        if (content[x.src] != a.step || seq_held[logical(a.src)] != a.step)
          return bad(n, S, nspare, i, "reverse step reads the wrong start state");
        readers[x.src].push_back(next_index);
        set_last_reader[x.set] = next_index;
        ++next_index;
        break;
      }
    }
  }
  if (expect_step != -1) return bad(n, S, nspare, plan.size(), "not every step reversed");
  *waits_out = waits;
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  std::vector<std::pair<int, int>> cases = {{2000, 45}, {1234, 400}, {300, 3}, {100, 2}, {57, 7},
                                            {1000, 10}, {24, 3},     {2, 1},    {5, 1}};
  for (int n = 2; n <= 40; ++n)
    for (int S = 1; S <= 6; ++S) cases.push_back({n, S});
  if (argc == 3) cases = {{std::atoi(argv[1]), std::atoi(argv[2])}};
  for (const auto& c : cases) {
    long long w[3] = {0, 0, 0};
    for (int nspare = 0; nspare <= 2; ++nspare)
      if (check(c.first, std::min(c.second, c.first), nspare, &w[nspare])) return 1;
    if (c.first >= 100)
      std::printf("OK n=%d S=%d: side-stream waits with 0 / 1 / 2 spares: %lld / %lld / %lld\n", c.first, c.second,
                  w[0], w[1], w[2]);
  }
  std::printf("OK all %zu cases\n", cases.size());
  return 0;
}
