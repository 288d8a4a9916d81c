// Binomial checkpointing schedule for reversing a time-stepping loop (host code).
//
// Reversing T steps needs the state u_k before the adjoint of step k, for k = T-1 .. 0. Holding
// every state costs T states; holding none costs T(T-1)/2 recomputed steps. With c free slots
// besides the one that holds the segment's first state, the fewest forward steps F(t, c) to
// reverse a segment of t steps satisfy
//   F(1, c) = 0,   F(t, 0) = t (t - 1) / 2,
//   F(t, c) = min_{1 <= m < t} [ m + F(t - m, c - 1) + F(m, c) ]
// (advance m steps and store u_m, reverse the right part with one slot fewer, restore the first
// state and reverse the left part). Its minima are the binomial numbers of Griewank's revolve
// (Griewank & Walther, ACM TOMS 26(1), 2000); here they are found by dynamic programming, which
// also yields the split points the schedule follows.
#pragma once

#include <vector>

namespace exa_ck {

enum { STORE = 0, RESTORE = 1, ADVANCE = 2, ADJOINT = 3 };

struct Action {
  int action, a, b;
};

class Planner {
 public:
  Planner(int steps, int free_slots) : T_(steps), C_(free_slots) {
    F_.assign((size_t)(T_ + 1) * (C_ + 1), 0);
    split_.assign((size_t)(T_ + 1) * (C_ + 1), 0);
    for (int t = 1; t <= T_; t++) {
      for (int c = 0; c <= C_; c++) {
        long long best;
        int bm = 0;
        if (t == 1) {
          best = 0;
        } else if (c == 0) {
          best = (long long)t * (t - 1) / 2;
        } else {
          best = -1;
          for (int m = 1; m < t; m++) {
            const long long v = m + F(t - m, c - 1) + F(m, c);
            if (best < 0 || v < best) {
              best = v;
              bm = m;
            }
          }
        }
        F_[(size_t)t * (C_ + 1) + c] = best;
        split_[(size_t)t * (C_ + 1) + c] = bm;
      }
    }
  }
  long long F(int t, int c) const { return F_[(size_t)t * (C_ + 1) + c]; }

  // the whole schedule: store u_0 in slot 0, then reverse [0, T)
  std::vector<Action> schedule() {
    out_.clear();
    top_ = 1;
    cur_ = 0;
    out_.push_back({STORE, 0, 0});
    rec(0, T_, C_, 0);
    return out_;
  }

 private:
  // precondition: the state u_l is stored in `slot`
  void rec(int l, int r, int c, int slot) {
    const int t = r - l;
    if (t == 1) {
      ensure(l, slot);
      out_.push_back({ADJOINT, l, 0});
      return;
    }
    if (c == 0) {
      for (int j = r - 1; j >= l; j--) {
        ensure(l, slot);
        if (j > l) advance(l, j);
        out_.push_back({ADJOINT, j, 0});
      }
      return;
    }
    const int m = l + split_[(size_t)t * (C_ + 1) + c];
    ensure(l, slot);
    advance(l, m);
    const int s2 = top_++;
    out_.push_back({STORE, s2, m});
    rec(m, r, c - 1, s2);
    top_--;
    rec(l, m, c, slot);
  }
  void ensure(int l, int slot) {
    if (cur_ != l) {
      out_.push_back({RESTORE, slot, l});
      cur_ = l;
    }
  }
  void advance(int from, int to) {
    out_.push_back({ADVANCE, from, to});
    cur_ = to;
  }

  int T_, C_;
  std::vector<long long> F_;
  std::vector<int> split_;
  std::vector<Action> out_;
  int top_ = 1, cur_ = 0;
};

}  // namespace exa_ck
