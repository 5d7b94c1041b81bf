// ladder.cuh -- device-side escalation test of the adaptive ladder.
//
// AdaptiveSelector::should_escalate (adaptive_selector.cpp:238-267) evaluated on the
// device after every Krylov step, on the history of relative residuals BEFORE the
// current one (as its callers pass it, tests/test_adaptive.cpp:82-106 in the reference):
//   divergence  history >= 2 entries and rel > 10 * history[0]
//   stall       history >= window entries and rel / history[size - window] > threshold
//   budget      EASY and iteration > max_iter*4/10, MODERATE and iteration > max_iter*7/10
// The reference defines this test but its solve loop never calls it (it escalates only
// when an attempt exhausts max_iter); ladder_mode = 1 turns it on.  With no_stall set (the
// CG rung under ladder_mode = 3) the windowed stall rule is skipped: CG's recursive
// residual is not monotone, and on variable-coefficient problems it rises and falls over
// tens of iterations, so a 15-iteration window ends attempts that were converging.
#pragma once

#include "common.cuh"

namespace hamlss {

constexpr int kLadderRing = 64;

struct LadderCfg {
    int on = 0;
    int state = HAMLSS_STATE_EASY;
    int window = 15;
    double threshold = 0.95;
    int max_iter = 2000;
    int no_stall = 0;
};

struct LadderDev {
    int on, state, window, max_iter, count, reason, no_stall;
    double threshold, first;
    double ring[kLadderRing];
};

// reason codes match hamlss_escalation.reason
enum : int { ESC_NONE = 0, ESC_STALL = 1, ESC_BUDGET = 2, ESC_DIVERGENCE = 3 };

inline LadderDev ladder_init(const LadderCfg* c) {
    LadderDev d{};
    if (c && c->on) {
        d.on = 1;
        d.state = c->state;
        d.window = c->window < 1 ? 1 : (c->window > kLadderRing ? kLadderRing : c->window);
        d.threshold = c->threshold;
        d.max_iter = c->max_iter;
        d.no_stall = c->no_stall;
    }
    return d;
}

// Returns the escalation reason (0 = keep going) and records rel in the history.
__device__ __forceinline__ int ladder_check(LadderDev* L, int iteration, double rel) {
    if (!L->on) return ESC_NONE;
    int reason = ESC_NONE;
    const int k = L->count;
    if (k >= 2 && rel > 10.0 * L->first) reason = ESC_DIVERGENCE;
    else if (!L->no_stall && k >= L->window) {
        double prev = L->ring[(k - L->window) % kLadderRing];
        if (prev > 2.220446049250313e-16 && rel / prev > L->threshold) reason = ESC_STALL;
    }
    if (!reason && L->state == HAMLSS_STATE_EASY && iteration > L->max_iter * 4 / 10) reason = ESC_BUDGET;
    if (!reason && L->state == HAMLSS_STATE_MODERATE && iteration > L->max_iter * 7 / 10)
        reason = ESC_BUDGET;
    if (k == 0) L->first = rel;
    L->ring[k % kLadderRing] = rel;
    L->count = k + 1;
    if (reason) L->reason = reason;
    return reason;
}

}  // namespace hamlss
