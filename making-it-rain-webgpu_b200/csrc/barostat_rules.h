// barostat_rules.h -- the Monte Carlo barostat's acceptance rules (host code).
//
// Kept apart from the engine so that a test can run the same compiled rules
// on a CPU toy chain (tests/test_barostat_rules.py) and check that they keep
// the target distribution.  No CUDA here.
#pragma once

#include <algorithm>
#include <cmath>

namespace mdb {

// The plain Metropolis test of a volume move with reduced work w = dU +
// P dV - N kT dlnV (kJ/mol) at kT (src/reference/barostat.ts:248): a move
// with w <= 0 is accepted without a draw; otherwise `draw()` gives a uniform
// number in (0, 1) and the move is accepted unless it exceeds exp(-w/kT).
// Drawing only when w > 0 keeps the stream of draws the reference's.
template <class Draw>
inline bool plain_accept(double w, double kT, Draw&& draw) {
  return !(w > 0 && draw() > std::exp(-w / kT));
}

// Delayed acceptance (Christen & Fox 2005), stage 1: the probability that a
// move goes on to the exact energy, from the screening network's predicted
// potential change du_pred and the move's volume term.
inline double screen_probability(double du_pred, double volume_term, double kT) {
  return std::min(1.0, std::exp(-(du_pred + volume_term) / kT));
}

// Stage 2: the probability of accepting a move that passed stage 1 with
// probability a1, from its exact work w and the network's prediction
// du_rev_pred for the reverse move (made from the proposal, whose volume term
// is -volume_term).  The factor a1(y->x) / a1(x->y) makes the two stages
// together satisfy detailed balance with respect to exp(-w/kT) whatever the
// network predicts.
inline double exact_stage_probability(double w, double du_rev_pred, double volume_term, double kT, double a1) {
  const double a1_rev = std::min(1.0, std::exp(-(du_rev_pred - volume_term) / kT));
  return std::min(1.0, std::exp(-w / kT) * a1_rev / a1);
}

}  // namespace mdb
