"""The barostat's acceptance rules keep the target distribution (CPU).

The engine decides every volume move with the three functions of
`csrc/barostat_rules.h`: the plain Metropolis test (the reference's
`barostat.ts:248`), the screening stage's probability and the exact stage's
probability of delayed acceptance (Christen & Fox 2005).  This test compiles
that header into a small C++ program and runs the rules on a one-dimensional
chain whose target is known in closed form: x with potential U(x) = x^2 / 2
and a "volume term" G(x) = x / 2, so exp(-(U + G) / kT) at kT = 1 is a
Gaussian of mean -0.5 and variance 1.  Proposals are symmetric steps.  The
screening model is deliberately wrong (half the true change, plus a tilt and
a wiggle in x), as a poorly trained network would be.

* the plain rule and the two-stage rule both sample mean -0.5 and variance 1;
* the two-stage rule rejects a good share of proposals on the prediction
  alone (the saving the network is there for);
* a two-stage rule without the reverse-move factor a1(y->x) / a1(x->y),
  planted in the test program, samples a visibly different distribution, so
  the test can tell a wrong rule from a right one.
"""

from __future__ import annotations

import json
import shutil
import subprocess
from pathlib import Path

import pytest

CSRC = Path(__file__).resolve().parents[1] / "making-it-rain-webgpu_b200" / "csrc"

PROGRAM = r"""
#include <cmath>
#include <cstdint>
#include <cstdio>
#include "barostat_rules.h"

namespace {
uint64_t state = 0x9e3779b97f4a7c15ull;
double uniform() {  // splitmix64, (0, 1)
  uint64_t z = (state += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  return (double(z >> 11) + 0.5) * 0x1.0p-53;
}
const double kT = 1.0, half_width = 1.6;
double potential(double x) { return 0.5 * x * x; }
double volume(double x) { return 0.5 * x; }
// a wrong but deterministic prediction of the potential change of the move x -> x + d
double predicted(double x, double d) {
  return 0.5 * (potential(x + d) - potential(x)) + 0.8 * d + 0.7 * std::sin(3.0 * x);
}

struct Result { double mean, var, screened, accepted; };

Result chain(int rule, long steps) {
  double x = 0, sum = 0, sum2 = 0;
  long screened = 0, accepted = 0;
  for (long i = 0; i < steps; ++i) {
    const double d = half_width * (2 * uniform() - 1), y = x + d;
    const double vt = volume(y) - volume(x), w = potential(y) - potential(x) + vt;
    bool ok = false;
    if (rule == 0) {
      ok = mdb::plain_accept(w, kT, uniform);
    } else {
      const double a1 = mdb::screen_probability(predicted(x, d), vt, kT);
      if (uniform() < a1) {
        const double a2 = rule == 1 ? mdb::exact_stage_probability(w, predicted(y, -d), vt, kT, a1)
                                    : std::fmin(1.0, std::exp(-w / kT));  // planted mistake: no reverse factor
        ok = uniform() < a2;
      } else {
        ++screened;
      }
    }
    if (ok) { x = y; ++accepted; }
    sum += x;
    sum2 += x * x;
  }
  const double mean = sum / steps;
  return {mean, sum2 / steps - mean * mean, double(screened) / steps, double(accepted) / steps};
}
}  // namespace

int main() {
  const long steps = 4000000;
  const char* names[3] = {"plain", "delayed", "no_reverse_factor"};
  std::printf("{");
  for (int rule = 0; rule < 3; ++rule) {
    const Result r = chain(rule, steps);
    std::printf("%s\"%s\": {\"mean\": %.6f, \"var\": %.6f, \"screened\": %.6f, \"accepted\": %.6f}",
                rule ? ", " : "", names[rule], r.mean, r.var, r.screened, r.accepted);
  }
  std::printf("}\n");
  return 0;
}
"""

MEAN, VAR = -0.5, 1.0
# about six standard errors of 4 M correlated steps (integrated correlation
# time of a few steps at this proposal width)
MEAN_TOL, VAR_TOL = 0.012, 0.02


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    compiler = shutil.which("g++")
    if compiler is None:
        pytest.skip("g++ is not installed")
    work = tmp_path_factory.mktemp("barostat_rules")
    source = work / "chain.cpp"
    source.write_text(PROGRAM)
    binary = work / "chain"
    subprocess.run([compiler, "-O2", "-std=c++17", "-I", str(CSRC), str(source), "-o", str(binary)], check=True)
    out = subprocess.run([str(binary)], check=True, capture_output=True, text=True, timeout=120).stdout
    return json.loads(out)


def test_plain_rule_samples_the_target(results):
    r = results["plain"]
    print(r)
    assert abs(r["mean"] - MEAN) < MEAN_TOL and abs(r["var"] - VAR) < VAR_TOL


def test_delayed_acceptance_samples_the_target_with_a_wrong_network(results):
    r = results["delayed"]
    print(r)
    assert abs(r["mean"] - MEAN) < MEAN_TOL and abs(r["var"] - VAR) < VAR_TOL
    # the first stage alone turns away a good share of the proposals
    assert r["screened"] > 0.2


def test_a_rule_without_the_reverse_factor_is_caught(results):
    r = results["no_reverse_factor"]
    print(r)
    assert abs(r["mean"] - MEAN) > 5 * MEAN_TOL or abs(r["var"] - VAR) > 5 * VAR_TOL
