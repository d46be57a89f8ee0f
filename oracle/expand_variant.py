"""Reference scheme variants for the test oracle (TEST INFRASTRUCTURE ONLY).

The reference generates src/library/mhd_solver.inl from the Ruby template
src/library/mhd_solver.inlrb for one scheme chosen by
src/nushio_script/generate_config.rb (-s: SpaceInterpolation, -t:
TimeIntegral); the repository ships the expansion for minbee2 + midpoint2
only, and Ruby is not available here.  The two options change exactly two
things in the template, and this filter applies the template's own rules for
the other choices to the shipped expansion (read on stdin, written to
stdout), so that oracle/Makefile can host-compile the reference's
piecewiseconst1 and euler1 schemes:

* --space 1 (piecewiseconst1, mhd_solver.inlrb:128-136): interpolate() sets
  left and right to the two cells beside the face.  The template then
  generates a 2-cell stencil c0 = center - hex, c1 = center + hex
  (:580-586); these are the inner two of the shipped 4-cell stencil
  (center - hex - ex, center - hex, center + hex, center + hex + ex), and
  every interpolate() argument is a pure expression of its cell, so the
  4-argument interpolate() of the shipped file is replaced by one that
  returns its two inner arguments: the same values the template's
  piecewiseconst1 expansion computes.  The minbee helper absolute_smaller()
  goes with it.
* --time 1 (euler1, :966-969): proceed() runs integrator['dt', '', '', '']
  (:908-962) instead of integrator['dt/2', '', '', 'predictor_'] followed by
  integrator['dt', 'predictor_', '', ''].  The second midpoint stage is the
  integrator with opera = 'predictor_', bef = aft = ''; the Euler stage is
  the same text with opera = '', so the first stage is deleted and the
  second stage's add_flux_kernel_caller reads the current state instead of
  the predictor.

Each rewrite asserts that the text it replaces occurs exactly once.

Usage: expand_variant.py --space {1,2} --time {1,2} < mhd_solver.inl > variant.inl
"""
from __future__ import annotations

import argparse
import re
import sys

MINBEE = re.compile(
    r"__device__ Real absolute_smaller\(Real a, Real b\) \{.*?\}\s*"
    r"__device__ void interpolate\(const Real x0, const Real x1, const Real x2, const Real x3, "
    r"Real &left, Real &right\) \{.*?\n\}\n",
    re.S)

PIECEWISE_CONST = """__device__ void interpolate(const Real x0, const Real x1, const Real x2, const Real x3, Real &left, Real &right) {
  left  = x1;
  right = x2;
}
"""

STAGE = "    //// Zero-Initialize Pace\n"
PREDICTOR_FLUX = ("density_predictor_, velocity_predictor_, pressure_predictor_, magnet_predictor_,\n"
                  "       density_pace_")
CURRENT_FLUX = "density_, velocity_, pressure_, magnet_,\n       density_pace_"


def one(count, what):
    if count != 1:
        raise SystemExit(f"expand_variant: expected one {what}, found {count}")


def piecewise_constant(text: str) -> str:
    one(len(MINBEE.findall(text)), "minbee interpolate()")
    return MINBEE.sub(lambda _: PIECEWISE_CONST, text)


def euler(text: str) -> str:
    start = text.index("bool MHDSolver::proceed")
    body = text[start:]
    stages = [m.start() for m in re.finditer(re.escape(STAGE), body)]
    if len(stages) != 2:
        raise SystemExit(f"expand_variant: expected the two RK stages of proceed(), found {len(stages)}")
    first, second = stages
    one(body.count(PREDICTOR_FLUX), "predictor flux call")
    body = body[:first] + body[second:]
    body = body.replace(PREDICTOR_FLUX, CURRENT_FLUX)
    return text[:start] + body


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--space", type=int, choices=(1, 2), default=2)
    ap.add_argument("--time", type=int, choices=(1, 2), default=2)
    a = ap.parse_args()
    text = sys.stdin.read()
    if a.space == 1:
        text = piecewise_constant(text)
    if a.time == 1:
        text = euler(text)
    sys.stdout.write(text)


if __name__ == "__main__":
    main()
