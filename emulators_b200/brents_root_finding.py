"""Brent's root finder driven one abscissa at a time, the drop-in for
``emu_base.math.brents_root_finding`` (reference emu_base/math/brents_root_finding.py:1-121).

The Monte Carlo stepper brackets the time of a quantum jump (where ||psi(t)||^2 crosses the
jump threshold) and asks for one abscissa at a time, evolving the state between requests.
The steps are Brent's published method: inverse quadratic interpolation, the secant step
when two ordinates nearly coincide, and bisection whenever the interpolated step leaves the
bracket or does not shrink it fast enough.  The tests and their floating-point order are
the reference's, so that the same ordinates give the same abscissae.
"""

from __future__ import annotations

from typing import Callable, Optional


class BrentsRootFinder:
    """brents_root_finding.py:4-94.  The bracket is kept as the best abscissa so far
    (smallest |ordinate|) and the opposite end of the bracket (ordinate of the other sign);
    the two previous best abscissae steer the choice between an interpolated step and
    bisection."""

    def __init__(self, *, start: float, end: float, f_start: float, f_end: float,
                 epsilon: float = 1e-6):
        self.epsilon = epsilon
        assert start <= end, "the bracket needs start <= end"
        self._far, self._best = start, end
        self._f_far, self._f_best = f_start, f_end
        assert self._f_far * self._f_best < 0, "f(start) and f(end) must have opposite signs"
        self._keep_best_smallest()
        self._prev, self._f_prev = self._far, self._f_far
        self._prev2 = self._prev
        self._bisected = True
        self.current_guess = self._best
        self.next_abscissa: Optional[float] = None

    def _keep_best_smallest(self) -> None:
        if abs(self._f_far) < abs(self._f_best):
            self._far, self._best = self._best, self._far
            self._f_far, self._f_best = self._f_best, self._f_far

    def get_next_abscissa(self) -> float:
        x0, x1, xp = self._far, self._best, self._prev
        f0, f1, fp = self._f_far, self._f_best, self._f_prev
        if abs(fp - f0) < self.epsilon or abs(fp - f1) < self.epsilon:
            step = f1 * (x1 - x0) / (f0 - f1)  # secant through the bracket ends
        else:  # inverse quadratic interpolation through the three points
            s, r, t = f1 / f0, f1 / fp, f0 / fp
            q = (t - 1) * (s - 1) * (r - 1)
            p = s * (t * (r - t) * (xp - x1) + (r - 1) * (x1 - x0))
            step = p / q
        tol = abs(2 * self.epsilon * x1)
        span = x0 - x1
        recent = abs(x1 - xp) if self._bisected else abs(xp - self._prev2)
        leaves_bracket = abs(step) >= abs(3 * span / 4) or step * span < 0
        too_slow = abs(step) >= recent / 2 or recent < tol
        self._bisected = leaves_bracket or too_slow
        if self._bisected:
            step = span / 2
        self.next_abscissa = x1 + step
        self._prev2 = xp
        self._prev, self._f_prev = x1, f1
        return self.next_abscissa

    def provide_ordinate(self, abscissa: float, ordinate: float) -> None:
        assert self.next_abscissa is not None and abscissa == self.next_abscissa, \
            "provide_ordinate expects the ordinate of the last get_next_abscissa"
        if self._f_far * ordinate < 0:
            self._best, self._f_best = abscissa, ordinate
        else:
            self._far, self._f_far = abscissa, ordinate
        self._keep_best_smallest()
        self.current_guess = self._best

    def is_converged(self, tolerance: float) -> bool:
        return abs(self._best - self._far) < tolerance


def find_root_brents(f: Callable[[float], float], *, start: float, end: float,
                     f_start: Optional[float] = None, f_end: Optional[float] = None,
                     tolerance: float = 1e-6, epsilon: float = 1e-6) -> float:
    """brents_root_finding.py:97-121."""
    f_start = f(start) if f_start is None else f_start
    f_end = f(end) if f_end is None else f_end
    rf = BrentsRootFinder(start=start, end=end, f_start=f_start, f_end=f_end, epsilon=epsilon)
    while not rf.is_converged(tolerance):
        x = rf.get_next_abscissa()
        rf.provide_ordinate(x, f(x))
    return rf.current_guess
