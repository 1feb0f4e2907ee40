"""Brent's root finder driven one abscissa at a time, the drop-in for
``emu_base.math.brents_root_finding`` (reference emu_base/math/brents_root_finding.py:1-121).

The Monte Carlo stepper brackets the time of a quantum jump (where ||psi(t)||^2 crosses the
jump threshold) and asks for one abscissa at a time, evolving the state between requests.
The steps are Brent's published method: inverse quadratic interpolation, the secant step
when two ordinates nearly coincide, and bisection whenever the interpolated step leaves the
bracket or does not shrink it fast enough; the same tests and bookkeeping as the reference,
so that the same ordinates give the same abscissae.
"""

from __future__ import annotations

from typing import Callable, Optional


class BrentsRootFinder:
    """brents_root_finding.py:4-94."""

    def __init__(self, *, start: float, end: float, f_start: float, f_end: float,
                 epsilon: float = 1e-6):
        self.epsilon = epsilon
        assert start <= end
        self.a, self.b = start, end
        self.fa, self.fb = f_start, f_end
        assert self.fa * self.fb < 0, "Function root needs to be between a and b"
        if abs(self.fa) < abs(self.fb):  # b is the better guess
            self.a, self.b, self.fa, self.fb = self.b, self.a, self.fb, self.fa
        self.c, self.fc = self.a, self.fa
        self.d = self.c
        self.bisection = True
        self.current_guess = self.b
        self.next_abscissa: Optional[float] = None

    def get_next_abscissa(self) -> float:
        a, b, c, fa, fb, fc = self.a, self.b, self.c, self.fa, self.fb, self.fc
        if abs(fc - fa) < self.epsilon or abs(fc - fb) < self.epsilon:
            dx = fb * (b - a) / (fa - fb)  # secant
        else:  # inverse quadratic interpolation through (a, fa), (b, fb), (c, fc)
            s, r, t = fb / fa, fb / fc, fa / fc
            q = (t - 1) * (s - 1) * (r - 1)
            p = s * (t * (r - t) * (c - b) + (r - 1) * (b - a))
            dx = p / q
        tol = abs(2 * self.epsilon * b)
        adx, dbc, dcd, dab = abs(dx), abs(b - c), abs(c - self.d), a - b
        reject = (adx >= abs(3 * dab / 4) or dx * dab < 0
                  or (adx >= (dbc if self.bisection else dcd) / 2)
                  or ((dbc if self.bisection else dcd) < tol))
        if reject:
            dx = dab / 2
        self.bisection = reject
        self.next_abscissa = b + dx
        self.d = c
        self.c, self.fc = b, fb
        return self.next_abscissa

    def provide_ordinate(self, abscissa: float, ordinate: float) -> None:
        assert self.next_abscissa is not None and abscissa == self.next_abscissa, \
            "Something went wrong"
        if self.fa * ordinate < 0:
            self.b, self.fb = abscissa, ordinate
        else:
            self.a, self.fa = abscissa, ordinate
        if abs(self.fa) < abs(self.fb):
            self.a, self.b, self.fa, self.fb = self.b, self.a, self.fb, self.fa
        self.current_guess = self.b

    def is_converged(self, tolerance: float) -> bool:
        return abs(self.b - self.a) < tolerance


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
