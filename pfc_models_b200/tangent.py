"""Common-tangent (Maxwell) construction between free-energy branches f(phi).

The consumer of a phase-diagram sweep: for each temperature, the liquid branch is
analytic and the solid branch is the table of F per site against the mean density
that the device reductions produced. Mirrors the parts of the reference's
phase_diagram/common_tangent.py that a liquid-solid scan uses:
`analytic_branch` (:275), `tabulated_branch` (:336, a not-a-knot cubic spline of
each run of >= 4 finite points; mu is its derivative) and `common_tangent`
(:522): densities phi_a, phi_b with mu_a(phi_a) = mu_b(phi_b) = mu and equal grand
potential omega = f - mu phi.

Method: on every interval where a branch is convex (f'' > 0) mu(phi) is monotonic
and can be inverted, giving omega(mu) for that piece; a tangent is a root in mu of
omega_a(mu) - omega_b(mu) on the overlap of two pieces' mu ranges (brentq, after a
scan for sign changes).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.interpolate import CubicHermiteSpline, CubicSpline
from scipy.optimize import brentq


@dataclass
class Branch:
    name: str
    f: object          # f(phi)
    mu: object         # df/dphi
    d2f: object        # d2f/dphi2
    lo: float
    hi: float
    kind: str = "analytic"

    def convex_pieces(self, n=4097):
        """[lo, hi] split into the maximal intervals where f'' > 0 (ends refined by brentq)."""
        x = np.linspace(self.lo, self.hi, n)
        pos = np.asarray(self.d2f(x), dtype=float) > 0
        d2 = lambda p: float(self.d2f(p))  # noqa: E731
        pieces, i = [], 0
        while i < n:
            if not pos[i]:
                i += 1
                continue
            j = i
            while j + 1 < n and pos[j + 1]:
                j += 1
            a = x[i] if i == 0 else brentq(d2, x[i - 1], x[i])
            b = x[j] if j == n - 1 else brentq(d2, x[j], x[j + 1])
            if b > a:
                pieces.append((float(a), float(b)))
            i = j + 1
        return pieces


def analytic_branch(name, f, mu, lo, hi, d2f=None, h=1e-6):
    """Branch from closed forms (phase_diagram/common_tangent.py:275); f'' by central
    differences of mu when not given."""
    if d2f is None:
        def d2f(p):
            p = np.asarray(p, dtype=float)
            return (np.asarray(mu(p + h)) - np.asarray(mu(p - h))) / (2 * h)
    return Branch(name, f, mu, d2f, float(lo), float(hi))


def tabulated_branch(name, phi, f, min_points=4, mu=None, extend_lo=0.0):
    """Branch from a table (phase_diagram/common_tangent.py:336): the longest run of
    consecutive finite points (sorted by phi) as a not-a-knot cubic spline of f, or,
    when the table also holds mu = df/dphi at each point, as the cubic Hermite
    spline through (phi, f, mu) (then 2 points make a run). `extend_lo` lets the
    branch continue that far below its first point on the first cubic piece."""
    phi = np.asarray(phi, dtype=float).ravel()
    f = np.asarray(f, dtype=float).ravel()
    order = np.argsort(phi, kind="stable")
    phi, f = phi[order], f[order]
    good = np.isfinite(phi) & np.isfinite(f)
    if mu is not None:
        mu = np.asarray(mu, dtype=float).ravel()[order]
        good &= np.isfinite(mu)
    runs, start = [], None
    for i, g in enumerate(good):
        if g and start is None:
            start = i
        if (not g or i == len(good) - 1) and start is not None:
            runs.append((start, i + 1 if g else i))
            start = None
    runs = [r for r in runs if r[1] - r[0] >= min_points]
    if not runs:
        raise ValueError(f"tabulated_branch {name!r}: no run of >= {min_points} finite points")
    i, j = max(runs, key=lambda r: r[1] - r[0])
    if mu is not None:
        spl = CubicHermiteSpline(phi[i:j], f[i:j], mu[i:j])
    else:
        spl = CubicSpline(phi[i:j], f[i:j], bc_type="not-a-knot")
    d1, d2 = spl.derivative(1), spl.derivative(2)
    return Branch(name, spl, d1, d2, float(phi[i]) - float(extend_lo), float(phi[j - 1]), kind="tabulated")


@dataclass
class Tangent:
    phi_a: float
    phi_b: float
    mu: float
    omega: float

    @property
    def ok(self):
        return bool(np.isfinite(self.phi_a) and np.isfinite(self.phi_b))


NO_TANGENT = Tangent(float("nan"), float("nan"), float("nan"), float("nan"))


def _inverse(br, piece, m):
    a, b = piece
    return brentq(lambda p: float(br.mu(p)) - m, a, b, xtol=1e-15, rtol=4 * np.finfo(float).eps, maxiter=200)


def _omega(br, piece, m):
    p = _inverse(br, piece, m)
    return float(br.f(p)) - m * p, p


def common_tangent(a: Branch, b: Branch, n_scan=400) -> Tangent:
    """The common tangent between branches a and b (phase_diagram/common_tangent.py:522),
    or NO_TANGENT. Among several, the one with the lowest grand potential."""
    found = []
    for pa in a.convex_pieces():
        for pb in b.convex_pieces():
            ma = sorted((float(a.mu(pa[0])), float(a.mu(pa[1]))))
            mb = sorted((float(b.mu(pb[0])), float(b.mu(pb[1]))))
            lo, hi = max(ma[0], mb[0]), min(ma[1], mb[1])
            if not hi > lo:
                continue
            span = hi - lo
            ms = np.linspace(lo + 1e-12 * span, hi - 1e-12 * span, n_scan)

            def dw(m):
                return _omega(a, pa, m)[0] - _omega(b, pb, m)[0]

            vals = np.array([dw(m) for m in ms])
            for k in range(len(ms) - 1):
                if np.sign(vals[k]) != np.sign(vals[k + 1]) or vals[k] == 0:
                    m = brentq(dw, ms[k], ms[k + 1], xtol=1e-16, rtol=4 * np.finfo(float).eps, maxiter=200)
                    wa, phia = _omega(a, pa, m)
                    _, phib = _omega(b, pb, m)
                    if abs(phia - phib) > 1e-9:
                        found.append(Tangent(phia, phib, m, wa))
    if not found:
        return NO_TANGENT
    return min(found, key=lambda t: t.omega)


# ---- stdPFC (Gamma = beta = q0 = 1, g = 0, epsilon = r) uniform branch:
# models/stdpfc_cpu/phase_diagram.py:301-320 with v0 = 1
def std_liquid_branch(r, lo=-1.0, hi=1.0, beta=1.0, q0=1.0, g=0.0):
    c = beta * q0 ** 4 + r
    return analytic_branch("liquid",
                           lambda p: 0.5 * c * np.asarray(p) ** 2 + g / 3 * np.asarray(p) ** 3 + 0.25 * np.asarray(p) ** 4,
                           lambda p: c * np.asarray(p) + g * np.asarray(p) ** 2 + np.asarray(p) ** 3,
                           lo, hi, d2f=lambda p: c + 2 * g * np.asarray(p) + 3 * np.asarray(p) ** 2)
