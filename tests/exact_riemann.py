"""Exact solution of the 1-D Riemann problem of an ideal gas (Toro, "Riemann
Solvers and Numerical Methods for Fluid Dynamics", 3rd ed., ch. 4): the star
pressure by Newton iteration on the pressure function, then the sampled
density / velocity / pressure at x/t.  Test infrastructure (a physics check
of the hydro, not a reference restatement)."""
import math

import numpy as np


def _f(p, rk, pk, ck, g):
    if p > pk:  # shock
        a = 2.0 / ((g + 1.0) * rk)
        b = (g - 1.0) / (g + 1.0) * pk
        q = math.sqrt(a / (p + b))
        return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (b + p))
    pr = p / pk  # rarefaction
    f = 2.0 * ck / (g - 1.0) * (pr ** ((g - 1.0) / (2.0 * g)) - 1.0)
    df = 1.0 / (rk * ck) * pr ** (-(g + 1.0) / (2.0 * g))
    return f, df


def star_state(rl, ul, pl, rr, ur, pr, g=1.4):
    cl = math.sqrt(g * pl / rl)
    cr = math.sqrt(g * pr / rr)
    p = max(1e-12, 0.5 * (pl + pr) - 0.125 * (ur - ul) * (rl + rr) * (cl + cr))
    for _ in range(100):
        fl, dfl = _f(p, rl, pl, cl, g)
        fr, dfr = _f(p, rr, pr, cr, g)
        dp = (fl + fr + ur - ul) / (dfl + dfr)
        pn = max(1e-12, p - dp)
        if abs(pn - p) < 1e-14 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _f(p, rl, pl, cl, g)
    fr, _ = _f(p, rr, pr, cr, g)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    return p, u


def sample(x, t, x0, rl, ul, pl, rr, ur, pr, g=1.4):
    """rho, u, p at the positions x (array) at time t."""
    ps, us = star_state(rl, ul, pl, rr, ur, pr, g)
    cl = math.sqrt(g * pl / rl)
    cr = math.sqrt(g * pr / rr)
    out = np.zeros((3, len(x)))
    for n, xx in enumerate(x):
        s = (xx - x0) / t
        if s <= us:  # left of the contact
            if ps > pl:
                sh = ul - cl * math.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if s < sh:
                    out[:, n] = (rl, ul, pl)
                else:
                    r = rl * ((ps / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pl + 1))
                    out[:, n] = (r, us, ps)
            else:
                shl = ul - cl
                csl = cl * (ps / pl) ** ((g - 1) / (2 * g))
                stl = us - csl
                if s < shl:
                    out[:, n] = (rl, ul, pl)
                elif s > stl:
                    out[:, n] = (rl * (ps / pl) ** (1 / g), us, ps)
                else:
                    u = 2 / (g + 1) * (cl + (g - 1) / 2 * ul + s)
                    c = 2 / (g + 1) * (cl + (g - 1) / 2 * (ul - s))
                    r = rl * (c / cl) ** (2 / (g - 1))
                    out[:, n] = (r, u, pl * (c / cl) ** (2 * g / (g - 1)))
        else:
            if ps > pr:
                sh = ur + cr * math.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if s > sh:
                    out[:, n] = (rr, ur, pr)
                else:
                    r = rr * ((ps / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pr + 1))
                    out[:, n] = (r, us, ps)
            else:
                shr = ur + cr
                csr = cr * (ps / pr) ** ((g - 1) / (2 * g))
                str_ = us + csr
                if s > shr:
                    out[:, n] = (rr, ur, pr)
                elif s < str_:
                    out[:, n] = (rr * (ps / pr) ** (1 / g), us, ps)
                else:
                    u = 2 / (g + 1) * (-cr + (g - 1) / 2 * ur + s)
                    c = 2 / (g + 1) * (cr - (g - 1) / 2 * (ur - s))
                    r = rr * (c / cr) ** (2 / (g - 1))
                    out[:, n] = (r, u, pr * (c / cr) ** (2 * g / (g - 1)))
    return out
