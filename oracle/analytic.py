"""ORACLE — test infrastructure only.

Analytic H-wave in the 1 m PEC box, restated from the reference's own known
answer (analytic_value_excite_h, src/DGA/Utilities.hpp:393-510, with the
Bessel integrals of src/DGA/bessel.cpp, lossless case).  The H source on
the z = 0 face drives the TE10 mode sin(pi x / a); each field amplitude obeys
the Klein-Gordon equation u_tt - c^2 u_zz + alpha^2 u = 0 with cut-off
alpha = pi c / a, whose signalling solution for u(0, t) = sin(w t) is, at
delay k = z / c,

    u(t, k) = sin(w (t - k)) - alpha k Int_k^t J1(alpha sqrt(tau^2 - k^2))
              / sqrt(tau^2 - k^2) sin(w (t - tau)) d tau      (t > k; else 0).

The PEC face at z = a_z adds image waves at delays (4 j a_z + z) / c (+),
(4 j a_z + 2 a_z + z) / c (-), (4 j a_z + 2 a_z - z) / c (+) and
(4 j a_z + 4 a_z - z) / c (-), j = 0, 1, ...; Hx = sin(pi x / a) times their
sum.  The integral is evaluated with scipy's adaptive quadrature where the
reference uses GSL's qags.
"""
from __future__ import annotations

import math

C0 = 299792458.0


def signal(t: float, k: float, alpha: float, w: float) -> float:
    """u(t, k) above."""
    from scipy import integrate, special

    if t <= k:
        return 0.0
    if k == 0.0:
        return math.sin(w * t)

    def f(tau):
        r = math.sqrt(tau * tau - k * k)
        return special.j1(alpha * r) / r * math.sin(w * (t - tau))

    val, _ = integrate.quad(f, k, t, limit=400, epsabs=1e-12, epsrel=1e-9)
    return math.sin(w * (t - k)) - alpha * k * val


def hx(x: float, z: float, t: float, freq: float, c: float = C0, a: float = 1.0, az: float = 1.0) -> float:
    """Hx of the analytic H-wave at (x, z) and time t (amplitude 1 source)."""
    alpha = math.pi * c / a
    w = 2.0 * math.pi * freq
    s = 0.0
    j = 0
    while True:
        waves = ((+1.0, (z + 4 * az * j) / c), (-1.0, (4 * az * j + 2 * az + z) / c),
                 (+1.0, (4 * az * j + 2 * az - z) / c), (-1.0, (4 * az * j + 4 * az - z) / c))
        live = [(sg, k) for sg, k in waves if t > k]
        if not live:
            break
        for sg, k in live:
            s += sg * signal(t, k, alpha, w)
        j += 1
    return math.sin(math.pi * x / a) * s
