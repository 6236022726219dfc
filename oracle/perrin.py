"""ORACLE (test infrastructure only): Perrin's analytic friction of a triaxial ellipsoid with stick
boundary conditions, the physics check of BEST's results on an ellipsoid mesh.

F. Perrin, "Mouvement brownien d'un ellipsoide (I)", J. Phys. Radium 5, 497 (1934); the rotational
coefficients as corrected by S. H. Koenig, "Brownian motion of an ellipsoid. A correction to
Perrin's results", Biopolymers 14, 2421 (1975).  For semi-axes a_1, a_2, a_3 and
    Delta(s) = sqrt((a_1^2 + s)(a_2^2 + s)(a_3^2 + s)),
    chi      = int_0^inf ds / Delta(s)                     = 2 R_F(a_1^2, a_2^2, a_3^2),
    alpha_i  = int_0^inf ds / ((a_i^2 + s) Delta(s))        = (2/3) R_D(a_j^2, a_k^2, a_i^2),
(R_F, R_D: Carlson's symmetric elliptic integrals, B. C. Carlson, Numer. Algorithms 10, 13 (1995))
the friction for translation along axis i and rotation about it are
    f_i = 16 pi eta / (chi + a_i^2 alpha_i),
    F_i = 16 pi eta (a_j^2 + a_k^2) / (3 (a_j^2 alpha_j + a_k^2 alpha_k)),
and D_t,i = kT / f_i, D_r,i = kT / F_i.  BEST reports D_t = (1/3) Tr D_tt in cm^2/s and
D_r = (1/3) Tr D_rr in 1/s at T = 293.15 K and eta = 0.01002 P (best/output.f:16-29).
A sphere of radius a gives the Stokes-Einstein values kT / (6 pi eta a) and kT / (8 pi eta a^3).
"""
import math

import numpy as np
from scipy.special import elliprd, elliprf

KB = 1.38066e-16      # erg / K, as BEST's output.f
TEMPERATURE = 293.15  # K
ETA = 0.01002         # P


def perrin(axes_angstrom):
    """(D_t cm^2/s, D_r 1/s, per-axis D_t (3,), per-axis D_r (3,)) for the ellipsoid with the given
    semi-axes in Angstrom."""
    a = np.asarray(axes_angstrom, dtype=np.float64) * 1e-8  # cm
    a2 = a * a
    chi = 2.0 * elliprf(a2[0], a2[1], a2[2])
    alpha = np.array([(2.0 / 3.0) * elliprd(a2[(i + 1) % 3], a2[(i + 2) % 3], a2[i]) for i in range(3)])
    kt = KB * TEMPERATURE
    f = 16.0 * math.pi * ETA / (chi + a2 * alpha)
    F = np.array([16.0 * math.pi * ETA * (a2[j] + a2[k]) / (3.0 * (a2[j] * alpha[j] + a2[k] * alpha[k]))
                  for j, k in ((1, 2), (2, 0), (0, 1))])
    dt = kt / f
    dr = kt / F
    return float(dt.mean()), float(dr.mean()), dt, dr
