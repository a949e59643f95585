"""Exact log-likelihood of the AR(1) + Gaussian-noise model and its gradient
(Kalman filter with forward-mode derivatives), vectorised over many
parameter sets: the yardstick that particle-filter estimates and their
gradients are reported against.

Model: x_0 ~ N(0, sx^2 / (1 - phi^2)), x_t = phi x_{t-1} + sx eps_t,
y_t = x_t + sy eta_t for t = 1..T (y_0 is not observed).
"""
from __future__ import annotations

import math

import numpy as np


def kalman_ar1(y, phi, sx, sy):
    """y: [F, T + 1] (or [T + 1]); phi, sx, sy: [F] (or scalars).  Returns
    (loglik [F], grad [F, 3]) with grad = d loglik / d (phi, sx, sy)."""
    y = np.atleast_2d(np.asarray(y, dtype=np.float64))
    F = y.shape[0]
    phi = np.broadcast_to(np.asarray(phi, dtype=np.float64), (F,)).copy()
    sx = np.broadcast_to(np.asarray(sx, dtype=np.float64), (F,)).copy()
    sy = np.broadcast_to(np.asarray(sy, dtype=np.float64), (F,)).copy()
    one_m = 1.0 - phi * phi
    m = np.zeros(F)
    P = sx * sx / one_m
    # derivatives of (m, P) with respect to (phi, sx, sy), one row per parameter
    dm = np.zeros((3, F))
    dP = np.stack([2.0 * phi * sx * sx / (one_m * one_m), 2.0 * sx / one_m, np.zeros(F)])
    ll = np.zeros(F)
    g = np.zeros((3, F))
    e_phi = np.array([1.0, 0.0, 0.0])[:, None]
    e_sx = np.array([0.0, 1.0, 0.0])[:, None]
    e_sy = np.array([0.0, 0.0, 1.0])[:, None]
    log2pi = math.log(2.0 * math.pi)
    for t in range(1, y.shape[1]):
        mp = phi * m
        Pp = phi * phi * P + sx * sx
        dmp = phi * dm + e_phi * m
        dPp = phi * phi * dP + e_phi * (2.0 * phi * P) + e_sx * (2.0 * sx)
        S = Pp + sy * sy
        v = y[:, t] - mp
        dS = dPp + e_sy * (2.0 * sy)
        dv = -dmp
        ll += -0.5 * (log2pi + np.log(S) + v * v / S)
        g += -0.5 * (dS / S + 2.0 * v * dv / S - v * v * dS / (S * S))
        K = Pp / S
        dK = dPp / S - Pp * dS / (S * S)
        m = mp + K * v
        P = (1.0 - K) * Pp
        dm = dmp + dK * v + K * dv
        dP = -dK * Pp + (1.0 - K) * dPp
    return ll, g.T
