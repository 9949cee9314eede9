"""Sedov-Taylor point-blast similarity solution (spherical, strong shock into
a uniform medium at rest), the exact solution the Sedov workload approaches
(the reference checks its shock radius in test/test_sedov.jl:16-80).

With R(t) = beta (E t^2 / rho0)^(1/5), xi = r / R, the flow is
    v = R' u(xi),  rho = rho0 g(xi),  p = rho0 R'^2 pi(xi),   R' = 2R/(5t),
and mass, momentum and entropy conservation become three ODEs in xi,
    (u - xi) g' + g u'                    = -2 g u / xi
    (u - xi) u' + pi' / g                 =  3/2 u
    (u - xi) (pi'/pi - gamma g'/g)        =  3,
integrated inward from the Rankine-Hugoniot state behind the shock,
u = 2/(gamma+1), g = (gamma+1)/(gamma-1), pi = 2/(gamma+1) at xi = 1.
beta follows from the energy integral
    1 = (4/25) beta^5 * int_0^1 4 pi xi^2 (g u^2 / 2 + pi / (gamma-1)) dxi.
"""
from __future__ import annotations

import functools

import numpy as np


@functools.lru_cache(maxsize=8)
def _profile(gamma: float, n: int = 4000):
    from scipy.integrate import solve_ivp

    def rhs(xi, y):
        g, u, p = y
        a = u - xi
        # linear system for (g', u', p')
        M = np.array([[a, g, 0.0],
                      [0.0, a, 1.0 / g],
                      [-gamma * a / g, 0.0, a / p]])
        b = np.array([-2.0 * g * u / xi, 1.5 * u, 3.0])
        return np.linalg.solve(M, b)

    y1 = [(gamma + 1) / (gamma - 1), 2 / (gamma + 1), 2 / (gamma + 1)]
    xs = np.concatenate([np.linspace(1.0, 0.05, n), np.geomspace(0.05, 1e-4, n // 4)[1:]])
    sol = solve_ivp(rhs, (1.0, xs[-1]), y1, t_eval=xs, rtol=1e-10, atol=1e-13, method="DOP853")
    if not sol.success:
        raise RuntimeError(f"Sedov similarity integration failed: {sol.message}")
    xi = sol.t[::-1]
    g, u, p = (sol.y[i][::-1] for i in range(3))
    f = 4 * np.pi * xi ** 2 * (0.5 * g * u ** 2 + p / (gamma - 1))
    I = float(np.sum(0.5 * (f[1:] + f[:-1]) * np.diff(xi)))
    beta = (25.0 / (4.0 * I)) ** 0.2
    return xi, g, u, p, beta


def sedov_beta(gamma: float) -> float:
    """R(t) = beta (E t^2 / rho0)^(1/5); beta ~ 1.1517 for gamma = 5/3."""
    return _profile(float(gamma))[4]


def sedov_taylor(r, t, *, E, rho0=1.0, gamma=5 / 3, p0=0.0):
    """(rho, v_r, p) of the similarity solution at radii r and time t;
    ambient (rho0, 0, p0) outside the shock."""
    xi_t, g, u, p, beta = _profile(float(gamma))
    r = np.asarray(r, dtype=np.float64)
    R = beta * (E * t * t / rho0) ** 0.2
    Rd = 0.4 * R / t
    xi = r / R
    inside = xi < 1.0
    xq = np.clip(xi, xi_t[0], 1.0)
    rho = np.where(inside, rho0 * np.interp(xq, xi_t, g), rho0)
    v = np.where(inside, Rd * np.interp(xq, xi_t, u), 0.0)
    pr = np.where(inside, rho0 * Rd * Rd * np.interp(xq, xi_t, p), p0)
    return rho, v, pr
