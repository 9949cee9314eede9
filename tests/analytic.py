"""Analytic reference solutions used by the reference's own tests.

``sod_exact`` restates the exact Riemann solver of test/test_sod3d.jl:80-142
(Toro section 4.2); ``run_sod_3d`` restates the runner of test_sod3d.jl:146-215
around a pluggable ``step``/``cfl_dt`` pair so the same driver exercises the
oracle and the CUDA path.
"""
import math

import numpy as np

NG = 3


def sod_exact(x, t, gamma=1.4):
    rL, vL, pL = 1.0, 0.0, 1.0
    rR, vR, pR = 0.125, 0.0, 0.1
    g = gamma
    csL = math.sqrt(g * pL / rL)
    csR = math.sqrt(g * pR / rR)

    def fk(p, rK, pK, csK):
        if p > pK:
            AK = 2 / ((g + 1) * rK)
            BK = (g - 1) / (g + 1) * pK
            sq = math.sqrt(AK / (p + BK))
            return (p - pK) * sq, sq * (1 - (p - pK) / (2 * (p + BK)))
        fv = 2 * csK / (g - 1) * ((p / pK) ** ((g - 1) / (2 * g)) - 1)
        dv = (p / pK) ** (-(g + 1) / (2 * g)) / (rK * csK)
        return fv, dv

    p = 0.5 * (pL + pR)
    for _ in range(100):
        fL, dfL = fk(p, rL, pL, csL)
        fR, dfR = fk(p, rR, pR, csR)
        dp = (fL + fR + vR - vL) / (dfL + dfR)
        p = max(1e-12, p - dp)
        if abs(dp) / p < 1e-12:
            break
    fL, _ = fk(p, rL, pL, csL)
    fR, _ = fk(p, rR, pR, csR)
    v_star = 0.5 * (vL + vR) + 0.5 * (fR - fL)
    r_starL = (rL * (p / pL + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * p / pL + 1) if p > pL
               else rL * (p / pL) ** (1 / g))
    r_starR = (rR * (p / pR + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * p / pR + 1) if p > pR
               else rR * (p / pR) ** (1 / g))
    if p > pL:
        SL_shock = vL - csL * math.sqrt((g + 1) / (2 * g) * p / pL + (g - 1) / (2 * g))
        SL_head = SL_tail = SL_shock
    else:
        SL_head = vL - csL
        SL_tail = v_star - math.sqrt(g * p / r_starL)
        SL_shock = SL_head
    SR = (vR + csR * math.sqrt((g + 1) / (2 * g) * p / pR + (g - 1) / (2 * g)) if p > pR else vR + csR)
    ro, vo, po = np.zeros(len(x)), np.zeros(len(x)), np.zeros(len(x))
    for k, xk in enumerate(x):
        xi = xk / t if t > 0 else math.copysign(math.inf, xk)
        if p > pL:
            if xi < SL_shock:
                ro[k], vo[k], po[k] = rL, vL, pL
            elif xi < v_star:
                ro[k], vo[k], po[k] = r_starL, v_star, p
            elif xi < SR:
                ro[k], vo[k], po[k] = r_starR, v_star, p
            else:
                ro[k], vo[k], po[k] = rR, vR, pR
        else:
            if xi < SL_head:
                ro[k], vo[k], po[k] = rL, vL, pL
            elif xi < SL_tail:
                cs_fan = (2 * csL + (g - 1) * (vL - xi)) / (g + 1)
                vo[k] = xi + cs_fan
                ro[k] = rL * (cs_fan / csL) ** (2 / (g - 1))
                po[k] = pL * (ro[k] / rL) ** g
            elif xi < v_star:
                ro[k], vo[k], po[k] = r_starL, v_star, p
            elif xi < SR:
                ro[k], vo[k], po[k] = r_starR, v_star, p
            else:
                ro[k], vo[k], po[k] = rR, vR, pR
    return ro, vo, po


def sod_errors(U, direction, dims, d_cell, t_end, gamma=1.4, n_trans=4):
    """L1 errors of test/test_sod3d.jl:182-214 for a finished run."""
    ax = "xyz".index(direction)
    n_cells = dims[ax]
    rho = np.zeros(n_cells)
    vel = np.zeros(n_cells)
    prs = np.zeros(n_cells)
    for i in range(n_cells):
        if direction == "x":
            vals = [U[:, NG + i, NG + j, NG] for j in range(n_trans)]
        elif direction == "y":
            vals = [U[:, NG, NG + i, NG + j] for j in range(n_trans)]
        else:
            vals = [U[:, NG, NG + j, NG + i] for j in range(n_trans)]
        row = sum(vals) / len(vals)
        rv = row[0]
        mn = row[1 + ax]
        E = row[4]
        rho[i] = rv
        vel[i] = mn / max(rv, 1e-30)
        prs[i] = (gamma - 1) * (E - 0.5 * mn ** 2 / max(rv, 1e-30))
    xs = np.array([-0.5 + (i + 0.5) * d_cell for i in range(n_cells)])
    re, ve, pe = sod_exact(xs, t_end, gamma)
    buf = 5
    s = slice(buf, n_cells - buf)
    return (np.sum(np.abs(rho[s] - re[s])) * d_cell, np.sum(np.abs(vel[s] - ve[s])) * d_cell,
            np.sum(np.abs(prs[s] - pe[s])) * d_cell)
