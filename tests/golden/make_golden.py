"""Generates tests/golden/scb_exact.json: exact solutions of the SCB discrete equations for tiny cases.

The reference ships no golden vectors for its sweep, and its corner solver (LA_TOOLS.GAUSS_COMPLETE)
is not available, so these fixtures come from the discrete equations themselves: every input is a
double, converted exactly to a rational, and the sweep of TRANSPORT_SOLVES.f08:45-242 (the matrix of
SCB_BGEN, :332-371) and the moment sums of COLLAPSE_INTENSITIES (:441-509) are evaluated in exact
rational arithmetic (fractions.Fraction), then rounded once to double.  Any correct floating-point
implementation must agree with them to a few ulp times the conditioning of the 4x4 systems.

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import math
import os
from fractions import Fraction as Fr

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def lqn4():
    # LQ_4 first quadrant (mu1 = 0.3500212), equal weights; cosines from the level-symmetric relation
    m1 = 0.3500212
    m2 = math.sqrt(1.0 - 2.0 * m1 * m1)
    ox1 = [m1, m2, m1]
    oy1 = [m1, m1, m2]
    return ox1, oy1, [1.0, 1.0, 1.0]


def expand(ox1, oy1, w1):
    ox = np.array(ox1 + [-x for x in ox1] + [-x for x in ox1] + ox1)
    oy = np.array(oy1 + oy1 + [-y for y in oy1] + [-y for y in oy1])
    w = np.array(w1 * 4, dtype=np.float64)
    w = 4.0 * math.pi * w / np.sum(w)
    return ox, oy, w


def solve4(B, Q):
    n = 4
    M = [[B[r][c] for c in range(n)] + [Q[r]] for r in range(n)]
    for k in range(n):
        p = max(range(k, n), key=lambda r: abs(M[r][k]))
        M[k], M[p] = M[p], M[k]
        for r in range(k + 1, n):
            f = M[r][k] / M[k][k]
            for c in range(k, n + 1):
                M[r][c] -= f * M[k][c]
    x = [Fr(0)] * n
    for k in reversed(range(n)):
        x[k] = (M[k][n] - sum(M[k][c] * x[c] for c in range(k + 1, n))) / M[k][k]
    return x


def exact_case(name, nx, ny, ng, quad, seed, c=2.99792458e2, dt=2e-3):
    rng = np.random.default_rng(seed)
    ox, oy, w = quad
    nm = len(ox)
    dx = rng.uniform(0.2, 0.8, nx)
    dy = rng.uniform(0.2, 0.8, ny)
    A = np.outer(dx, dy)
    kap = 10 ** rng.uniform(-1, 2, (nx, ny, ng))
    src = rng.uniform(0.0, 2.0, (nx, ny, ng))
    iold = rng.uniform(0.0, 2.0, (2 * nx, 2 * ny, nm, ng))
    bV = rng.uniform(0.0, 3.0, (2, 2 * ny, nm, ng))     # inflow corner-edge values, faces x=0 / x=nx
    bH = rng.uniform(0.0, 3.0, (2, 2 * nx, nm, ng))     # faces y=0 / y=ny
    F = Fr
    rcdt = F(1) / (F(c) * F(dt))
    q = nm // 4
    Icrn = {}
    # corner-edge values: V[(f, iy, m, g)], H[(ix, f, m, g)]
    V, H = {}, {}
    for g in range(ng):
        for m in range(nm):
            for iy in range(2 * ny):
                V[(0, iy, m, g)] = F(bV[0, iy, m, g])
                V[(nx, iy, m, g)] = F(bV[1, iy, m, g])
            for ix in range(2 * nx):
                H[(ix, 0, m, g)] = F(bH[0, ix, m, g])
                H[(ix, ny, m, g)] = F(bH[1, ix, m, g])
    for g in range(ng):
        for quadn in range(4):
            fx = quadn in (1, 2)
            fy = quadn in (2, 3)
            for m in range(quadn * q, (quadn + 1) * q):
                Ox, Oy = F(ox[m]), F(oy[m])
                for jj in range(ny):
                    j = ny - 1 - jj if fy else jj
                    for ii in range(nx):
                        i = nx - 1 - ii if fx else ii
                        kE = F(kap[i, j, g]) + rcdt
                        Dx, Dy, Aij = F(dx[i]), F(dy[j]), F(A[i, j])
                        area = Dx * Dy
                        gam = (abs(Ox) * Dy + abs(Oy) * Dx + kE * area) / 4
                        a, b = Ox * Dy / 4, Oy * Dx / 4
                        B = [[gam, a, 0, b], [-a, gam, b, 0], [0, -b, gam, -a], [-b, 0, a, gam]]
                        S = {}
                        for cx in range(2):
                            for cy in range(2):
                                S[(cx, cy)] = F(src[i, j, g]) + F(iold[2 * i + cx, 2 * j + cy, m, g]) * rcdt
                        # inflow terms: the faces the reference reads for this quadrant (:72-76 etc.)
                        vL_b, vL_t = V.get((i, 2 * j, m, g)), V.get((i, 2 * j + 1, m, g))
                        vR_b, vR_t = V.get((i + 1, 2 * j, m, g)), V.get((i + 1, 2 * j + 1, m, g))
                        hB_l, hB_r = H.get((2 * i, j, m, g)), H.get((2 * i + 1, j, m, g))
                        hT_l, hT_r = H.get((2 * i, j + 1, m, g)), H.get((2 * i + 1, j + 1, m, g))
                        Q = [Aij * S[(0, 0)] / 4, Aij * S[(1, 0)] / 4, Aij * S[(1, 1)] / 4, Aij * S[(0, 1)] / 4]
                        if not fx:
                            Q[0] += Ox * Dy * vL_b / 2
                            Q[3] += Ox * Dy * vL_t / 2
                        else:
                            Q[1] -= Ox * Dy * vR_b / 2
                            Q[2] -= Ox * Dy * vR_t / 2
                        if not fy:
                            Q[0] += Oy * Dx * hB_l / 2
                            Q[1] += Oy * Dx * hB_r / 2
                        else:
                            Q[3] -= Oy * Dx * hT_l / 2
                            Q[2] -= Oy * Dx * hT_r / 2
                        x = solve4(B, Q)
                        Icrn[(2 * i, 2 * j, m, g)] = x[0]
                        Icrn[(2 * i + 1, 2 * j, m, g)] = x[1]
                        Icrn[(2 * i + 1, 2 * j + 1, m, g)] = x[2]
                        Icrn[(2 * i, 2 * j + 1, m, g)] = x[3]
                        if not fx:
                            V[(i + 1, 2 * j, m, g)] = x[1]
                            V[(i + 1, 2 * j + 1, m, g)] = x[2]
                        else:
                            V[(i, 2 * j, m, g)] = x[0]
                            V[(i, 2 * j + 1, m, g)] = x[3]
                        if not fy:
                            H[(2 * i, j + 1, m, g)] = x[3]
                            H[(2 * i + 1, j + 1, m, g)] = x[2]
                        else:
                            H[(2 * i, j, m, g)] = x[0]
                            H[(2 * i + 1, j, m, g)] = x[1]
    # outputs in Fortran layouts
    I_crn = np.zeros((2 * nx, 2 * ny, nm, ng), order="F")
    for k, v in Icrn.items():
        I_crn[k] = float(v)
    I_avg = np.zeros((nx, ny, nm, ng), order="F")
    I_avgF = {}
    for g in range(ng):
        for m in range(nm):
            for j in range(ny):
                for i in range(nx):
                    v = (Icrn[(2 * i, 2 * j, m, g)] + Icrn[(2 * i + 1, 2 * j, m, g)] + Icrn[(2 * i + 1, 2 * j + 1, m, g)]
                         + Icrn[(2 * i, 2 * j + 1, m, g)]) / 4
                    I_avgF[(i, j, m, g)] = v
                    I_avg[i, j, m, g] = float(v)
    I_edgVF = {(f, j, m, g): (V[(f, 2 * j, m, g)] + V[(f, 2 * j + 1, m, g)]) / 2
               for f in range(nx + 1) for j in range(ny) for m in range(nm) for g in range(ng)}
    I_edgHF = {(i, f, m, g): (H[(2 * i, f, m, g)] + H[(2 * i + 1, f, m, g)]) / 2
               for i in range(nx) for f in range(ny + 1) for m in range(nm) for g in range(ng)}
    comp_unit = 1e13
    eps = F(1e-25) / F(comp_unit)
    cl = F(2.99792458e2)
    Wf = [F(x) for x in w]
    Oxf = [F(x) for x in ox]
    Oyf = [F(x) for x in oy]

    def msum(I, key, fn):
        return sum(fn(m) * (I[key(m)] + eps) for m in range(nm))

    Eg_avg = np.zeros((nx, ny, ng), order="F")
    fxx = np.zeros((nx, ny, ng), order="F")
    fyy = np.zeros((nx, ny, ng), order="F")
    fxy = np.zeros((nx, ny, ng), order="F")
    for g in range(ng):
        for j in range(ny):
            for i in range(nx):
                e = msum(I_avgF, lambda m: (i, j, m, g), lambda m: Wf[m]) / cl
                hxx = msum(I_avgF, lambda m: (i, j, m, g), lambda m: Oxf[m] * Oxf[m] * Wf[m])
                hyy = msum(I_avgF, lambda m: (i, j, m, g), lambda m: Oyf[m] * Oyf[m] * Wf[m])
                hxy = msum(I_avgF, lambda m: (i, j, m, g), lambda m: Oxf[m] * Oyf[m] * Wf[m])
                Eg_avg[i, j, g] = float(e)
                fxx[i, j, g] = float(hxx / (cl * e))
                fyy[i, j, g] = float(hyy / (cl * e))
                fxy[i, j, g] = float(hxy / (cl * e))
    Eg_edgV = np.zeros((nx + 1, ny, ng), order="F")
    Fxg_edgV = np.zeros((nx + 1, ny, ng), order="F")
    for g in range(ng):
        for j in range(ny):
            for f in range(nx + 1):
                Eg_edgV[f, j, g] = float(msum(I_edgVF, lambda m: (f, j, m, g), lambda m: Wf[m]) / cl)
                Fxg_edgV[f, j, g] = float(msum(I_edgVF, lambda m: (f, j, m, g), lambda m: Oxf[m] * Wf[m]))
    Eg_edgH = np.zeros((nx, ny + 1, ng), order="F")
    for g in range(ng):
        for f in range(ny + 1):
            for i in range(nx):
                Eg_edgH[i, f, g] = float(msum(I_edgHF, lambda m: (i, f, m, g), lambda m: Wf[m]) / cl)
    Ic_edgV = np.zeros((nx + 1, 2 * ny, nm, ng), order="F")
    for k, v in V.items():
        Ic_edgV[k] = float(v)
    Ic_edgH = np.zeros((2 * nx, ny + 1, nm, ng), order="F")
    for k, v in H.items():
        Ic_edgH[k] = float(v)

    def enc(a):
        return np.asarray(a, dtype=np.float64).ravel(order="F").tolist()

    return dict(name=name, nx=nx, ny=ny, nm=nm, ng=ng, c=c, dt=dt, comp_unit=comp_unit,
                Omega_x=enc(ox), Omega_y=enc(oy), w=enc(w), dx=enc(dx), dy=enc(dy), A=enc(A), kap=enc(kap),
                src=enc(src), I_crn_old=enc(iold), bV=enc(bV), bH=enc(bH),
                I_crn=enc(I_crn), I_avg=enc(I_avg), Ic_edgV=enc(Ic_edgV), Ic_edgH=enc(Ic_edgH),
                Eg_avg=enc(Eg_avg), fg_avg_xx=enc(fxx), fg_avg_yy=enc(fyy), fg_avg_xy=enc(fxy),
                Eg_edgV=enc(Eg_edgV), Fxg_edgV=enc(Fxg_edgV), Eg_edgH=enc(Eg_edgH))


def main():
    test1d = expand([0.92388, 0.382683], [0.382683, 0.92388], [0.5, 0.5])
    cases = [
        exact_case("cell1x1_1dtest", 1, 1, 1, test1d, 11),
        exact_case("grid2x2_1dtest", 2, 2, 2, test1d, 12),
        exact_case("grid3x2_lq4", 3, 2, 1, expand(*lqn4()), 13),
        exact_case("grid2x3_lq4_thick", 2, 3, 2, expand(*lqn4()), 14, dt=2e-6),
    ]
    with open(os.path.join(HERE, "scb_exact.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": cases}, f)
    print("wrote", len(cases), "cases")


if __name__ == "__main__":
    main()
