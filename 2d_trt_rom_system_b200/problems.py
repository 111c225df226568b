"""Synthetic problem definitions for the sweep: grids, group structures, materials and boundaries.

The reference reads its problem from input/input.inp (MainSrc/INPUTS.f08:10-163) and builds materials
with MATERIAL_UPDATE (MainSrc/UPDATES.f08:110-156): KapE = KapB(T) * multiplier and an isotropic
corner source RT_Src = KapB * Bg(T) (:141-150).  The workloads here are seeded synthetic instances:

  C0  [0,6]^2, 20x20 cells, 17 groups log-spaced on [1e-3, 1e2], S8, kappa0 = 10 (1000 in cells whose
      centre lies in [2,4]^2), c_v = 0.5, Planckian T = 1 on the left, vacuum elsewhere, T0 = 0.01,
      dt = 2e-3.
  C1  256^2 cells, 50 groups, S16, 16 material rectangles from default_rng(1) with
      kappa0 in U{10, 100, 1000}, c_v in U[0.1, 1]; physics and boundaries as C0.
  C2  instance i of 64 from default_rng(2): N in {32,64,96,128,192,256}, G in {17,50}, S8 or S12,
      6 rectangles with kappa0 log-uniform on [1, 1e4], T_bc in U[0.5, 2].
  C4  1024^2 cells, 64 groups, S16, 8 rectangles from default_rng(4), kappa0 log-uniform [1, 1e4].

Units: temperatures and photon energies in units of kT_ref = 1 keV, lengths in cm, time in sh,
c = 2.99792458e2 cm/sh (main.f08:19).  The reference's Planck function takes eV
(TEMP_FUNCTIONS.f08:90-108), so it is called with 1e3 * T and 1e3 * nu; Comp_Unit = 1e13
(input/input.inp [SOLVER_OPTS]).  Opacity: kappa_g(T) = kappa0 (1 - exp(-nu_g/T)) / (nu_g^3 sqrt(T)),
nu_g the geometric mean of the group edges.
"""
import dataclasses
import math

import numpy as np

from . import quadrature

C_LIGHT = 2.99792458e2      # cm/sh, MainSrc/main.f08:19
COMP_UNIT = 1e13            # MainSrc/input/input.inp
KEV = 1e3                   # eV per kT_ref


def sigint(z):
    """sigint of TEMP_FUNCTIONS.f08:114-141 (vectorised)."""
    z = np.asarray(z, dtype=np.float64)
    pi4 = (math.pi * math.pi) * (math.pi * math.pi)

    def low(x):
        return ((x * x) * x) * (1.0 / 3.0 - x / 8.0 + (x * x) / 62.4)

    def high(x):
        return pi4 / 15.0 - np.exp(-x) * (((x * x) * x) + 3.0 * (x * x) + 6.0 * x + 7.28)

    y1 = low(np.float64(1.95))
    y2 = high(np.float64(2.05))
    mid = y1 + (y2 - y1) * (z - 1.95) / (2.05 - 1.95)
    with np.errstate(over="ignore", invalid="ignore"):
        return np.where(z <= 1.95, low(z), np.where(z > 2.05, high(z), mid))


def bg_planck(T_eV, nu_lo_eV, nu_hi_eV, comp_unit=COMP_UNIT):
    """Bg_planck_calc of TEMP_FUNCTIONS.f08:90-108 (vectorised; T in eV)."""
    T = np.asarray(T_eV, dtype=np.float64)
    h, c, erg = 6.62613e-19, 2.99792458e2, 6.24150934e11
    safe = np.where(T <= 1e-15, 1.0, T)
    sig = sigint(nu_hi_eV / safe) - sigint(nu_lo_eV / safe)
    e2 = erg * erg
    sig = sig / ((((h * h) * h) * (c * c)) * (e2 * e2) * comp_unit)
    t2 = safe * safe
    return np.where(T <= 1e-15, 0.0, (2.0 * (t2 * t2)) * sig)


def log_groups(G, lo=1e-3, hi=1e2):
    """G+1 log-spaced group edges (kT_ref units)."""
    return np.logspace(math.log10(lo), math.log10(hi), G + 1)


def opacity(kappa0, T, nu_mid):
    """kappa_g(T) = kappa0 (1 - exp(-nu/T)) / (nu^3 sqrt(T)); kappa0, T (nx,ny); nu_mid (G,) ->
    (nx, ny, G) Fortran-ordered."""
    T = np.asarray(T)[..., None]
    k = np.asarray(kappa0)[..., None] * (-np.expm1(-nu_mid / T)) / (nu_mid ** 3 * np.sqrt(T))
    return np.asfortranarray(k)


@dataclasses.dataclass
class Problem:
    name: str
    nx: int
    ny: int
    xlen: float
    ylen: float
    edges: np.ndarray           # (G+1,) kT_ref units
    quad: str
    kappa0: np.ndarray          # (nx, ny)
    cv: np.ndarray              # (nx, ny)
    T0: float
    bcT: tuple                  # (left, bottom, right, top) in kT_ref
    bc_type: tuple = (0, 0, 0, 0)
    dt: float = 2e-3
    steps: int = 10

    @property
    def ng(self):
        return len(self.edges) - 1

    @property
    def nu_mid(self):
        return np.sqrt(self.edges[:-1] * self.edges[1:])

    @property
    def nu_eV(self):
        return self.edges * KEV

    @property
    def delx(self):
        return np.full(self.nx, self.xlen / self.nx)

    @property
    def dely(self):
        return np.full(self.ny, self.ylen / self.ny)

    def directions(self):
        return quadrature.by_name(self.quad)

    @property
    def nm(self):
        return len(self.directions()[0])

    def updates_per_sweep(self):
        return self.nx * self.ny * self.nm * self.ng

    def material(self, T):
        """KapE_in and the isotropic source KapB*Bg at temperature field T (nx, ny), both
        (nx, ny, G) Fortran-ordered (MATERIAL_UPDATE, UPDATES.f08:130-150, with this opacity law)."""
        T = np.broadcast_to(np.asarray(T, dtype=np.float64), (self.nx, self.ny))
        kap = opacity(self.kappa0, T, self.nu_mid)
        nu = self.nu_eV
        B = bg_planck(T[..., None] * KEV, nu[None, None, :-1], nu[None, None, 1:])
        return kap, np.asfortranarray(kap * B)

    def boundary_planck(self):
        """Planck boundary intensity per (side, group): (4, G) in L, B, R, T order."""
        nu = self.nu_eV
        return np.array([[bg_planck(t * KEV, nu[g], nu[g + 1]) for g in range(self.ng)] for t in self.bcT])


def _paint_rectangles(rng, nx, ny, xlen, ylen, n_rect, draw_kappa, draw_cv):
    kappa0 = np.full((nx, ny), 10.0)
    cv = np.full((nx, ny), 0.5)
    xc = (np.arange(nx) + 0.5) * xlen / nx
    yc = (np.arange(ny) + 0.5) * ylen / ny
    for _ in range(n_rect):
        x0, x1 = np.sort(rng.uniform(0.0, xlen, 2))
        y0, y1 = np.sort(rng.uniform(0.0, ylen, 2))
        k = draw_kappa(rng)
        c = draw_cv(rng)
        mask = ((xc[:, None] >= x0) & (xc[:, None] <= x1)) & ((yc[None, :] >= y0) & (yc[None, :] <= y1))
        kappa0[mask] = k
        cv[mask] = c
    return kappa0, cv


def config0():
    nx = ny = 20
    xc = (np.arange(nx) + 0.5) * 6.0 / nx
    inside = ((xc[:, None] >= 2.0) & (xc[:, None] <= 4.0)) & ((xc[None, :] >= 2.0) & (xc[None, :] <= 4.0))
    kappa0 = np.where(inside, 1000.0, 10.0)
    return Problem("C0", nx, ny, 6.0, 6.0, log_groups(17), "S8", kappa0, np.full((nx, ny), 0.5), 0.01,
                   (1.0, 0.0, 0.0, 0.0), steps=10)


def config1(n=256, groups=50, quad="S16", steps=20):
    rng = np.random.default_rng(1)
    kappa0, cv = _paint_rectangles(rng, n, n, 6.0, 6.0, 16, lambda r: float(r.choice([10.0, 100.0, 1000.0])),
                                   lambda r: float(r.uniform(0.1, 1.0)))
    return Problem("C1", n, n, 6.0, 6.0, log_groups(groups), quad, kappa0, cv, 0.01, (1.0, 0.0, 0.0, 0.0),
                   steps=steps)


def config2_instances(count=64):
    rng = np.random.default_rng(2)
    out = []
    for k in range(count):
        n = int(rng.choice([32, 64, 96, 128, 192, 256]))
        G = int(rng.choice([17, 50]))
        quad = "S8" if rng.uniform() < 0.5 else "S12"
        kappa0, cv = _paint_rectangles(rng, n, n, 6.0, 6.0, 6, lambda r: float(10 ** r.uniform(0.0, 4.0)),
                                       lambda r: float(r.uniform(0.1, 1.0)))
        tbc = float(rng.uniform(0.5, 2.0))
        out.append(Problem(f"C2-{k}", n, n, 6.0, 6.0, log_groups(G), quad, kappa0, cv, 0.01,
                           (tbc, 0.0, 0.0, 0.0), steps=10))
    return out


def config4(n=1024):
    rng = np.random.default_rng(4)
    kappa0, cv = _paint_rectangles(rng, n, n, 6.0, 6.0, 8, lambda r: float(10 ** r.uniform(0.0, 4.0)),
                                   lambda r: float(r.uniform(0.1, 1.0)))
    return Problem("C4", n, n, 6.0, 6.0, log_groups(64), "S16", kappa0, cv, 0.01, (1.0, 0.0, 0.0, 0.0), steps=10)


def random_small(seed, nx, ny, G, quad="S8", bc_type=(0, 0, 0, 0)):
    """Small seeded instance for parity tests: random rectangles, random boundary temperatures."""
    rng = np.random.default_rng(seed)
    kappa0, cv = _paint_rectangles(rng, nx, ny, 1.0 * nx / 10, 1.0 * ny / 10, 3,
                                   lambda r: float(10 ** r.uniform(-1.0, 4.0)), lambda r: float(r.uniform(0.1, 1.0)))
    bcT = tuple(float(rng.uniform(0.2, 1.5)) for _ in range(4))
    return Problem(f"R{seed}", nx, ny, 1.0 * nx / 10, 1.0 * ny / 10, log_groups(G, 1e-2, 10.0), quad, kappa0, cv,
                   0.3, bcT, bc_type=bc_type)


# ---------------------------------------------------------------------------------------------
# Transport-only time stepping (the reference's run_type 'tr_no_qd') with the reference's own
# material: the Fleck-Cummings opacity kapB_calc (TEMP_FUNCTIONS.f08:11-32) scaled per cell by
# Kappa_Mult(Mat(i,j)), Kap0 = 27e9 eV^3/cm (main.f08:22) and the heat capacity of INPUTS.f08:89-121.
# Temperatures and photon energies are in eV.
# ---------------------------------------------------------------------------------------------
KAP0_FC = 27.0 * 1e9


def fc_cv(bcT_left_eV, comp_unit=COMP_UNIT):
    """Cv of INPUTS.f08:121 (with sig_R, aR of :89-90)."""
    h, c, erg = 6.62613e-19, C_LIGHT, 6.24150934e11
    pi = math.pi
    sig_R = 2.0 * pi ** 5 / (15.0 * c ** 2 * h ** 3 * erg ** 4 * comp_unit)
    aR = 4.0 * sig_R / c
    return 0.5917 * aR * bcT_left_eV ** 3 * ((1.38e-16) ** 4 * (11600.0 ** 4) * erg ** 4)


@dataclasses.dataclass
class TimeStepSetup:
    """Inputs of trt_tstep_setup for a Problem: the Problem's grid, groups, quadrature and material map,
    with the reference's Fleck-Cummings physics (kappa_mult = kappa0 / min(kappa0))."""
    nu_eV: np.ndarray
    kappa_mult: np.ndarray
    cv: float
    Kap0: float
    Tini_eV: float
    bcT_eV: tuple
    dt: float


def fc_timestep_setup(prob, Tini_eV=None):
    k0 = np.asarray(prob.kappa0, dtype=np.float64)
    bcT = tuple(t * KEV for t in prob.bcT)
    Tini = prob.T0 * KEV if Tini_eV is None else Tini_eV
    return TimeStepSetup(nu_eV=prob.nu_eV, kappa_mult=np.asfortranarray(k0 / k0.min()),
                         cv=fc_cv(max(bcT[0], 1.0)), Kap0=KAP0_FC, Tini_eV=Tini, bcT_eV=bcT, dt=prob.dt)


def config_timestep_setup(prob, Tini_eV=None):
    """Inputs of trt_tstep_setup for a Problem with its own physics (TRT_LAW_CONFIG): the opacity law
    kappa0 (1 - exp(-nu/T)) / (nu^3 sqrt(T)) with kappa0 passed as kappa_mult, the per-cell c_v (given per
    kT_ref = 1 keV in the radiation-energy unit of the reference's Comp_Unit scaling, converted here to per
    eV, the library's temperature unit), T0 and the boundary temperatures in eV.  Kap0 is unused."""
    bcT = tuple(t * KEV for t in prob.bcT)
    Tini = prob.T0 * KEV if Tini_eV is None else Tini_eV
    return TimeStepSetup(nu_eV=prob.nu_eV, kappa_mult=np.asfortranarray(np.asarray(prob.kappa0, dtype=np.float64)),
                         cv=np.asfortranarray(np.asarray(prob.cv, dtype=np.float64) / KEV), Kap0=0.0, Tini_eV=Tini,
                         bcT_eV=bcT, dt=prob.dt)


def mgqd_inputs(nx, ny, ng, seed=0, theta=1.0, kap_range=(1e-4, 1e4), xlen=6.0, ylen=6.0, dt=2e-3, uniform=False):
    """Seeded synthetic inputs of MLOQD_FV / OLD_MGQD_COEFS (MLOQD_SOLVES.f08:12-362) with the value
    ranges a time step produces: per-group opacities log-uniform over kap_range (thick and thin groups
    side by side, constant on random rectangles), QD factors near 1/3 with small smooth off-diagonal
    parts, boundary factors of magnitude 0.3-0.6 with Cg_Calc's signs, positive energies.  Returns (d, c, dt, theta); d holds every
    input by its reference name (Fortran-ordered) plus Eg_avg/Eg_edgV/Eg_edgH (the initial guess) and
    G_old/Pold_* from the previous-step fields."""
    rng = np.random.default_rng(seed)
    Fo = np.asfortranarray
    dx = np.full(nx, xlen / nx) if uniform else xlen / nx * rng.uniform(0.7, 1.3, nx)
    dy = np.full(ny, ylen / ny) if uniform else ylen / ny * rng.uniform(0.7, 1.3, ny)
    d = {"Delx": dx, "Dely": dy, "A": Fo(np.outer(dx, dy))}
    lo, hi = math.log10(kap_range[0]), math.log10(kap_range[1])
    kap = np.empty((nx, ny, ng))
    for g in range(ng):
        base = 10 ** (hi - (hi - lo) * (g + 0.5) / ng)
        field = np.ones((nx, ny))
        for _ in range(4):
            x0, y0 = rng.integers(0, nx), rng.integers(0, ny)
            field[x0:x0 + max(1, nx // 3), y0:y0 + max(1, ny // 3)] = 10 ** rng.uniform(-1, 1)
        kap[:, :, g] = base * field
    d["KapE"] = Fo(kap)
    d["KapR"] = Fo(kap * rng.uniform(0.8, 1.2, (1, 1, ng)))
    d["Src"] = Fo(kap * rng.uniform(0.5, 2.0, (nx, ny, ng)))

    def smooth(shape, mean, amp):
        s = [np.linspace(0, np.pi * rng.uniform(1, 3), n) for n in shape[:2]]
        phase = rng.uniform(0, 2 * np.pi, shape[2])
        return Fo(mean + amp * np.sin(s[0][:, None, None] + phase) * np.cos(s[1][None, :, None]))
    V, H, Cc = (nx + 1, ny, ng), (nx, ny + 1, ng), (nx, ny, ng)
    for suf in ("", "_old"):
        d["fg_avg_xx" + suf] = smooth(Cc, 1 / 3, 0.05)
        d["fg_avg_yy" + suf] = smooth(Cc, 1 / 3, 0.05)
        d["fg_edgV_xx" + suf] = smooth(V, 1 / 3, 0.06)
        d["fg_edgV_xy" + suf] = smooth(V, 0.0, 0.03)
        d["fg_edgH_yy" + suf] = smooth(H, 1 / 3, 0.06)
        d["fg_edgH_xy" + suf] = smooth(H, 0.0, 0.03)
    for s_ in ("L", "B", "R", "T"):
        n = ny if s_ in "LR" else nx
        # Cg_Calc (MLOQD_SOLVES.f08:367-488) weights by the signed direction cosine of the outgoing
        # directions: negative on the left and bottom faces, positive on the right and top
        d["Cg_" + s_] = Fo(rng.uniform(0.3, 0.6, (n, ng)) * (-1.0 if s_ in "LB" else 1.0))
        d["Eg_in_" + s_] = Fo(rng.uniform(0.0, 1.0, (n, ng)) * (s_ == "L"))
        d["Fg_in_" + s_] = Fo(rng.uniform(0.0, 50.0, (n, ng)) * (s_ == "L"))
    d["Eg_avg_old"] = Fo(rng.uniform(0.5, 1.5, Cc))
    d["Eg_edgV_old"] = Fo(rng.uniform(0.5, 1.5, V))
    d["Eg_edgH_old"] = Fo(rng.uniform(0.5, 1.5, H))
    d["Fxg_edgV_old"] = Fo(rng.uniform(-20, 20, V))
    d["Fyg_edgH_old"] = Fo(rng.uniform(-20, 20, H))
    d["KapE_old"], d["KapR_old"], d["Src_old"] = d["KapE"], d["KapR"], d["Src"]
    d["Eg_avg"] = d["Eg_avg_old"].copy(order="F")
    d["Eg_edgV"] = d["Eg_edgV_old"].copy(order="F")
    d["Eg_edgH"] = d["Eg_edgH_old"].copy(order="F")
    return d, C_LIGHT, dt, theta
