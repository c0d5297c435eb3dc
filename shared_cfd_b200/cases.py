"""Synthetic workloads with the shapes of the benchmark configurations.

All inputs are generated here from seeds; no dataset is read.

* sod(...)            Sod shock tube, 400x4 cells, ideal gas, MUSCL + SLAU,
                      explicit Euler at CFL 0.5 with a global dt.
* flat_plate(...)     supersonic laminar flat plate, 256x128 cells, N2 ideal
                      gas with Sutherland viscosity and Pr 0.72, LU-SGS with
                      local time stepping.
* reacting_step(...)  axisymmetric backward-facing step with a central H2 jet,
                      4 blocks (2 x 512x512 + 2 x 512x256 at scale 1), 9
                      species and 19 seeded reversible reactions, NR dual time
                      with dt = 1e-7 s and 20 inner iterations, chemistry split.
* forward_step(...)   two-block ideal-gas case in the four orientations of the
                      reference's forward-step samples (halo exchange checks).
* reactor_batch(...)  constant-volume H2/air 0-D reactors on the reacting-step
                      mechanism: T0 uniform in [900, 1600] K, p uniform in
                      [1, 20] atm, equivalence ratio uniform in [0.3, 3.0].
"""
import math
import os

import numpy as np

from . import abi
from . import chem as CH
from . import formats as F
from .solver import Case

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def base_desc(ny=1, dim=abi.DIM_2D, dt_mode=abi.DT_GLOBAL, scheme=abi.SCHEME_EULER, viscous=0,
              thermo=abi.THERMO_IDEAL, cfl=0.5):
    d = abi.Desc()
    d.abi_version = abi.ABI_VERSION
    d.ny = ny
    d.dim = dim
    d.dt_mode = dt_mode
    d.scheme = scheme
    d.recon = abi.RECON_MUSCL
    d.viscous = viscous
    d.thermo = thermo
    d.mu_model = abi.MU_REFERENCE
    d.precision = abi.PREC_FP64
    d.quirk_q1 = 1
    d.num_internal_loop = 21
    d.phi_mus, d.k_mus = 1.0, 1.0 / 3.0           # control.part.inp defaults: order 3
    d.kappa, d.rgas, d.nu_gas = 1.4, 287.0, 1.6e-5  # checkout_flow.py:216-221 defaults
    d.suth_mu0, d.suth_t0, d.suth_s = 1.663e-5, 273.15, 106.7
    d.prandtl, d.schmidt = 1.0, 1.0
    d.cfl = cfl
    d.dt_fixed = 0.0
    d.omega_max, d.omega_min, d.dq_max = 1e-1, 1e-3, 1e-2   # NR/q2d/control.part.inp
    d.res_rate_warn, d.res_rate_err = 1e-5, 1e-3
    d.chem_max_substeps = 100000
    d.cfl_tau = 1e-2                                        # dual/2d/control.part.inp
    return d


def rect_plane(xs, rs):
    """Node arrays of a rectangular block from 1-D node coordinates."""
    xh = np.repeat(np.asarray(xs, dtype=np.float64)[:, None], len(rs), axis=1)
    rh = np.repeat(np.asarray(rs, dtype=np.float64)[None, :], len(xs), axis=0)
    return xh, rh


def bc(plane, side, first, last, kind, value=()):
    b = abi.BC()
    b.plane, b.side, b.first, b.last, b.kind = plane, side, first, last, kind
    for k, v in enumerate(value):
        b.value[k] = v
    return b


def ideal_state(case, rho, u, v, p):
    """q, w, vhi of a calorically perfect state (ideal thermal model)."""
    d = case.desc
    kg, Rg = d.kappa, d.rgas
    T = p / (rho * Rg)
    E = p / (kg - 1.0) + 0.5 * rho * (u * u + v * v)
    q = np.array([rho, rho * u, rho * v, E])
    w = np.zeros(case.W)
    w[0], w[1], w[2], w[3], w[4] = rho, u, v, p, 1.0
    w[case.D + 1] = kg
    w[case.D + 2] = (E + p) / rho
    w[case.D + 3] = Rg
    if d.mu_model == abi.MU_SUTHERLAND:
        w[case.D + 4] = d.suth_mu0 * (T / d.suth_t0) ** 1.5 * (d.suth_t0 + d.suth_s) / (T + d.suth_s)
    else:
        w[case.D + 4] = rho * d.nu_gas
    vhi = np.array([kg / (kg - 1.0) * Rg * T])
    return q, w, vhi


def fill_all(case, p, q, w, vhi):
    case.q[p, :, :, :] = q
    case.w[p, :, :, :] = w
    case.vhi[p, :, :, :] = vhi


def all_sides(planes_ij, kind, value=()):
    out = []
    for p, (ni, nj) in enumerate(planes_ij):
        out += [bc(p + 1, abi.SIDE_ILO, 1, nj, kind, value), bc(p + 1, abi.SIDE_IHI, 1, nj, kind, value),
                bc(p + 1, abi.SIDE_JLO, 1, ni, kind, value), bc(p + 1, abi.SIDE_JHI, 1, ni, kind, value)]
    return out


# ---------------------------------------------------------------------------
def sod(ni=400, nj=4, precision=abi.PREC_FP64):
    """Sod shock tube: x in [0,1], dx = dy = 1/ni; left rho=1,p=1, right
    rho=0.125, p=0.1, u=0 (nondimensional values used as given)."""
    xs = np.linspace(0.0, 1.0, ni + 1)
    rs = np.arange(nj + 1) / ni
    planes = [rect_plane(xs, rs)]
    d = base_desc(cfl=0.5)
    d.precision = precision
    case = Case(planes, d, bcs=all_sides([(ni, nj)], abi.BC_EXTRAP))
    ql, wl, vl = ideal_state(case, 1.0, 0.0, 0.0, 1.0)
    qr, wr, vr = ideal_state(case, 0.125, 0.0, 0.0, 0.1)
    for i in range(-1, ni + 3):
        left = i <= ni // 2
        case.q[0, :, i + 1] = ql if left else qr
        case.w[0, :, i + 1] = wl if left else wr
        case.vhi[0, :, i + 1] = vl if left else vr
    case.steps = 200
    case.name = "sod_%dx%d" % (ni, nj)
    return case


def plate_nodes_y(nj, dy1=1e-6, ratio=1.05, height=0.02):
    """Wall-normal nodes: geometric spacing dy1*ratio**k while the remaining
    height can still be covered by the remaining cells at no smaller spacing,
    then uniform spacing up to `height` (so the last node is exactly height)."""
    ys = [0.0]
    dy = dy1
    m = 0
    while m < nj:
        rest = nj - m
        if (height - ys[-1]) / rest <= dy:
            break
        ys.append(ys[-1] + dy)
        dy *= ratio
        m += 1
    rest = nj - m
    if rest > 0:
        step = (height - ys[-1]) / rest
        y0 = ys[-1]
        for k in range(1, rest + 1):
            ys.append(y0 + step * k)
    ys[-1] = height
    return np.array(ys)


def flat_plate(ni=256, nj=128, cfl=1.0, precision=abi.PREC_FP64, wall_start=0.005):
    """Laminar supersonic flat plate of N2: M=2, T=300 K, p=10 kPa.  The
    configuration names no CFL number; at 1.0 the LU-SGS local-time-step run
    converges over its 5000 iterations (at 2.0 it diverges near iteration 750,
    in the CUDA path and the CPU restatement alike)."""
    xs = np.linspace(0.0, 0.1, ni + 1)
    ys = plate_nodes_y(nj)
    planes = [rect_plane(xs, ys)]
    d = base_desc(dt_mode=abi.DT_LOCAL, scheme=abi.SCHEME_LUSGS, viscous=1, cfl=cfl)
    d.rgas = 296.8
    d.mu_model = abi.MU_SUTHERLAND
    d.prandtl = 0.72
    d.precision = precision
    case = Case(planes, d)
    T, p = 300.0, 1e4
    rho = p / (d.rgas * T)
    a = math.sqrt(d.kappa * d.rgas * T)
    u = 2.0 * a
    q, w, vhi = ideal_state(case, rho, u, 0.0, p)
    fill_all(case, 0, q, w, vhi)
    xc = 0.5 * (xs[1:] + xs[:-1])
    iw = int(np.argmax(xc >= wall_start)) + 1  # first no-slip cell
    fixed = list(w) + list(vhi)
    case.bcs = [
        bc(1, abi.SIDE_ILO, 1, nj, abi.BC_FIXED, fixed),
        bc(1, abi.SIDE_IHI, 1, nj, abi.BC_EXTRAP),
        bc(1, abi.SIDE_JLO, 1, iw - 1, abi.BC_SLIP),
        bc(1, abi.SIDE_JLO, iw, ni, abi.BC_NOSLIP, (0.0, 0.0)),
        bc(1, abi.SIDE_JHI, 1, ni, abi.BC_EXTRAP),
    ]
    case.steps = 5000
    case.name = "flat_plate_%dx%d" % (ni, nj)
    return case


# ---------------------------------------------------------------------------
# H2 / air mechanism with seeded Arrhenius parameters
# ---------------------------------------------------------------------------
SPECIES9 = ["H2", "O2", "H2O", "H", "O", "OH", "HO2", "H2O2", "N2"]
REACTIONS19 = [
    "H+O2=O+OH", "O+H2=H+OH", "OH+H2=H+H2O", "OH+OH=O+H2O", "H+H+M=H2+M", "O+O+M=O2+M", "H+O+M=OH+M",
    "H+OH+M=H2O+M", "H+O2+M=HO2+M", "HO2+H=H2+O2", "HO2+H=OH+OH", "HO2+O=O2+OH", "HO2+OH=H2O+O2",
    "HO2+HO2=H2O2+O2", "H2O2+M=OH+OH+M", "H2O2+H=H2O+OH", "H2O2+H=HO2+H2", "H2O2+O=OH+HO2",
    "H2O2+OH=HO2+H2O",
]


def seeded_chem_inp(seed=20240607, a_range=(10.0, 17.0), beta_range=(-1.0, 1.0), ea_kcal=(0.0, 30.0)):
    """chem.inp text: 9 species with the NASA-7 data shipped in data/, and 19
    element-conserving reversible reactions with A log-uniform in a_range
    (mol-cm-s), beta uniform in beta_range and Ea uniform in ea_kcal."""
    rng = np.random.default_rng(seed)
    with open(os.path.join(DATA, "h2air9_thermo.dat")) as f:
        thermo = f.read().rstrip("\n").splitlines()
    out = ["elements", " H O N", "end", "species", " " + " ".join(SPECIES9), "end", "thermo all"]
    out += thermo
    out += ["end", "reactions      cal/mole  moles"]
    for r in REACTIONS19:
        A = 10.0 ** rng.uniform(*a_range)
        beta = rng.uniform(*beta_range)
        ea = rng.uniform(*ea_kcal) * 1000.0
        out.append(" %-28s %10.3E %8.3f %10.1f" % (r, A, beta, ea))
    out.append("end")
    return "\n".join(out) + "\n"


def control_chem_text(po, To, ox, pf, Tf, fuel, rtol=1e-6, atol=1e-6):
    def blk(comp):
        return "\n".join("%s %g" % (k, v) for k, v in comp.items())
    return ("#Control parameters for chemistry\n"
            "Oxidizer Pressure(Pa)   : %-15.7e\n" % po +
            "Oxidizer Temperature(K) : %-15.7e\n" % To +
            "Oxygen Composition(mole ratio):\n" + blk(ox) + "\nend\n" +
            "Fuel Pressure(Pa)       : %-15.7e\n" % pf +
            "Fuel Temperature(K)     : %-15.7e\n" % Tf +
            "Fuel Composition(mole ratio):\n" + blk(fuel) + "\nend\n" +
            "Relative Torelance VODE : %-15.7e\n" % rtol +
            "Absolute Torelance VODE : %-15.7e\n" % atol)


def with_trace(comp, trace):
    """A control_chem.inp composition (mole ratios) in which every species of
    SPECIES9 that the stream lacks appears at `trace` times the stream's total
    ratio."""
    if trace <= 0.0:
        return dict(comp)
    tot = sum(comp.values())
    out = dict(comp)
    for sp in SPECIES9:
        out.setdefault(sp, trace * tot)
    return out


def h2air_mechanism(seed=20240607, po=1e5, To=1500.0, pf=1e5, Tf=300.0, trace=0.0, **kw):
    """(Mechanism, fuel/oxidiser states) after the reference's set-up.  trace > 0
    lists every absent species in both stream compositions of control_chem.inp
    at that mole ratio (relative to the stream), so no species starts at zero."""
    m = CH.parse_chem(seeded_chem_inp(seed, **kw), open(os.path.join(DATA, "elements_mw.dat")).read())
    CH.parse_trans(open(os.path.join(DATA, "h2air9_trans.dat")).read(), m)
    comp = CH.parse_control_chem(control_chem_text(po, To, with_trace({"O2": 1, "N2": 3.76}, trace), pf, Tf,
                                                   with_trace({"H2": 1}, trace)), m)
    fo = CH.fuel_oxidizer(m, comp, len(m.species))
    return m, fo


def moving_state(st, u, v, D):
    """q, w of a fuel / oxidiser state of read_fo_composition given a velocity
    (as set_IC of sample/no27.chemkin_reaction/condition.f90:1-28 does)."""
    q = st["q"].copy()
    w = st["w"].copy()
    rho = w[0]
    q[D - 3] = rho * u
    q[D - 2] = rho * v
    q[D - 1] = st["q"][D - 1] + 0.5 * rho * (u * u + v * v)
    w[1], w[2] = u, v
    w[D + 2] = st["w"][D + 2] + 0.5 * (u * u + v * v)
    return q, w


def reacting_step(scale=1.0, seed=20240607, precision=abi.PREC_FP64, inner=20, dt=1e-7, mech_kw=None, trace=0.0,
                  omega_max=0.1, checks="relaxed", wake="air"):
    """Axisymmetric backward-facing step with a central H2 jet.

    Blocks (x axial, r radial, axis r=0; at scale 1 the cell counts are exact):
      1  upstream air annulus    x in [-0.02, 0],  r in [0.010, 0.020]  512 x 512
      2  downstream outer        x in [ 0, 0.04],  r in [0.010, 0.020]  512 x 512
      3  downstream jet core     x in [ 0, 0.04],  r in [0, 0.005]      512 x 256
      4  downstream step wake    x in [ 0, 0.04],  r in [0.005, 0.010]  512 x 256
    Air (O2:N2 = 1:3.76) enters block 1 at 1500 K, M = 2; H2 enters block 3
    at 300 K and 1200 m/s through the step face r < 0.005; r in [0.005, 0.01]
    of the step face and r = 0.01 upstream are no-slip walls; r = 0.02 is a
    slip wall; r = 0 is the axis; x = 0.04 is a supersonic outflow.

    trace: mole ratio of every absent species in both streams (h2air_mechanism).
    omega_max: control.inp "InternalLoop Omega Max".
    checks: "reference" keeps the shipped "InternalLoop Omega Min" (1e-3) and
    "ResRateErr" (1e-3) of NR/q2d/control.part.inp, so a step whose omega
    falls below 1e-3 or whose inner residual does not drop three orders stops
    with E_OMEGA / E_RESRATE as the reference stops; "relaxed" lowers Omega Min
    to 1e-8 and turns ResRateErr off (the impulsive start from the uniform
    initial state needs both).
    wake: "air" fills block 4 with air at rest; "premixed" with a
    stoichiometric H2 / air mixture at rest at 1500 K, which ignites, so the
    chemistry's intervals there run out of CHEMEQ2 attempts and go to DVODE."""
    n = lambda k: max(4, int(round(k * scale)))
    n512, n256 = n(512), n(256)
    h1, h, H, Lu, Lx = 0.005, 0.010, 0.020, 0.02, 0.04
    xu = np.linspace(-Lu, 0.0, n512 + 1)
    xd = np.linspace(0.0, Lx, n512 + 1)
    r_out = np.linspace(h, H, n512 + 1)
    r_core = np.linspace(0.0, h1, n256 + 1)
    r_wake = np.linspace(h1, h, n256 + 1)
    planes = [rect_plane(xu, r_out), rect_plane(xd, r_out), rect_plane(xd, r_core), rect_plane(xd, r_wake)]
    # the connectivity generator compares text-parsed coordinates
    planes = F.roundtrip_plot3d_values(planes)
    m, fo = h2air_mechanism(seed, trace=trace, **(mech_kw or {}))
    ns = len(m.species)
    d = base_desc(ny=ns, dim=abi.DIM_Q2D, dt_mode=abi.DT_FIXED, scheme=abi.SCHEME_NR, viscous=1,
                  thermo=abi.THERMO_CHEMKIN_REACTIVE)
    d.dt_fixed = dt
    d.num_internal_loop = inner + 1
    d.omega_max = omega_max
    if checks == "relaxed":
        d.res_rate_err = 1e300
        d.omega_min = 1e-8
    elif checks != "reference":
        raise ValueError("checks must be 'reference' or 'relaxed'")
    d.precision = precision
    cut, _ = F.connectivity(planes)
    case = Case(planes, d, cut=cut, chem=CH.to_struct(m))
    case.mech = m
    D = case.D
    ox, fu = fo["o"], fo["f"]
    a_ox = math.sqrt(ox["kappa"] * ox["p"] / ox["rho"])
    u_air = 2.0 * a_ox
    q_air, w_air = moving_state(ox, u_air, 0.0, D)
    q_h2, w_h2 = moving_state(fu, 1200.0, 0.0, D)
    q_rest, w_rest = moving_state(ox, 0.0, 0.0, D)
    # blocks 1-2 hold the moving air, block 3 the jet, block 4 air at rest
    fill_all(case, 0, q_air, w_air, ox["vhi"])
    fill_all(case, 1, q_air, w_air, ox["vhi"])
    fill_all(case, 2, q_h2, w_h2, fu["vhi"])
    if wake == "premixed":
        comp = CH.parse_control_chem(control_chem_text(1e5, 1500.0, {"H2": 2, "O2": 1, "N2": 3.76}, 1e5, 300.0,
                                                       {"H2": 1}), m)
        pre = CH.fuel_oxidizer(m, comp, ns)["o"]
        q_pre, w_pre = moving_state(pre, 0.0, 0.0, D)
        fill_all(case, 3, q_pre, w_pre, pre["vhi"])
    elif wake == "air":
        fill_all(case, 3, q_rest, w_rest, ox["vhi"])
    else:
        raise ValueError("wake must be 'air' or 'premixed'")
    air = list(w_air) + list(ox["vhi"])
    h2 = list(w_h2) + list(fu["vhi"])
    case.bcs = [
        bc(1, abi.SIDE_ILO, 1, n512, abi.BC_FIXED, air),
        bc(3, abi.SIDE_ILO, 1, n256, abi.BC_FIXED, h2),
        bc(4, abi.SIDE_ILO, 1, n256, abi.BC_NOSLIP, (0.0, 0.0)),
        bc(2, abi.SIDE_IHI, 1, n512, abi.BC_EXTRAP),
        bc(3, abi.SIDE_IHI, 1, n256, abi.BC_EXTRAP),
        bc(4, abi.SIDE_IHI, 1, n256, abi.BC_EXTRAP),
        bc(1, abi.SIDE_JLO, 1, n512, abi.BC_NOSLIP, (0.0, 0.0)),
        bc(3, abi.SIDE_JLO, 1, n512, abi.BC_SLIP),
        bc(1, abi.SIDE_JHI, 1, n512, abi.BC_SLIP),
        bc(2, abi.SIDE_JHI, 1, n512, abi.BC_SLIP),
    ]
    case.steps = 500
    case.name = "reacting_step_%g" % scale
    case.states = fo
    return case


# ---------------------------------------------------------------------------
def forward_step(orientation=0, n=12, scheme=abi.SCHEME_EULER, dt_mode=abi.DT_GLOBAL, viscous=0,
                 dim=abi.DIM_2D, precision=abi.PREC_FP64):
    """Two ideal-gas blocks joined along one edge, in one of four layouts
    that give the i-i, j-j, j-i and i-j (reversed) interfaces of the
    reference's forward-step samples no06-no09."""
    L = 1.0
    a = np.linspace(0.0, L, n + 1)
    b = np.linspace(L, 2 * L, 2 * n + 1)
    c = np.linspace(0.2, 0.2 + L, n + 1)
    if orientation == 0:      # i-i: block 2 continues block 1 in x
        planes = [rect_plane(a, c), rect_plane(b, c)]
    elif orientation == 1:    # j-j: block 2 on top of block 1
        planes = [rect_plane(c, a), rect_plane(c, b)]
    elif orientation == 2:    # j-i: block 1's j-hi edge meets block 2's i-lo edge
        xh1, rh1 = rect_plane(c, a)
        # block 2 above: i runs down along r (right-handed with j along x),
        # so its i-hi edge lies on block 1's j-hi edge
        xs = c
        rs = b[::-1]
        xh2 = np.repeat(xs[None, :], len(rs), axis=0)
        rh2 = np.repeat(rs[:, None], len(xs), axis=1)
        planes = [(xh1, rh1), (xh2, rh2)]
    else:                     # i-j reversed: block 2's j-lo edge runs against block 1's i-hi edge
        xh1, rh1 = rect_plane(a, c)
        rs = c[::-1]
        xs = b
        xh2 = np.repeat(xs[None, :], len(rs), axis=0)
        rh2 = np.repeat(rs[:, None], len(xs), axis=1)
        planes = [(xh1, rh1), (xh2, rh2)]
    planes = F.roundtrip_plot3d_values(planes)
    d = base_desc(dim=dim, dt_mode=dt_mode, scheme=scheme, viscous=viscous, cfl=0.4)
    d.precision = precision
    cut, tsm = F.connectivity(planes)
    case = Case(planes, d, cut=cut)
    bcs = []
    for p in range(2):
        for cind in range(2):
            for lu in range(2):
                side = [abi.SIDE_ILO, abi.SIDE_IHI, abi.SIDE_JLO, abi.SIDE_JHI][cind * 2 + lu]
                for lo, hi in tsm[p][cind][lu]:
                    bcs.append(bc(p + 1, side, lo, hi, abi.BC_EXTRAP))
    case.bcs = bcs
    for p in range(2):
        q, w, vhi = ideal_state(case, 1.0, 50.0, 10.0, 1e5)
        fill_all(case, p, q, w, vhi)
    case.name = "forward_step_%d" % orientation
    return case


def adjoint_channel(n=24, steps=60, mach=0.5, seed=3, cfl=0.25):
    """Two ideal-gas blocks joined i-i (the first forward-step layout): a fixed
    inflow (descriptor 0, plane 1 i-lo) slightly off the initial state, slip walls
    at j-lo and j-hi, zero-gradient outflow (plane 2 i-hi); a seeded smooth
    perturbation of the initial state; explicit Euler, inviscid, fixed dt at
    acoustic CFL 0.25 (forward Euler with MUSCL lets this perturbed flow grow
    unboundedly at 0.4 within 60 steps).  The case of the discrete adjoint
    (scfd_adjoint_run)."""
    L = 1.0
    a = np.linspace(0.0, L, n + 1)
    b = np.linspace(L, 2 * L, 2 * n + 1)
    c = np.linspace(0.2, 0.2 + L, n + 1)
    planes = F.roundtrip_plot3d_values([rect_plane(a, c), rect_plane(b, c)])
    d = base_desc(dt_mode=abi.DT_FIXED, scheme=abi.SCHEME_EULER, viscous=0)
    cut, _ = F.connectivity(planes)
    case = Case(planes, d, cut=cut)
    rho, p = 1.2, 1e5
    snd = math.sqrt(1.4 * p / rho)
    d.dt_fixed = cfl * (L / n) / (snd * (1.0 + mach))
    for pl in range(2):
        q, w, vhi = ideal_state(case, rho, mach * snd, 0.0, p)
        fill_all(case, pl, q, w, vhi)
    perturb(case, seed=seed, amp=0.02)
    qi, wi, vi = ideal_state(case, 1.02 * rho, 1.05 * mach * snd, 0.02 * snd, 1.01 * p)
    case.bcs = [bc(1, abi.SIDE_ILO, 1, n, abi.BC_FIXED, list(wi) + list(vi)),
                bc(2, abi.SIDE_IHI, 1, n, abi.BC_EXTRAP),
                bc(1, abi.SIDE_JLO, 1, n, abi.BC_SLIP), bc(1, abi.SIDE_JHI, 1, n, abi.BC_SLIP),
                bc(2, abi.SIDE_JLO, 1, 2 * n, abi.BC_SLIP), bc(2, abi.SIDE_JHI, 1, 2 * n, abi.BC_SLIP)]
    case.steps = steps
    case.name = "adjoint_channel_%d" % n
    return case


def split_planes_i(case, k):
    """The same case with every plane cut along i into k pieces of (nearly)
    equal width, joined again by i-i block interfaces that the connectivity
    generator finds (the pieces share their cut node columns exactly).  The
    boundary descriptors, the initial state (ghost layers included) and the
    chemistry carry over; the LU-SGS sweeps then stop at the cuts, as they do
    at the sub-domain edges of the reference's MPI decomposition."""
    if k <= 1:
        return case
    planes, origin = [], []  # origin[n] = (plane, a, b): interior columns a+1..b
    for p, (xh, rh) in enumerate(case.planes):
        ni = xh.shape[0] - 1
        cuts = [int(round(m * ni / k)) for m in range(k + 1)]
        if min(b - a for a, b in zip(cuts, cuts[1:])) < 2:
            raise ValueError("plane %d (ni=%d) is too narrow for %d pieces" % (p + 1, ni, k))
        for a, b in zip(cuts, cuts[1:]):
            planes.append((xh[a:b + 1].copy(), rh[a:b + 1].copy()))
            origin.append((p, a, b))
    if len(planes) > abi.MAX_PLANES:
        raise ValueError("%d planes exceed the %d of the ABI" % (len(planes), abi.MAX_PLANES))
    desc = abi.Desc.from_buffer_copy(case.desc)
    cut, _ = F.connectivity(planes)
    new = Case(planes, desc, cut=cut, chem=case.chem)
    for b in case.bcs:
        pieces = [(n, a, e) for n, (p, a, e) in enumerate(origin) if p == b.plane - 1]
        if b.side == abi.SIDE_ILO:
            targets = [(pieces[0][0], b.first, b.last)]
        elif b.side == abi.SIDE_IHI:
            targets = [(pieces[-1][0], b.first, b.last)]
        else:
            targets = [(n, max(b.first, a + 1) - a, min(b.last, e) - a) for n, a, e in pieces]
            targets = [t for t in targets if t[1] <= t[2]]
        for n, lo, hi in targets:
            nb = abi.BC.from_buffer_copy(b)
            nb.plane, nb.first, nb.last = n + 1, lo, hi
            new.bcs.append(nb)
    for n, (p, a, b) in enumerate(origin):
        nj, ni = case.nj[p], b - a
        for dst, src in ((new.q, case.q), (new.w, case.w), (new.vhi, case.vhi)):
            dst[n, :nj + 4, :ni + 4] = src[p, :nj + 4, a:b + 4]
    for attr in ("mech", "steps", "states"):
        if hasattr(case, attr):
            setattr(new, attr, getattr(case, attr))
    new.name = "%s_i%d" % (getattr(case, "name", "case"), k)
    return new


def perturb(case, seed=1, amp=0.05):
    """Seeded smooth perturbation of the initial state (density, velocity,
    pressure for the ideal gas; temperature and mixing for chemistry) so that
    every term of the residual is exercised."""
    rng = np.random.default_rng(seed)
    D = case.D
    for p in range(len(case.planes)):
        ni, nj = case.ni[p], case.nj[p]
        xh, rh = case.planes[p]
        jj, ii = np.meshgrid(np.arange(-1, nj + 3), np.arange(-1, ni + 3), indexing="ij")
        ph = rng.uniform(0, 2 * np.pi, size=4)
        f1 = np.sin(2 * np.pi * ii / max(ni, 1) + ph[0]) * np.cos(2 * np.pi * jj / max(nj, 1) + ph[1])
        f2 = np.cos(2 * np.pi * ii / max(ni, 1) + ph[2]) * np.sin(2 * np.pi * jj / max(nj, 1) + ph[3])
        q = case.q[p, :nj + 4, :ni + 4]
        rho = q[:, :, :case.nY].sum(axis=2)
        u = q[:, :, case.nY] / rho
        v = q[:, :, case.nY + 1] / rho
        ke = 0.5 * rho * (u * u + v * v)
        e_int = q[:, :, D - 1] - ke
        s = 1.0 + amp * f1
        q[:, :, :case.nY] *= s[:, :, None]
        rho2 = rho * s
        u2 = u * (1.0 + amp * f2) + amp * 0.1 * np.sqrt(np.abs(e_int / rho)) * f1
        v2 = v + amp * 0.1 * np.sqrt(np.abs(e_int / rho)) * f2
        q[:, :, case.nY] = rho2 * u2
        q[:, :, case.nY + 1] = rho2 * v2
        q[:, :, D - 1] = e_int * (1.0 + 0.5 * amp * f2) + 0.5 * rho2 * (u2 * u2 + v2 * v2)
        w = case.w[p, :nj + 4, :ni + 4]
        w[:, :, 0] = rho2
        w[:, :, 1] = u2
        w[:, :, 2] = v2
        w[:, :, 3] = w[:, :, 3] * (1.0 + 0.5 * amp * f2)
    return case


ATM = 101325.0


def reactor_batch(n=8192, seed=20240611, mech_seed=20240607, T_range=(900.0, 1600.0), p_atm=(1.0, 20.0),
                  phi_range=(0.3, 3.0)):
    """Initial states of n constant-volume H2/air reactors.

    Mole fractions H2 : O2 : N2 = 2 phi : 1 : 3.76; the partial densities follow
    from p and T0 as rho_rel2abs (sub_chem.f90:1036-1085) forms them from
    relative densities (here the mass fractions).  Returns (mechanism, scfd_chem,
    T0[n], vrho0[n][ns], draws) with draws = (T0, p [Pa], phi)."""
    m, _ = h2air_mechanism(mech_seed)
    ns = len(m.species)
    rng = np.random.default_rng(seed)
    T0 = rng.uniform(T_range[0], T_range[1], n)
    p = rng.uniform(p_atm[0], p_atm[1], n) * ATM
    phi = rng.uniform(phi_range[0], phi_range[1], n)
    idx = {s.strip().upper(): k for k, s in enumerate(m.species)}
    mw = np.asarray(m.mws)
    vrho = np.zeros((n, ns))
    for r in range(n):
        X = np.zeros(ns)
        X[idx["H2"]] = 2.0 * phi[r]
        X[idx["O2"]] = 1.0
        X[idx["N2"]] = 3.76
        Y = X * mw
        Y = Y / Y.sum()
        _, _, v = CH.rho_rel2abs(m, p[r], T0[r], list(Y))
        vrho[r] = v
    return m, CH.to_struct(m), T0, vrho, (T0, p, phi)
