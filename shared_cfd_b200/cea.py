"""CEA equilibrium thermochemistry through the C ABI (scfd_cea_*).

    from shared_cfd_b200 import cea
    data = cea.h2_air_data()                 # NASA-9 tables of the H/O/N set
    with cea.Cea(data) as m:
        info = m.info()                      # fuel / oxidizer stream states
        out = m.solve(rho, Y, e, T, n)       # numpy in, numpy out (copies)
        m.solve_device(rho_d, Y_d, e_d, T_d, n_d, ...)   # torch CUDA tensors

Set-up that runs once (store/therm_lib/NASA/core/sub_chem.f90):
  * set_therm_data (70-171): NASA-9 blocks of thermo.inp, element weights of
    MW.inp, the element counts Ac(i,j),
  * set_trans_data (172-255): single-species viscosity fits of trans.inp (the
    'V' lines; binary-interaction blocks and 'C' lines are skipped),
  * read_fo_composition (256-305): the fuel and oxidizer stream compositions,
    pressures and temperatures.
The per-cell `cea` (sub_chem.f90:1320-1651) and initialize_cea's stream states
run in the library (CUDA kernel, or the CPU restatement when `lib` is it).

Arrays are component-major: Y[2, ncell], n[ns, ncell], Yv / vhi [ns, ncell],
DHi[2, ncell]; n in mol/kg, e in J/kg, T in K, rho in kg/m^3.
"""
import ctypes as C
import os

import numpy as np

from . import abi
from .solver import load_library

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
H2AIR_SPECIES = ["H2", "O2", "H2O", "H", "O", "OH", "HO2", "H2O2", "N2"]
H2AIR_ELEMENTS = ["H", "O", "N"]
HON17_SPECIES = H2AIR_SPECIES + ["N", "NO", "NO2", "N2O", "NH", "NH2", "NH3", "HNO"]


def _fnum(s):
    """A Fortran D/E field read with blanks ignored ('0.7E 00' -> 0.7)."""
    s = s.replace(" ", "").replace("D", "E").replace("d", "E")
    return float(s) if s else 0.0


def parse_mw(text, elements):
    """MW.inp read with '(A2,f10.5)' (set_therm_data, sub_chem.f90:86-95)."""
    mwe = {}
    for ln in text.splitlines():
        name = ln[:2].strip()
        if name in elements and name not in mwe:
            mwe[name] = _fnum(ln[2:12])
    missing = [e for e in elements if e not in mwe]
    if missing:
        raise ValueError("Some elements have not found in MW.inp: %s" % missing)
    return [mwe[e] for e in elements]


def parse_nasa9(text, species, elements):
    """NASA-9 blocks of thermo.inp (set_therm_data, sub_chem.f90:97-147): the
    name line '(A18,A62)', then '(i2,8x,5(a2,f6.2),2x,f13.7)' (sections,
    element counts, MW), then per section '(2(1x,f10.3))' for the range,
    '(5D16.9)' and '(2D16.8,16x,2D16.8)' for co(1:9).  Species not listed are
    skipped; the first block of each listed name is used."""
    lines = text.splitlines()
    i = 0
    while lines[i][:1] == "!":
        i += 1
    i += 2  # 'thermo' and the default-ranges line
    out = {}
    while i < len(lines):
        name = lines[i][:18].strip()
        if lines[i][:3] == "END":
            if len(out) == len(species):
                break
            i += 1
            continue
        nsec = int(lines[i + 1][:2])
        if name in species and name not in out:
            l2 = lines[i + 1]
            ac = [0.0] * len(elements)
            for k in range(5):
                en = l2[10 + 8 * k:12 + 8 * k]
                if en == "  " or not en.strip():
                    break
                cnt = _fnum(l2[12 + 8 * k:18 + 8 * k])
                if en.strip() in elements:
                    ac[elements.index(en.strip())] = cnt
            mw = _fnum(l2[52:65])
            tr, co = [], []
            for l in range(nsec):
                a, b, c = lines[i + 2 + 3 * l:i + 5 + 3 * l]
                tr.append((_fnum(a[1:11]), _fnum(a[12:22])))
                row = [_fnum(b[16 * k:16 * k + 16]) for k in range(5)]
                row += [_fnum(c[0:16]), _fnum(c[16:32]), _fnum(c[48:64]), _fnum(c[64:80])]
                co.append(row)
            out[name] = {"nsec": nsec, "trange": tr, "co": co, "mw": mw, "ac": ac}
        i += 2 + 3 * nsec
    missing = [s for s in species if s not in out]
    if missing:
        raise ValueError("Some species have not found in thermo.inp: %s" % missing)
    return [out[s] for s in species]


def parse_trans(text, species):
    """Single-species viscosity fits of trans.inp (set_trans_data,
    sub_chem.f90:187-240), in file order: name line '(A15,x,A15,3x,A1,I1,A1,I1)',
    'V' lines '(1x,a1,2(f7.1,2x),4e15.8)'.  Returns [(species index, ranges,
    coefficients)]."""
    lines = text.splitlines()
    fits = []
    i = 1
    while i < len(lines):
        ln = lines[i]
        if ln[:1] == "!":
            i += 1
            continue
        if ln[:3] in ("END", "end"):
            break
        name, comment = ln[0:15].strip(), ln[16:31].strip()
        iv, ic = int(ln[35:36]), int(ln[37:38])
        if comment or name not in species:
            i += 1 + iv + ic
            continue
        tr, cf = [], []
        for k in range(iv):
            v = lines[i + 1 + k]
            if v[1:2] != "V":
                raise ValueError("ERROR : ODD FORMAT AT trans.inp")
            tr.append((_fnum(v[2:9]), _fnum(v[11:18])))
            cf.append([_fnum(v[20 + 15 * m:35 + 15 * m]) for m in range(4)])
        fits.append((species.index(name), tr, cf))
        i += 1 + iv + ic
    return fits


def make_data(species, elements, thermo_text, trans_text, mw_text, fuel, oxidizer, pf=1e5, Tf=300.0,
              po=1e5, To=300.0, init_hp=False):
    """scfd_cea_data of a species set; fuel / oxidizer map species names to
    mole ratios (control_chem.inp); init_hp selects initialize_cea('hp') for
    the stream states (default 'uv')."""
    d = abi.CeaData()
    d.abi_version = abi.ABI_VERSION
    d.init_hp = 1 if init_hp else 0
    ns, ne = len(species), len(elements)
    if ns > abi.CEA_MAX_SPECIES or ne > abi.CEA_MAX_ELEMENTS:
        raise ValueError("species set too large")
    d.ns, d.ne = ns, ne
    th = parse_nasa9(thermo_text, species, elements)
    S, L = abi.CEA_MAX_SECTIONS, abi.CEA_MAX_ELEMENTS
    for j, t in enumerate(th):
        d.nsec[j] = t["nsec"]
        d.mw[j] = t["mw"]
        for l in range(t["nsec"]):
            d.trange[(j * S + l) * 2] = t["trange"][l][0]
            d.trange[(j * S + l) * 2 + 1] = t["trange"][l][1]
            for k in range(9):
                d.co[(j * S + l) * 9 + k] = t["co"][l][k]
        for i in range(ne):
            d.ac[j * L + i] = t["ac"][i]
    for i, w in enumerate(parse_mw(mw_text, elements)):
        d.mwe[i] = w
    fits = parse_trans(trans_text, species)
    d.nt = len(fits)
    TS = abi.CEA_MAX_TSECTIONS
    for i, (j, tr, cf) in enumerate(fits):
        d.tr2th[i] = j
        d.ntsec[i] = len(tr)
        for l in range(len(tr)):
            d.trange_t[(i * TS + l) * 2] = tr[l][0]
            d.trange_t[(i * TS + l) * 2 + 1] = tr[l][1]
            for k in range(4):
                d.trans[(i * TS + l) * 4 + k] = cf[l][k]
    d.pf, d.Tf, d.po, d.To = pf, Tf, po, To
    for name, amount in fuel.items():
        d.nf[species.index(name)] = amount
    for name, amount in oxidizer.items():
        d.no[species.index(name)] = amount
    return d


def _rd(name):
    with open(os.path.join(DATA, name)) as f:
        return f.read()


def h2_air_data(pf=1e5, Tf=300.0, po=1e5, To=300.0, fuel=None, oxidizer=None, species=None, init_hp=False):
    """Hydrogen fuel against air (O2 : N2 = 1 : 3.76) over H2 O2 H2O H O OH
    HO2 H2O2 N2 (or `species`, a subset of them) with the NASA-9 tables of the
    reference's NASA/core."""
    return make_data(species or H2AIR_SPECIES, H2AIR_ELEMENTS, _rd("h2air9_nasa9.dat"),
                     _rd("h2air9_nasa_trans.dat"), _rd("elements_mw_nasa.dat"), fuel or {"H2": 1.0},
                     oxidizer or {"O2": 1.0, "N2": 3.76}, pf, Tf, po, To, init_hp)


def hon17_data(pf=1e5, Tf=300.0, po=1e5, To=300.0, fuel=None, oxidizer=None):
    """The hydrogen-air streams over 17 H/O/N species (adds N NO NO2 N2O NH
    NH2 NH3 HNO): more than 12 species, so the library takes its generic
    kernel."""
    return make_data(HON17_SPECIES, H2AIR_ELEMENTS, _rd("hon17_nasa9.dat"), _rd("hon17_nasa_trans.dat"),
                     _rd("elements_mw_nasa.dat"), fuel or {"H2": 1.0}, oxidizer or {"O2": 1.0, "N2": 3.76},
                     pf, Tf, po, To)


def random_states(info, m, seed=0, de=3e6, rho=(0.2, 2.0), T0=1500.0):
    """Seeded cells between the two streams: Y_fuel = u^3 (u uniform), the
    mixed stream energy plus up to `de` J/kg, rho uniform in `rho`."""
    rng = np.random.default_rng(seed)
    yf = rng.uniform(0.0, 1.0, m) ** 3
    Y = np.stack([yf, 1.0 - yf])
    r = rng.uniform(rho[0], rho[1], m)
    e = yf * info.fuel.e + (1.0 - yf) * info.oxidizer.e + rng.uniform(0.0, de, m)
    return r, Y, e, np.full(m, T0)


def energy(data, T, n):
    """Internal energy (J/kg) of composition n[ns, m] (mol/kg) at T[m]: the
    sum of n_j (h_j/RT - 1) R T that `cea` balances (sub_chem.f90:1397-1408)."""
    T = np.asarray(T, dtype=np.float64)
    n = np.asarray(n, dtype=np.float64)
    e = np.zeros_like(T)
    co = np.frombuffer(data.co, dtype=np.float64).reshape(abi.CEA_MAX_SPECIES, abi.CEA_MAX_SECTIONS, 9)
    tr = np.frombuffer(data.trange, dtype=np.float64).reshape(abi.CEA_MAX_SPECIES, abi.CEA_MAX_SECTIONS, 2)
    lt = np.log(T)
    v = np.stack([-1 / T**2, lt / T, np.ones_like(T), T / 2, T**2 / 3, T**3 / 4, T**4 / 5, 1 / T,
                  np.zeros_like(T)])
    for j in range(data.ns):
        ns_ = data.nsec[j]
        s = np.full(T.shape, ns_ - 1)
        for l in range(ns_ - 1, -1, -1):
            s = np.where(tr[j, l, 1] > T, l, s)
        s = np.where(tr[j, 0, 0] > T, 0, s)
        h = np.einsum("k...,...k->...", v, co[j][s])
        e += (h - 1.0) * n[j]
    return e * 8.3144621 * T


class Cea:
    """One species set on one device.  `lib` selects another library with the
    same entry points (the CPU restatement, prefix orc_); the default loads
    the CUDA library and fails if it is missing."""

    def __init__(self, data, lib=None):
        self.lib = lib if lib is not None else load_library()
        self.on_device = self.lib.prefix == "scfd_"
        self.data = data
        self.ns = data.ns
        self.h = C.c_void_p()
        code = self.lib.cea_create(C.byref(data), C.byref(self.h))
        if code:
            raise RuntimeError("cea_create failed: %s" % abi.STATUS_NAMES.get(code, code))

    def close(self):
        if self.h:
            self.lib.cea_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def info(self):
        inf = abi.CeaInfo()
        code = self.lib.cea_info_get(self.h, C.byref(inf))
        if code:
            raise RuntimeError("cea_info_get failed: %d" % code)
        return inf

    def initial_n(self, ncell):
        """n_save of every cell as initialize_cea leaves it: sum(no + nf) / ns."""
        return np.full((self.ns, ncell), self.info().n_init)

    def status(self):
        counts = (C.c_int64 * 2)()
        code = self.lib.cea_status(self.h, counts)
        return code, int(counts[0]), int(counts[1])

    def solve_ptr(self, ncell, rho, Y, e, T, n, mwave=None, kappa=None, mu=None, Yv=None, vhi=None, DHi=None,
                  iters=None, stream=None):
        """scfd_cea_solve on raw pointers (ints or None)."""
        code = self.lib.cea_solve(self.h, int(ncell), rho, Y, e, T, n, mwave, kappa, mu, Yv, vhi, DHi, iters,
                                  stream)
        if code:
            raise RuntimeError("cea_solve failed: %s" % abi.STATUS_NAMES.get(code, code))

    def solve_device(self, rho, Y, e, T, n, mwave=None, kappa=None, mu=None, Yv=None, vhi=None, DHi=None,
                     iters=None, stream=None):
        """Asynchronous solve on torch CUDA tensors (float64, contiguous,
        component-major); enqueued on `stream` (a torch stream) or torch's
        current stream."""
        import torch
        if stream is None:
            stream = torch.cuda.current_stream()

        def p(t):
            return None if t is None else t.data_ptr()
        self.solve_ptr(rho.numel(), p(rho), p(Y), p(e), p(T), p(n), p(mwave), p(kappa), p(mu), p(Yv), p(vhi),
                       p(DHi), p(iters), stream.cuda_stream)

    def solve(self, rho, Y, e, T, n):
        """One `cea` per cell on host arrays; returns a dict of numpy arrays
        (T and n updated copies, plus MWave, kappa, mu, Yv, vhi, DHi, iters)
        and raises on a singular cell (the reference stops there)."""
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        m = rho.size
        ns = self.ns
        arrs = {
            "rho": rho, "Y": np.ascontiguousarray(Y, dtype=np.float64).reshape(2, m),
            "e": np.ascontiguousarray(e, dtype=np.float64).reshape(m),
            "T": np.array(T, dtype=np.float64).reshape(m), "n": np.array(n, dtype=np.float64).reshape(ns, m),
            "MWave": np.zeros(m), "kappa": np.zeros(m), "mu": np.zeros(m), "Yv": np.zeros((ns, m)),
            "vhi": np.zeros((ns, m)), "DHi": np.zeros((2, m)), "iters": np.zeros(m, dtype=np.int32),
        }
        order = ["rho", "Y", "e", "T", "n", "MWave", "kappa", "mu", "Yv", "vhi", "DHi", "iters"]
        if self.on_device:
            import torch
            dev = {k: torch.from_numpy(arrs[k]).cuda() for k in order}
            self.solve_device(*[dev[k] for k in order])
            code, nc, ng = self.status()
            for k in order:
                arrs[k] = dev[k].cpu().numpy()
        else:
            self.solve_ptr(m, *[arrs[k].ctypes.data for k in order])
            code, nc, ng = self.status()
        if code:
            raise RuntimeError("cea: %d cells met a singular matrix twice" % ng)
        arrs["not_converged"] = nc
        return arrs

    def _host_call(self, fn, order, arrs):
        if self.on_device:
            import torch
            dev = {k: (torch.from_numpy(arrs[k]).cuda() if arrs[k] is not None else None) for k in order}
            fn(*[dev[k].data_ptr() if dev[k] is not None else None for k in order])
            code, nc, ng = self.status()
            for k in order:
                if dev[k] is not None:
                    arrs[k] = dev[k].cpu().numpy()
        else:
            fn(*[arrs[k].ctypes.data if arrs[k] is not None else None for k in order])
            code, nc, ng = self.status()
        arrs["not_converged"] = nc
        return arrs

    def solve_hp(self, p, Y, h, T, n):
        """cea_hp per cell at fixed p (Pa) and h (J/kg) on host arrays: returns
        T, n, MWave, kappa, mu, Yv, vhi, iters (sub_chem.f90:1652-1962)."""
        p = np.ascontiguousarray(p, dtype=np.float64)
        m, ns = p.size, self.ns
        arrs = {"p": p, "Y": np.ascontiguousarray(Y, dtype=np.float64).reshape(2, m),
                "h": np.ascontiguousarray(h, dtype=np.float64).reshape(m),
                "T": np.array(T, dtype=np.float64).reshape(m), "n": np.array(n, dtype=np.float64).reshape(ns, m),
                "MWave": np.zeros(m), "kappa": np.zeros(m), "mu": np.zeros(m), "Yv": np.zeros((ns, m)),
                "vhi": np.zeros((ns, m)), "iters": np.zeros(m, dtype=np.int32)}
        order = ["p", "Y", "h", "T", "n", "MWave", "kappa", "mu", "Yv", "vhi", "iters"]

        def fn(*ptr):
            code = self.lib.cea_solve_hp(self.h, m, *ptr, None)
            if code:
                raise RuntimeError("cea_solve_hp failed: %d" % code)
        return self._host_call(fn, order, arrs)

    def solve_tp(self, p, Y, T, n):
        """cea_tp per cell at fixed p (Pa) and T (K) on host arrays: returns n,
        h (J/kg), MWave, kappa, mu, Yv, vhi, iters (sub_chem.f90:1963-2248)."""
        p = np.ascontiguousarray(p, dtype=np.float64)
        m, ns = p.size, self.ns
        arrs = {"p": p, "Y": np.ascontiguousarray(Y, dtype=np.float64).reshape(2, m),
                "T": np.array(T, dtype=np.float64).reshape(m), "n": np.array(n, dtype=np.float64).reshape(ns, m),
                "h": np.zeros(m), "MWave": np.zeros(m), "kappa": np.zeros(m), "mu": np.zeros(m),
                "Yv": np.zeros((ns, m)), "vhi": np.zeros((ns, m)), "iters": np.zeros(m, dtype=np.int32)}
        order = ["p", "Y", "T", "n", "h", "MWave", "kappa", "mu", "Yv", "vhi", "iters"]

        def fn(*ptr):
            code = self.lib.cea_solve_tp(self.h, m, *ptr, None)
            if code:
                raise RuntimeError("cea_solve_tp failed: %d" % code)
        return self._host_call(fn, order, arrs)
