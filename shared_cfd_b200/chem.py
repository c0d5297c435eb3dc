"""Chemkin input handling on the host: the parts of
store/therm_lib/chemkin/core/sub_chem.f90 that run once at set-up.

* read_cheminp (sub_chem.f90:191-502): elements, species, NASA-7 thermo,
  reactions with third bodies, REV / LOW / TROE auxiliary lines,
* set_trans_data (sub_chem.f90:788-889): trans.inp viscosity fits,
* read_fo_composition (sub_chem.f90:890-1030): control_chem.inp, the fuel and
  oxidiser states, and the species reordering that puts the reactants first
  (quirk Q6; swap_species, sub_chem.f90:1088-1166),
* rho_rel2abs and calc_T (sub_chem.f90:1036-1085, 1507-1645) for those two
  states only.  The per-cell calc_T of the time loop runs on the GPU.
"""
import math

import numpy as np

from . import abi

RU_CGS = 8.3144621e7            # mod_chem.raw.f90:8
INVRC = 1.0 / float(np.float32(1.987))   # mod_chem.raw.f90:9, single-precision literal
R_UNI = 8.3144621e3             # store/core/prmtr.f90:4


def _ffloat(s):
    """A Fortran numeric field read with blanks ignored ('0.6E 00' -> 0.6)."""
    s = s.replace(" ", "")
    if not s:
        return 0.0
    if "E" not in s.upper() and "D" not in s.upper():
        # Fortran exponent without letter, e.g. '1.5-03'
        for k in range(len(s) - 1, 0, -1):
            if s[k] in "+-" and s[k - 1].isdigit():
                s = s[:k] + "E" + s[k:]
                break
    return float(s.replace("D", "E").replace("d", "E"))


def _next_lines(text):
    """next_line (sub_chem.f90:510-531): 100-column lines, '!' comments
    stripped, blank lines skipped."""
    for raw in text.splitlines():
        ln = raw[:100]
        k = ln.find("!")
        if k == 0:
            continue
        if k > 0:
            ln = ln[:k]
        ln = ln.rstrip()
        if ln.strip():
            yield ln


def _fixed(ln, a, b):
    return ln[a:b] if len(ln) > a else ""


class Mechanism:
    """Parsed mechanism in the reference's (1-based) index conventions, before
    the species reordering."""

    def __init__(self):
        self.elements = []
        self.species = []
        self.mwe = {}
        self.mws = []
        self.tthre = []     # [(Tlow, Thigh, Tcommon)]
        self.coeff = []     # [ [hi(7), lo(7)] ]  coeff(:,1)=low, coeff(:,2)=high
        self.reactions = []  # dicts
        self.trans = []     # dicts: tr2th (1-based), nsec, trange, coef
        self.rtol = 0.0
        self.atol = 0.0


def parse_mw(text):
    mwe = {}
    for ln in _next_lines(text):
        toks = ln.split()
        if len(toks) >= 2:
            mwe[toks[0]] = float(toks[-1])
    return mwe


def _tail_numbers(line, num):
    """read_tail_number_arr (sub_chem.f90:489-508): the last num blank-separated
    numbers of the line; returns (values, rest)."""
    vals = [0.0] * num
    for i in range(num - 1, -1, -1):
        line = line.rstrip()
        k = line.rfind(" ")
        vals[i] = _ffloat(line[k + 1:])
        line = line[:k + 1].rstrip()
    if num == 3:
        vals[0] = math.log(vals[0])
        vals[2] = vals[2] * INVRC
    elif num == 4:
        vals[1] = 1.0 / vals[1]
        vals[2] = 1.0 / vals[2]
    return vals, line


def _species_list(side, species):
    """search_SYM loop (sub_chem.f90:566-587): '+'-separated names."""
    out = []
    for tok in side.split("+"):
        name = tok.strip()
        out.append(species.index(name) + 1 if name in species else -1)
    return out


def parse_chem(text, mw_text):
    m = Mechanism()
    mwe_all = parse_mw(mw_text)
    it = _next_lines(text)
    ln = next(it)
    if ln.strip() != "elements":
        raise ValueError("elements declaration not found.")
    for ln in it:
        s = ln.strip()
        if s in ("end", "END"):
            break
        m.elements.extend(s.split())
    for e in m.elements:
        if e not in mwe_all:
            raise ValueError("Error. There is Element which does not exit in MW.inp.")
        m.mwe[e] = mwe_all[e]
    ln = next(it)
    if ln.strip() != "species":
        raise ValueError("species declaration not found.")
    for ln in it:
        s = ln.strip()
        if s in ("end", "END"):
            break
        m.species.extend(s.split())
    ns = len(m.species)
    ln = next(it)
    if ln.strip() != "thermo all":
        raise ValueError("'thermo all' declaration not found.")
    ln = next(it)
    tdef = [_ffloat(_fixed(ln, 0, 10)), _ffloat(_fixed(ln, 10, 20)), _ffloat(_fixed(ln, 20, 30))]
    m.mws = [0.0] * ns
    m.tthre = [None] * ns
    m.coeff = [None] * ns
    found = 0
    for ln in it:
        if ln.strip() in ("end", "END"):
            break
        name = ln[:24].split(" ")[0]
        l2, l3, l4 = next(it), next(it), next(it)
        if name not in m.species:
            continue
        k = m.species.index(name)
        if _fixed(ln, 44, 45) != "G":
            raise ValueError("Error! Other than Gas phase is contained.")
        found += 1
        mw = 0.0
        es = {}
        for f in range(4):
            sym = _fixed(ln, 24 + 5 * f, 26 + 5 * f).strip()
            cnt = _fixed(ln, 26 + 5 * f, 29 + 5 * f).strip()
            if sym:
                es[sym.upper()] = es.get(sym.upper(), 0) + (int(cnt) if cnt else 0)
        sym5 = _fixed(ln, 73, 75).strip()
        if sym5:
            es[sym5.upper()] = es.get(sym5.upper(), 0) + int(_fixed(ln, 75, 78).strip() or 0)
        # MWs = dot_product(ES(:ne,k), MWe(:ne)) in element order
        for e in m.elements:
            mw += es.get(e.upper(), 0) * m.mwe[e]
        m.mws[k] = mw
        tb = [_ffloat(_fixed(ln, 45, 55)), _ffloat(_fixed(ln, 55, 65)), _ffloat(_fixed(ln, 65, 73))]
        m.tthre[k] = tb if tb[0] != 0.0 else list(tdef)
        c = [[0.0] * 7, [0.0] * 7]  # c[0] = coeff(:,1) low, c[1] = coeff(:,2) high
        v2 = [_ffloat(_fixed(l2, 15 * i, 15 * i + 15)) for i in range(5)]
        v3 = [_ffloat(_fixed(l3, 15 * i, 15 * i + 15)) for i in range(5)]
        v4 = [_ffloat(_fixed(l4, 15 * i, 15 * i + 15)) for i in range(4)]
        c[1][0:5] = v2
        c[1][5:7] = v3[0:2]
        c[0][0:3] = v3[2:5]
        c[0][3:7] = v4
        m.coeff[k] = c
    if found != ns:
        raise ValueError("There is species which does not have thermal data.")
    ln = next(it)
    if ln.strip() != "reactions      cal/mole  moles":
        raise ValueError("'reactions' declaration not found.")
    for ln in it:
        s = ln.strip()
        if s in ("end", "END"):
            break
        if s in ("duplicate", "DUPLICATE"):
            continue
        if "/" not in s:
            abe, rest = _tail_numbers(s, 3)
            r = {"abe": abe, "cabe": [0.0, 0.0, 0.0], "troe": [0.0] * 4, "rstate": [0, 0],
                 "exist_m": False, "indm": [], "men": [], "text": rest.strip()}
            if "<=>" in rest:
                lhs, rhs = rest.split("<=>", 1)
            else:
                lhs, rhs = rest.split("=", 1)
            lhs = lhs.strip()
            rhs = rhs.strip()
            if rhs.startswith(">"):
                r["rstate"][0] = 1
                rhs = rhs[1:].strip()
            if "(+M)" in lhs:
                lhs = lhs[:lhs.index("(+M)")].rstrip()
                rhs = rhs[:len(rhs) - 4].rstrip()
                r["exist_m"] = True
            elif "+M" in lhs:
                if lhs.index("+M") + 2 != len(lhs):
                    raise ValueError("Error. +M must be end of each side.")
                lhs = lhs[:-2]
                rhs = rhs[:-2]
                r["exist_m"] = True
                r["rstate"][1] = 4
            r["reac"] = _species_list(lhs, m.species)
            r["prod"] = _species_list(rhs, m.species)
            m.reactions.append(r)
        else:
            r = m.reactions[-1]
            k = s.index("/")
            key = s[:k].strip()
            body = s[k:]
            inner = body[1:body.index("/", 1)]
            if key.upper() == "REV":
                r["rstate"][1] += 1
                r["cabe"], _ = _tail_numbers(inner, 3)
            elif key.upper() == "LOW":
                r["rstate"][1] = 2
                r["cabe"], _ = _tail_numbers(inner, 3)
            elif key.upper() == "TROE":
                r["rstate"][1] = 3
                r["troe"], _ = _tail_numbers(inner, 4)
            else:
                if not r["exist_m"]:
                    raise ValueError("Error at M enhanced")
                toks = s.split("/")
                names, vals = toks[0::2], toks[1::2]
                r["indm"], r["men"] = [], []
                for nm, v in zip(names, vals):
                    nm = nm.strip()
                    r["indm"].append(m.species.index(nm) + 1 if nm in m.species else -1)
                    r["men"].append(_ffloat(v) - 1.0)
    return m


def parse_trans(text, m):
    """set_trans_data (sub_chem.f90:788-889)."""
    lines = text.splitlines()
    k = 1
    m.trans = []
    while k < len(lines):
        ln = lines[k]
        k += 1
        if ln[:1] == "!":
            continue
        if ln[:3] in ("END", "end"):
            break
        sname = ln[0:15].strip()
        comment = ln[16:31].strip()
        iv = int(ln[35:36])
        ic = int(ln[37:38])
        itr = m.species.index(sname) + 1 if sname in m.species else -1
        if comment or itr == -1:
            k += iv + ic
            continue
        tr, co = [], []
        for _ in range(iv):
            v = lines[k]
            k += 1
            if v[1:2] != "V":
                raise ValueError("ERROR : ODD FORMAT AT trans.inp")
            tr.append([_ffloat(v[2:9]), _ffloat(v[11:18])])
            co.append([_ffloat(v[20 + 15 * i:35 + 15 * i]) for i in range(4)])
        k += ic
        m.trans.append({"tr2th": itr, "nsec": iv, "trange": tr, "coef": co})


def parse_control_chem(text, m):
    """read_fo_composition file part (sub_chem.f90:904-936)."""
    lines = text.splitlines()
    k = 1
    po = _ffloat(lines[k][25:40]); k += 1
    To = _ffloat(lines[k][25:40]); k += 1
    k += 1
    no = [0.0] * len(m.species)
    while not lines[k].startswith("end"):
        name, amt = lines[k].split()[:2]
        no[m.species.index(name)] = float(amt)
        k += 1
    k += 1
    pf = _ffloat(lines[k][25:40]); k += 1
    Tf = _ffloat(lines[k][25:40]); k += 1
    k += 1
    nf = [0.0] * len(m.species)
    while not lines[k].startswith("end"):
        name, amt = lines[k].split()[:2]
        nf[m.species.index(name)] = float(amt)
        k += 1
    k += 1
    m.rtol = _ffloat(lines[k][25:40]); k += 1
    m.atol = _ffloat(lines[k][25:40])
    return {"po": po, "To": To, "no": no, "pf": pf, "Tf": Tf, "nf": nf}


# ---------------------------------------------------------------------------
# set-up thermodynamics (host, FP64, reference operation order)
# ---------------------------------------------------------------------------
def _sec(m, k, T):
    return 0 if T <= m.tthre[k][2] else 1


def rho_rel2abs(m, p, T, vrho):
    """sub_chem.f90:1036-1085: relative partial densities -> absolute state."""
    ns = len(m.species)
    n = [vrho[j] * (1.0 / m.mws[j]) for j in range(ns)]
    tmp = 0.0
    for v in n:
        tmp += v
    tmp = tmp * RU_CGS * T
    tmp = p * 1e1 / tmp
    n = [v * tmp for v in n]
    rho = 0.0
    for j in range(ns):
        rho += n[j] * m.mws[j]
    rho = rho * 1e3
    vrho = [n[j] * m.mws[j] * 1e3 for j in range(ns)]
    logT = math.log(T)
    chrt = [1.0, T / 2.0, T * T / 3.0, T * T * T / 4.0, T * T * T * T / 5.0, 1.0 / T, 0.0]
    E = 0.0
    for j in range(ns):
        dh = 0.0
        s = _sec(m, j, T)
        for i in range(7):
            dh = dh + m.coeff[j][s][i] * chrt[i]
        E = E + (dh - 1.0) * n[j]
    E = E * RU_CGS * T / rho / 1e1
    _ = logT
    return rho, E, vrho


def calc_T(m, vrho, rho, E, T):
    """sub_chem.f90:1507-1645 (set-up use only).  Returns
    (T, kappa, MW, DHi, vhi, mu)."""
    ns = len(m.species)
    tmp = rho * 1e-11
    n = [vrho[j] * (1.0 / m.mws[j]) * 1e-3 if vrho[j] > tmp else 0.0 for j in range(ns)]
    Eobj = E * 1e1 * rho / RU_CGS
    k = 1
    while True:
        sec = [_sec(m, j, T) for j in range(ns)]
        T2 = T * T
        T3 = T2 * T
        T4 = T3 * T
        chrt = [1.0, T / 2.0, T2 / 3.0, T3 / 4.0, T4 / 5.0, 1.0 / T]
        ccpr = [1.0, T, T2, T3, T4, 0.0]
        Enow = 0.0
        cvnow = 0.0
        for j in range(ns):
            if n[j] > 0.0:
                de = -1.0
                dcv = -1.0
                for i in range(6):
                    de = de + m.coeff[j][sec[j]][i] * chrt[i]
                    dcv = dcv + m.coeff[j][sec[j]][i] * ccpr[i]
                Enow = Enow + de * n[j]
                cvnow = cvnow + dcv * n[j]
        dT = (Eobj - Enow * T) / cvnow
        if abs(dT) < 1e-8 or (abs(dT) < 1e-4 and abs(T - 1e3) < 1e-4) or k > 1000:
            break
        T = max(100.0, T + dT)
        k += 1
    if k > 1000:
        raise RuntimeError("Error: Exceed max_T_loop at temperature determination iteration")
    sn = 0.0
    for v in n:
        sn += v
    kappa = 1.0 + sn / cvnow
    MW = rho / sn * 1e-3
    tmp = RU_CGS * 1e-4 * T
    DHi, vhi = [], []
    for j in range(ns):
        dh = 0.0
        for i in range(6):
            dh = dh + m.coeff[j][sec[j]][i] * chrt[i]
        DHi.append(tmp * (1.0 / m.mws[j]) * (kappa - (kappa - 1.0) * dh))
        vhi.append(tmp * (1.0 / m.mws[j]) * dh)
    logT = math.log(T)
    invT = 1.0 / T
    cmu = [logT, invT, invT * invT, 1.0]
    muN = []
    for t in m.trans:
        sec_t = -1
        if t["trange"][0][0] > T:
            sec_t = 0
        for l in range(t["nsec"]):
            if t["trange"][l][1] > T:
                sec_t = l
                break
        if sec_t == -1:
            sec_t = t["nsec"] - 1
        if n[t["tr2th"] - 1] > 0.0:
            s = 0.0
            for j in range(4):
                s = s + cmu[j] * t["coef"][sec_t][j]
            muN.append(math.exp(s))
        else:
            muN.append(0.0)
    mu = 0.0
    nt = len(m.trans)
    for i in range(nt):
        if muN[i] > 0.0:
            it = m.trans[i]["tr2th"] - 1
            denom = 0.0
            for j in range(nt):
                if muN[j] > 0.0:
                    jt = m.trans[j]["tr2th"] - 1
                    phi = 0.25 * (1.0 + math.sqrt(muN[i] / muN[j]) * (m.mws[jt] / m.mws[it]) ** 0.25) ** 2 \
                        * math.sqrt(2.0 * m.mws[jt] / (m.mws[it] + m.mws[jt]))
                    denom = denom + n[jt] * phi
            mu = mu + n[it] * muN[i] / denom
    mu = mu * 1e-7
    return T, kappa, MW, DHi, vhi, mu


def swap_species(m, a, b, vectors):
    """swap_species (sub_chem.f90:1088-1166) with 1-based a, b.  `vectors` are
    per-species lists swapped alongside (vrhof, vrhoo, vwf, vwo, vhif, vhio)."""
    if a == b:
        return
    i, j = a - 1, b - 1
    for arr in (m.species, m.tthre, m.coeff, m.mws):
        arr[i], arr[j] = arr[j], arr[i]
    for v in vectors:
        v[i], v[j] = v[j], v[i]

    def sw(x):
        return b if x == a else (a if x == b else x)
    for r in m.reactions:
        r["reac"] = [sw(x) for x in r["reac"]]
        r["prod"] = [sw(x) for x in r["prod"]]
        r["indm"] = [sw(x) for x in r["indm"]]
    for t in m.trans:
        t["tr2th"] = sw(t["tr2th"])


def fuel_oxidizer(m, comp, nY):
    """read_fo_composition computation part (sub_chem.f90:938-991): returns a
    dict with the oxidiser / fuel q, w, vhi vectors after the reordering.
    `comp` comes from parse_control_chem.  m is reordered in place."""
    ns = len(m.species)
    vrhoo = [comp["no"][k] * m.mws[k] for k in range(ns)]
    vrhof = [comp["nf"][k] * m.mws[k] for k in range(ns)]
    out = {}
    states = {}
    for tag, p, T, vr in (("o", comp["po"], comp["To"], vrhoo), ("f", comp["pf"], comp["Tf"], vrhof)):
        rho, E, vra = rho_rel2abs(m, p, T, vr)
        T2, kappa, MW, DHi, vhi, mu = calc_T(m, vra, rho, E, T)
        states[tag] = {"p": p, "rho": rho, "E": E, "T": T2, "kappa": kappa, "MW": MW, "mu": mu,
                       "vrho": vra, "vw": [vra[k] / rho for k in range(nY)] + [0.0] * (ns - nY),
                       "vhi": vhi}
    vo, vf = states["o"], states["f"]
    vecs = [vf["vrho"], vo["vrho"], vf["vw"], vo["vw"], vf["vhi"], vo["vhi"]]
    vsum = [vf["vrho"][k] + vo["vrho"][k] for k in range(ns)]
    reac = [k + 1 for k in range(ns) if vsum[k] != 0.0]
    for i, r in enumerate(reac):
        swap_species(m, i + 1, r, vecs)
    D = nY + 3
    W = D + 5
    for tag in ("o", "f"):
        s = states[tag]
        q = np.zeros(D)
        w = np.zeros(W)
        for i in range(ns):
            q[i] = s["vrho"][i]
            w[i + 4] = s["vrho"][i] / s["rho"]
        q[nY + 2] = s["rho"] * s["E"]
        w[0] = s["rho"]
        w[3] = s["p"]
        w[D + 1] = s["kappa"]
        w[D + 2] = s["E"] + s["p"] / s["rho"]
        w[D + 3] = s["p"] / (s["rho"] * s["T"])
        w[D + 4] = s["mu"]
        out[tag] = {"q": q, "w": w, "vhi": np.array(s["vhi"]), "MW": s["MW"], "T": s["T"],
                    "rho": s["rho"], "E": s["E"], "kappa": s["kappa"], "mu": s["mu"], "p": s["p"]}
    return out


def to_struct(m):
    """scfd_chem for the library (0-based species indices)."""
    ch = abi.Chem()
    ns, nr = len(m.species), len(m.reactions)
    if ns > abi.MAX_SPECIES or nr > abi.MAX_REACTIONS:
        raise ValueError("mechanism exceeds the ABI limits")
    ch.ns, ch.nr, ch.nt = ns, max(nr, 1), len(m.trans)
    for k in range(ns):
        for s in range(2):
            for i in range(7):
                ch.coeff[k][s][i] = m.coeff[k][s][i]
        for i in range(3):
            ch.tthre[k][i] = m.tthre[k][i]
        ch.mws[k] = m.mws[k]
    for i, r in enumerate(m.reactions):
        ch.rstate[i][0], ch.rstate[i][1] = r["rstate"]
        ch.numnu[i][0], ch.numnu[i][1] = len(r["reac"]), len(r["prod"])
        if len(r["reac"]) > 3 or len(r["prod"]) > 3:
            raise ValueError("at most 3 species per side (IndNu(3,2,nr))")
        for k, v in enumerate(r["reac"]):
            ch.indnu[i][0][k] = v - 1
        for k, v in enumerate(r["prod"]):
            ch.indnu[i][1][k] = v - 1
        ch.snu[i] = len(r["prod"]) - len(r["reac"])
        ch.exist_m[i] = 1 if r["exist_m"] else 0
        ch.numm[i] = len(r["indm"])
        for k, (ix, e) in enumerate(zip(r["indm"], r["men"])):
            ch.indm[i][k] = ix - 1
            ch.men[i][k] = e
        for k in range(3):
            ch.abe[i][k] = r["abe"][k]
            ch.cabe[i][k] = r["cabe"][k]
        for k in range(4):
            ch.troe[i][k] = r["troe"][k]
    for i, t in enumerate(m.trans):
        ch.tr2th[i] = t["tr2th"] - 1
        ch.num_sctn_trans[i] = t["nsec"]
        for l in range(t["nsec"]):
            ch.trange_trans[i][l][0], ch.trange_trans[i][l][1] = t["trange"][l]
            for j in range(4):
                ch.trans[i][l][j] = t["coef"][l][j]
    ch.rtol, ch.atol = m.rtol, m.atol
    return ch
