"""Extract the data tables the synthetic H2/air cases need from a checkout of
the reference (read-only) into this folder.

    python shared_cfd_b200/data/make_data.py /path/to/shared_cfd

Writes
  h2air9_thermo.dat  NASA-7 'thermo all' blocks of H2 O2 H2O H O OH HO2 H2O2 N2
                     (from sample/no23.chemkin_mono_uv/chem.inp),
  h2air9_trans.dat   their single-species viscosity fits
                     (store/therm_lib/chemkin/core/trans.inp, same format),
  elements_mw.dat    element weights of H, O, N
                     (store/therm_lib/chemkin/core/MW.inp, same format),
  h2air9_nasa9.dat   NASA-9 blocks of the same species
                     (store/therm_lib/NASA/core/thermo.inp, first occurrence),
  h2air9_nasa_trans.dat  their single-species viscosity fits
                     (store/therm_lib/NASA/core/trans.inp, same format),
  hon17_nasa9.dat, hon17_nasa_trans.dat  the same for those species and
                     N NO NO2 N2O NH NH2 NH3 HNO,
  elements_mw_nasa.dat   element weights of H, O, N (store/therm_lib/NASA/core/MW.inp).
"""
import os
import sys

SPECIES = ["H2", "O2", "H2O", "H", "O", "OH", "HO2", "H2O2", "N2"]
ELEMENTS = ["H", "O", "N"]
# a larger H/O/N set for the generic (more than 12 species) CEA kernel
SPECIES_HON = SPECIES + ["N", "NO", "NO2", "N2O", "NH", "NH2", "NH3", "HNO"]


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(ref, "sample/no23.chemkin_mono_uv/chem.inp")) as f:
        lines = f.read().splitlines()
    k = lines.index("thermo all")
    blocks = {}
    i = k + 2
    while not lines[i].strip().lower().startswith("end"):
        name = lines[i][:24].split(" ")[0]
        blocks[name] = lines[i:i + 4]
        i += 4
    with open(os.path.join(here, "h2air9_thermo.dat"), "w") as f:
        f.write(lines[k + 1] + "\n")
        for s in SPECIES:
            f.write("\n".join(blocks[s]) + "\n")
    with open(os.path.join(ref, "store/therm_lib/chemkin/core/trans.inp")) as f:
        tl = f.read().splitlines()
    out = [tl[0]]
    i = 1
    while i < len(tl):
        ln = tl[i]
        if ln[:3] in ("END", "end"):
            break
        if ln[:1] == "!":
            i += 1
            continue
        iv, ic = int(ln[35:36]), int(ln[37:38])
        name, comment = ln[0:15].strip(), ln[16:31].strip()
        if name in SPECIES and not comment:
            out.extend(tl[i:i + 1 + iv + ic])
        i += 1 + iv + ic
    out.append("END")
    with open(os.path.join(here, "h2air9_trans.dat"), "w") as f:
        f.write("\n".join(out) + "\n")
    with open(os.path.join(ref, "store/therm_lib/chemkin/core/MW.inp")) as f:
        mw = [ln for ln in f.read().splitlines() if ln.split() and ln.split()[0] in ELEMENTS]
    with open(os.path.join(here, "elements_mw.dat"), "w") as f:
        f.write("\n".join(mw) + "\n")
    nasa_tables(ref, SPECIES, "h2air9")
    nasa_tables(ref, SPECIES_HON, "hon17")
    with open(os.path.join(os.path.join(ref, "store/therm_lib/NASA/core"), "MW.inp")) as f:
        mw = [ln for ln in f.read().splitlines() if ln.split() and ln.split()[0] in ELEMENTS]
    with open(os.path.join(here, "elements_mw_nasa.dat"), "w") as f:
        f.write("\n".join(mw) + "\n")


def nasa_tables(ref, species, prefix):
    """<prefix>_nasa9.dat and <prefix>_nasa_trans.dat of one species list."""
    here = os.path.dirname(os.path.abspath(__file__))
    nasa = os.path.join(ref, "store/therm_lib/NASA/core")
    with open(os.path.join(nasa, "thermo.inp")) as f:
        tl = f.read().splitlines()
    i = 0
    while tl[i][:1] == "!":
        i += 1
    out = [tl[i], tl[i + 1]]  # 'thermo' and the default ranges line
    i += 2
    found = {}
    while i < len(tl) and not tl[i].startswith("END"):
        name = tl[i][:18].strip()
        nsec = int(tl[i + 1][:2])
        if name in species and name not in found:
            found[name] = tl[i:i + 2 + 3 * nsec]
        i += 2 + 3 * nsec
    for s in species:
        out.extend(found[s])
    out.append("END PRODUCTS")
    with open(os.path.join(here, prefix + "_nasa9.dat"), "w") as f:
        f.write("\n".join(out) + "\n")
    with open(os.path.join(nasa, "trans.inp")) as f:
        tl = f.read().splitlines()
    out = [tl[0]]
    i = 1
    while i < len(tl):
        ln = tl[i]
        if ln[:3] in ("END", "end"):
            break
        if ln[:1] == "!":
            i += 1
            continue
        iv, ic = int(ln[35:36]), int(ln[37:38])
        name, comment = ln[0:15].strip(), ln[16:31].strip()
        if name in species and not comment:
            out.extend(tl[i:i + 1 + iv + ic])
        i += 1 + iv + ic
    out.append("END")
    with open(os.path.join(here, prefix + "_nasa_trans.dat"), "w") as f:
        f.write("\n".join(out) + "\n")

if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: %s" % "python shared_cfd_b200/data/make_data.py /path/to/shared_cfd")
    main(sys.argv[1])
