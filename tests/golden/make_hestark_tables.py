#!/usr/bin/env python3
"""Write fsg_hestark_tables.h: the tabulated Stark widths and shifts of 37 He I lines.

The data are published tables: Dimitrijevic & Sahal-Brechot (1990, A&AS 82,
519; 32 lines on six log T knots, electron, proton and He II perturbers) and Dimitrijevic &
Sahal-Brechot (1984, JQSRT 31, 301; 5 lines on four knots, electrons and protons).  Identical
results need identical numbers, so this script reads them from the reference's hestark.f90 (its
PARAMETER arrays WlcHe, EloHe, Tt90/Tt84, We90 ... Sp84) and writes them in this library's own
layout: one record per tabulated line holding its centre, lower level energy, knot count and, per
perturber, the width and shift at every knot.

    python tests/golden/make_hestark_tables.py [path/to/hestark.f90]
(default: src/hestark.f90 of the reference tree named by $FASTSPEC_REFERENCE).  The header is
committed beside the library's sources; the library and the oracle include it.
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
SRC = os.path.join(os.environ.get("FASTSPEC_REFERENCE", ""), "src", "hestark.f90")
OUT = os.path.join(REPO, "fastspec_b200", "csrc", "fsg_hestark_tables.h")


def parameter_array(text, name):
    """Numbers of the Fortran array constructor `name(...) = [ ... ]` (with or without RESHAPE)."""
    m = re.search(r"::\s*%s\s*(\([^)]*\))?\s*=\s*(RESHAPE\()?\s*\[(.*?)\]" % name, text, re.S)
    if not m:
        raise SystemExit("no PARAMETER array %s" % name)
    body = m.group(3).replace("&", " ")
    return [float(x.replace("D", "e").replace("d", "e")) for x in re.findall(r"[-+0-9.]+[DdEe][-+]?[0-9]+|[-+]?[0-9]+\.[0-9]*", body)]


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else SRC
    text = open(src).read()
    text = "\n".join(line.split("!")[0] for line in text.splitlines())
    wlc, elo = parameter_array(text, "WlcHe"), parameter_array(text, "EloHe")
    t90, t84 = parameter_array(text, "Tt90"), parameter_array(text, "Tt84")
    n90, n84 = len(wlc) - 5, 5
    assert len(wlc) == len(elo) == 37 and len(t90) == 6 and len(t84) == 4
    tab = {}
    for nm in ("We90", "Wp90", "Wh90", "Se90", "Sp90", "Sh90"):
        v = parameter_array(text, nm)
        assert len(v) == 6 * n90, nm
        tab[nm] = [v[6 * k:6 * k + 6] for k in range(n90)]       # Fortran (knot, line), knot fastest
    for nm in ("We84", "Wp84", "Se84", "Sp84"):
        v = parameter_array(text, nm)
        assert len(v) == 4 * n84, nm
        tab[nm] = [v[4 * k:4 * k + 4] + [0.0, 0.0] for k in range(n84)]
    zero = [[0.0] * 6 for _ in range(n84)]
    tab["Wh84"], tab["Sh84"] = zero, zero

    f = lambda x: repr(float(x))
    row = lambda v: "{" + ", ".join(f(x) for x in v) + "}"
    out = []
    out.append("/* Tabulated Stark widths and shifts of 37 He I lines: Dimitrijevic & Sahal-Brechot (1990,")
    out.append(" * A&AS 82, 519) entries 1-32 on six log T knots with electron, proton and He II perturbers;")
    out.append(" * Dimitrijevic & Sahal-Brechot (1984, JQSRT 31, 301) entries 33-37 on four knots, electrons and")
    out.append(" * protons (their He II rows are zero).  Units: width and shift in Angstrom per 1e16 perturbers")
    out.append(" * per cm^3; centres in air Angstrom; lower level energies in eV.  The numbers are those of the")
    out.append(" * reference's hestark.f90 (WlcHe, EloHe, Tt90/Tt84, We90..Sp84), written by")
    out.append(" * make_hestark_tables.py; data only, shared by the library and the CPU oracle. */")
    out.append("#ifndef FSG_HESTARK_TABLES_H")
    out.append("#define FSG_HESTARK_TABLES_H")
    out.append("")
    out.append("#ifndef FSG_HE_NTAB")
    out.append("#define FSG_HE_NTAB 37")
    out.append("#endif")
    out.append("#define FSG_HE_NDS90 32")
    out.append("")
    out.append("/* air centre [A], lower level energy [eV], number of log T knots (6 or 4), and per perturber")
    out.append("   (0 electrons, 1 protons, 2 He II) the width w and shift s at each knot */")
    out.append("typedef struct { double wlc, elo; int nknot; double w[3][6], s[3][6]; } fsg_he_line;")
    out.append("")
    out.append("static const double FSG_HE_LOGT90[6] = %s;" % row(t90))
    out.append("static const double FSG_HE_LOGT84[4] = %s;" % row(t84))
    out.append("")
    out.append("static const fsg_he_line FSG_HE_TAB[FSG_HE_NTAB] = {")
    for k in range(37):
        ds90 = k < n90
        j = k if ds90 else k - n90
        sfx = "90" if ds90 else "84"
        w = [tab["W" + p + sfx][j] for p in "eph"]
        s = [tab["S" + p + sfx][j] for p in "eph"]
        out.append("    {%s, %s, %d," % (f(wlc[k]), f(elo[k]), 6 if ds90 else 4))
        out.append("     {%s}," % ", ".join(row(v) for v in w))
        out.append("     {%s}}," % ", ".join(row(v) for v in s))
    out.append("};")
    out.append("")
    out.append("#endif")
    open(OUT, "w").write("\n".join(out) + "\n")
    print(OUT)


if __name__ == "__main__":
    main()
