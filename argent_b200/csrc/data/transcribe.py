"""Transcribe argent's measured spectral tables into a C header.

The renderer needs the same measured numbers as argent: the CIE 1931 2-degree
colour matching functions and D65 (argent-spectra/src/data/cie.rs), the
pure-metal n,k grids (argent-spectra/src/data/metals.rs) and the alloy
auxiliary tables (argent-spectra/src/data/alloys.rs).  These are physical data
sets (CIE 015:2018, Johnson & Christy 1972/1974, Rakic 1998, Querry 1985/1987,
Rioux 2014), so they are carried over as numbers, not rewritten.

This script parses the numeric literals of those files and writes
``spectral_tables.h`` next to itself.  It runs once, in a checkout that has the
argent sources; the generated header is committed, so nothing at build or run
time needs the argent tree.

Usage:  python argent_b200/csrc/data/transcribe.py <argent checkout>
"""

import os
import re
import sys

NUM = r"[-+]?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?"


def parse_const(src: str, name: str):
    m = re.search(r"const\s+" + name + r"\s*:[^=]*=\s*\[(.*?)\n\];", src, re.S)
    if not m:
        raise SystemExit(f"table {name} not found")
    body = m.group(1)
    # drop trailing comments
    body = "\n".join(line.split("//")[0] for line in body.splitlines())
    # Keep the literal text: converting through a double and back could round
    # a long literal differently from a direct decimal -> f32 conversion.
    return re.findall(NUM, body.replace("_", ""))


def fmt(vals, per_line=6):
    out = []
    for i in range(0, len(vals), per_line):
        out.append("    " + ", ".join(repr_f(v) for v in vals[i:i + per_line]) + ",")
    return "\n".join(out)


def repr_f(s: str) -> str:
    if "e" not in s and "E" not in s and "." not in s:
        s += ".0"
    elif s.endswith("."):
        s += "0"
    return s + "f"


def main(ref_root: str):
    base = os.path.join(ref_root, "crates", "argent-spectra", "src", "data")
    cie = open(os.path.join(base, "cie.rs")).read()
    metals = open(os.path.join(base, "metals.rs")).read()
    alloys = open(os.path.join(base, "alloys.rs")).read()

    cmf = parse_const(cie, "CMF_1931_2DEG")
    assert len(cmf) == 471 * 3, len(cmf)
    d65 = parse_const(cie, "D65_300_830_5NM")
    assert len(d65) == 107, len(d65)

    metal_names = ["AG", "AU", "CU", "PT", "PD", "RH", "NI", "TI", "AL", "CR", "FE", "ZN", "SN"]
    metal_tabs = {}
    for n in metal_names:
        v = parse_const(metals, n)
        assert len(v) == 190, (n, len(v))
        metal_tabs[n] = v
    alloy_names = ["AU_AG_EXCESS_50", "CU_QUERRY", "CU85ZN15_QUERRY", "CU70ZN30_QUERRY"]
    alloy_tabs = {}
    for n in alloy_names:
        v = parse_const(alloys, n)
        assert len(v) == 190, (n, len(v))
        alloy_tabs[n] = v

    out = []
    out.append("// Generated by transcribe.py from argent-spectra/src/data/{cie,metals,alloys}.rs.")
    out.append("// Measured physical data (CIE 015:2018 tables; metal optical constants from")
    out.append("// Johnson & Christy, Rakic, Querry, Weaver; Au-Ag excess permittivity from Rioux 2014).")
    out.append("// Do not edit by hand.")
    out.append("#pragma once")
    out.append("")
    out.append("// CIE 1931 2-degree observer, xbar/ybar/zbar at 1 nm, 360..=830 nm (cie.rs:7).")
    out.append("static const float ARGENT_CMF_1931_2DEG[471 * 3] = {")
    out.append(fmt(cmf, 6))
    out.append("};")
    out.append("")
    out.append("// CIE D65 relative SPD at 5 nm, 300..=830 nm (cie.rs:486).")
    out.append("static const float ARGENT_D65_300_830_5NM[107] = {")
    out.append(fmt(d65, 8))
    out.append("};")
    out.append("")
    out.append("// Pure metals: (n, k) pairs on the 5 nm grid 360..=830 nm, 95 rows (metals.rs).")
    out.append("// Order: " + ", ".join(metal_names))
    out.append("#define ARGENT_NUM_METALS 13")
    out.append("static const float ARGENT_METAL_NK[13][190] = {")
    for n in metal_names:
        out.append("  { // " + n)
        out.append(fmt(metal_tabs[n], 10))
        out.append("  },")
    out.append("};")
    out.append("")
    out.append("// Alloy auxiliary tables, (a, b) pairs on the same grid (alloys.rs):")
    out.append("// AU_AG_EXCESS_50 is (Re, Im) of the 50/50 excess permittivity; the Querry tables are (n, k).")
    for n in alloy_names:
        out.append(f"static const float ARGENT_{n}[190] = {{")
        out.append(fmt(alloy_tabs[n], 10))
        out.append("};")
    out.append("")
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "spectral_tables.h")
    with open(dst, "w") as f:
        f.write("\n".join(out))
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: transcribe.py <argent checkout (the directory holding crates/)>")
    main(sys.argv[1])
