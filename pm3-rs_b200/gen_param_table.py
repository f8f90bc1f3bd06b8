"""Generate ``pm3-rs_b200/csrc/pm3_param_table.h`` from the PM3 parameter tables of pm3-rs.

Reads (in this build container only) the reference's data files
``src/data/pm3_parameters.csv``, ``src/data/element_data.csv`` and
``src/data/pm3_pair_parameters.csv`` (values extracted by pm3-rs from MOPAC v23.2.5,
``parameters_for_PM3_C.F90`` / ``parameters_C.F90`` / ``alpb_and_xfac_pm3.F90``) and writes the
raw, undervived numbers for the elements the s/p analytic path covers as a C header. Both the
GPU library and the CPU oracle include the header; each derives its own multipole terms from it.

Covered elements: the s/p elements with Z <= 17 except He and Ne, i.e. exactly the set for
which the reference takes its closed-form Slater overlap (``src/overlap.rs:269``, MOPAC
``diat2``) and its s/p multipole integrals (``src/integrals.rs``).

Usage: python pm3-rs_b200/gen_param_table.py <reference_root>

(<reference_root> is the root of a pm3-rs checkout; it is required.)
"""
import csv
import os
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python pm3-rs_b200/gen_param_table.py <pm3-rs checkout root>")
REF = sys.argv[1]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "pm3_param_table.h")
SUPPORTED = [1, 3, 4, 5, 6, 7, 8, 9, 11, 12, 13, 14, 15, 16, 17]


def rows(path):
    with open(path) as fh:
        lines = [l for l in fh if l.strip() and not l.lstrip().startswith("#")]
    return list(csv.DictReader(lines))


def num(v):
    return float(v) if v.strip() else 0.0


def main():
    par = {int(r["z"]): r for r in rows(os.path.join(REF, "src/data/pm3_parameters.csv"))}
    ele = {int(r["z"]): r for r in rows(os.path.join(REF, "src/data/element_data.csv"))}
    pairs = rows(os.path.join(REF, "src/data/pm3_pair_parameters.csv"))
    out = []
    out.append("// Generated by pm3-rs_b200/gen_param_table.py -- do not edit by hand.")
    out.append("// PM3 raw parameters (MOPAC v23.2.5 parameters_for_PM3_C.F90, parameters_C.F90,")
    out.append("// alpb_and_xfac_pm3.F90; Apache-2.0), as tabulated in pm3-rs src/data/*.csv.")
    out.append("// Published scientific constants; units: eV, Bohr^-1 (zeta), Angstrom^-1 (alpha).")
    out.append("#pragma once")
    out.append("")
    out.append("struct Pm3RawElement {")
    out.append("  int z; const char* sym;")
    out.append("  double uss, upp, zs, zp, betas, betap, gss, gsp, gpp, gp2, hsp, alp;")
    out.append("  double gauss[4][3];")
    out.append("  double ios, iop; int npq_s, npq_p; double eheat_kcal, mass, tore;")
    out.append("};")
    out.append("")
    out.append("struct Pm3RawPair { int zi, zj; double alpb, xfac; };")
    out.append("")
    out.append(f"static const int PM3_N_RAW_ELEMENTS = {len(SUPPORTED)};")
    out.append("static const Pm3RawElement PM3_RAW_ELEMENTS[] = {")
    for z in SUPPORTED:
        p, e = par[z], ele[z]
        g = []
        for i in range(1, 5):
            g.append("{%r, %r, %r}" % (num(p[f"g{i}_k"]), num(p[f"g{i}_l"]), num(p[f"g{i}_m"])))
        vals = [num(p[k]) for k in ("uss", "upp", "zs", "zp", "betas", "betap", "gss", "gsp",
                                      "gpp", "gp2", "hsp", "alp")]
        out.append(
            "  {%d, \"%s\", %s, {%s}, %r, %r, %d, %d, %r, %r, %r},"
            % (z, p["sym"], ", ".join(repr(v) for v in vals), ", ".join(g), num(e["ios"]),
               num(e["iop"]), int(num(e["npq_s"])), int(num(e["npq_p"])), num(e["eheat_kcal"]),
               num(e["mass"]), num(e["tore"])))
    out.append("};")
    out.append("")
    sel = []
    for r in pairs:
        zi, zj = int(num(r["zi"])), int(num(r["zj"]))
        if zi in SUPPORTED and zj in SUPPORTED:
            key = (max(zi, zj), min(zi, zj))
            if key not in [s[0] for s in sel]:
                sel.append((key, num(r["alpb"]), num(r["xfac"])))
    out.append(f"static const int PM3_N_RAW_PAIRS = {len(sel)};")
    out.append("static const Pm3RawPair PM3_RAW_PAIRS[] = {")
    for (zi, zj), a, x in sel:
        out.append("  {%d, %d, %r, %r}," % (zi, zj, a, x))
    out.append("};")
    with open(OUT, "w") as fh:
        fh.write("\n".join(out) + "\n")
    print("wrote", os.path.normpath(OUT))


if __name__ == "__main__":
    main()
