"""Generate ``pm3-rs_b200/csrc/pm3_d3_table.h``: the Grimme D3 reference data of pm3-rs for the
elements the s/p path covers.

Reads (in this build container only) the reference's data files ``src/data/d3_c6_reference.csv``
(C6 reference tuples iat, jat, c6, cn_a, cn_b), ``src/data/d3_r0ab.csv`` (packed lower triangle of
the 94 x 94 cutoff radii, Angstrom) and ``src/data/d3_radii.csv`` (z, r2r4, rcov), which pm3-rs took
from MOPAC v23.2.5 (``copyc6.F90``, ``dftd3_bits.F90``), and writes the raw numbers as a C header
that both the GPU library and the CPU oracle include. The load-time transforms of the reference
(src/corrections/d3.rs:84-158) are left to the code that reads the header:

* C6 tuples are grouped under the key (max Z, min Z) in file order, a tuple whose row has
  iat < jat getting its two reference coordination numbers swapped (d3.rs:96-108);
* r0ab stays in Angstrom (divided by the Bohr radius at use, d3.rs:114-121);
* r2r4 and rcov stay raw (sqrt(0.5 r2r4 sqrt(Z)) and 4/3 rcov / a0 at use, d3.rs:135-143).

Usage: python pm3-rs_b200/gen_d3_table.py <pm3-rs checkout root>
"""
import csv
import os
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python pm3-rs_b200/gen_d3_table.py <pm3-rs checkout root>")
REF = sys.argv[1]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "pm3_d3_table.h")
SUPPORTED = [1, 3, 4, 5, 6, 7, 8, 9, 11, 12, 13, 14, 15, 16, 17]
MAX = 94


def rows(path):
    with open(path) as fh:
        lines = [l for l in fh if l.strip() and not l.lstrip().startswith("#")]
    return list(csv.DictReader(lines))


def main():
    idx = {z: k for k, z in enumerate(SUPPORTED)}
    ne = len(SUPPORTED)
    npair = ne * (ne + 1) // 2
    tuples = [[] for _ in range(npair)]
    for r in rows(os.path.join(REF, "src/data/d3_c6_reference.csv")):
        i, j = int(float(r["iat"])), int(float(r["jat"]))
        if i not in idx or j not in idx:
            continue
        a, b = max(idx[i], idx[j]), min(idx[i], idx[j])
        c6, cna, cnb = r["c6"].strip(), r["cn_a"].strip(), r["cn_b"].strip()
        tuples[a * (a + 1) // 2 + b].append((c6, cna, cnb) if i >= j else (c6, cnb, cna))

    packed = [r["value"].strip() for r in rows(os.path.join(REF, "src/data/d3_r0ab.csv"))]
    assert len(packed) == MAX * (MAX + 1) // 2
    r0 = {}
    k = 0
    for i in range(MAX):
        for j in range(i + 1):
            r0[(i + 1, j + 1)] = r0[(j + 1, i + 1)] = packed[k]
            k += 1

    radii = {int(float(r["z"])): (r["r2r4"].strip(), r["rcov"].strip())
             for r in rows(os.path.join(REF, "src/data/d3_radii.csv"))}

    out = ["// Generated by pm3-rs_b200/gen_d3_table.py from pm3-rs src/data/d3_c6_reference.csv,",
           "// d3_r0ab.csv and d3_radii.csv (Grimme D3 reference data via MOPAC v23.2.5). Do not edit.",
           "#pragma once", "",
           f"#define PM3_D3_NELEM {ne}",
           f"#define PM3_D3_NPAIR {npair}",
           f"#define PM3_D3_NREF {sum(len(t) for t in tuples)}", "",
           "// element index -> Z (ascending Z)",
           "static const int pm3_d3_z[PM3_D3_NELEM] = {" + ", ".join(str(z) for z in SUPPORTED) + "};",
           "// raw r2r4 and rcov (Angstrom) per element index",
           "static const double pm3_d3_r2r4_raw[PM3_D3_NELEM] = {" +
           ", ".join(radii[z][0] for z in SUPPORTED) + "};",
           "static const double pm3_d3_rcov_raw[PM3_D3_NELEM] = {" +
           ", ".join(radii[z][1] for z in SUPPORTED) + "};",
           "// r0ab (Angstrom) by element indices",
           "static const double pm3_d3_r0ab_ang[PM3_D3_NELEM][PM3_D3_NELEM] = {"]
    for zi in SUPPORTED:
        out.append("  {" + ", ".join(r0[(zi, zj)] for zj in SUPPORTED) + "},")
    out.append("};")
    out.append("// tuples of the element pair (a >= b) at a * (a + 1) / 2 + b: [off[p], off[p + 1])")
    offs = [0]
    for t in tuples:
        offs.append(offs[-1] + len(t))
    out.append("static const int pm3_d3_pair_off[PM3_D3_NPAIR + 1] = {" + ", ".join(map(str, offs)) + "};")
    out.append("// (c6, cn of the higher-Z atom, cn of the lower-Z atom) in file order")
    out.append("static const double pm3_d3_ref[PM3_D3_NREF][3] = {")
    for t in tuples:
        for c6, cna, cnb in t:
            out.append(f"  {{{c6}, {cna}, {cnb}}},")
    out.append("};")
    with open(OUT, "w") as fh:
        fh.write("\n".join(out) + "\n")
    print(f"wrote {OUT}: {ne} elements, {npair} pairs, {offs[-1]} C6 tuples")


if __name__ == "__main__":
    main()
