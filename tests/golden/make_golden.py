"""Extract the golden fixtures the parity tests use from the pm3-rs reference tree.

Run where a pm3-rs checkout is available (its root is a required argument):

    python tests/golden/make_golden.py <reference_root>

Writes tests/golden/mopac_sp.json: the rows of pm3-rs ``tests/data/mopac_oracle.tsv`` (MOPAC
v23.2.5 PM3 PRECISE NOMM results, the acceptance set of ``tests/mopac_oracle.rs``) whose atoms
all belong to the s/p element set the analytic path covers, plus the molecule geometries and
known answers written into the reference's own unit/integration tests.
"""
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py <pm3-rs checkout root>")
REF = sys.argv[1]
HERE = os.path.dirname(os.path.abspath(__file__))
SYM = {"H": 1, "Li": 3, "Be": 4, "B": 5, "C": 6, "N": 7, "O": 8, "F": 9, "Na": 11, "Mg": 12, "Al": 13,
       "Si": 14, "P": 15, "S": 16, "Cl": 17}


def tsv_rows():
    rows = []
    with open(os.path.join(REF, "tests/data/mopac_oracle.tsv")) as fh:
        for line in fh:
            if line.startswith("#") or line.startswith("name\t") or not line.strip():
                continue
            f = line.rstrip("\n").split("\t")
            atoms = [a.split() for a in f[9].split(";")]
            if not all(a[0] in SYM for a in atoms):
                continue
            rows.append({
                "name": f[0], "formula": f[1], "charge": float(f[2]), "multiplicity": int(f[3]),
                "hof_kcal": float(f[4]),
                "dipole_debye": float(f[5]) if f[5] else None,
                "ip_ev": float(f[6]) if f[6] else None,
                "charges": [float(q) for q in f[7].split(";")] if f[7] else [],
                "z": [SYM[a[0]] for a in atoms],
                "xyz_angstrom": [[float(a[1]), float(a[2]), float(a[3])] for a in atoms],
            })
    return rows


def main():
    out = {
        "source": "pm3-rs tests/data/mopac_oracle.tsv (MOPAC v23.2.5 PM3 PRECISE NOMM), s/p subset",
        "tolerances": {"hof_kcal": 2.0e-3, "dipole_debye": 5.0e-3, "charge_e": 1.0e-3, "ip_ev": 1.0e-3},
        "rows": tsv_rows(),
    }
    with open(os.path.join(HERE, "mopac_sp.json"), "w") as fh:
        json.dump(out, fh, indent=0)
    print(len(out["rows"]), "rows")


if __name__ == "__main__":
    main()
