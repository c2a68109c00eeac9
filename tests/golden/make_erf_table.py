"""Generate tests/golden/erf_table.csv from the reference's ERF table text files.

The reference ships its RBL Coulomb table twice: as C++ arrays (rbmd/framework/model/ERFTable.h)
and as text (rbmd/res/json_files/Gnear_table_leq2_2.txt for 0.1 <= d < 2,
Gnear_table_geq2_2.txt for 2 <= d < 12; columns: entry index, distance, spacing, G, dG).  This
script keeps every second row (and the last) of each text file as (index, distance, G) so that
the oracle's reconstruction of the table is pinned against the reference's own numbers.
Run it in a checkout that has the reference at REF (first argument, else $RBMD_REFERENCE,
default /root/reference).
"""
import os
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RBMD_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    out = ["index,distance,g"]
    for name in ("Gnear_table_leq2_2.txt", "Gnear_table_geq2_2.txt"):
        rows = [ln.split() for ln in open(os.path.join(REF, "rbmd/res/json_files", name)) if ln.strip()]
        keep = rows[::2] + ([rows[-1]] if (len(rows) - 1) % 2 else [])
        out += [f"{r[0]},{r[1]},{r[3]}" for r in keep]
    with open(os.path.join(HERE, "erf_table.csv"), "w") as f:
        f.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
