"""Generate ``mc_tri_table.inc``: the marching-cubes triangle table in a packed form.

The reconstructor's connectivity must be bit-identical to the reference crate's
``FEMTree::extract_surface`` (src/fem_tree.rs:576-636), which emits triangles from
``TRI_TABLE`` (src/tri_table.inl, the classic Lorensen-Cline / Bourke table, BSD-3 in
the crate) in row order.  The table's triangulation choices are arbitrary data, so
parity requires the same data.  This script reads the table from the reference source
tree (read-only) and writes it in this project's own encoding:

    PR_MC_NTRI[case]  : number of triangles of the case (0..5)
    PR_MC_TRIS[case]  : the case's edge indices, 4 bits each, first edge in the low nibble

The edge table is NOT copied: it is derived from corner signs (an edge is cut iff its
two corners classify differently), see ``mc_edge_mask`` in the CUDA and oracle sources.

Usage:  python gen_mc_table.py <path to src/tri_table.inl>  (writes mc_tri_table.inc
next to this script).  The generated file is committed; the GPU machine never runs this.
"""
import os
import re
import sys

# Corner / edge convention of src/fem_tree.rs:584-585 (corner k = (x,y,z) bits).
EDGES = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4),
         (0, 4), (1, 5), (2, 6), (3, 7)]


def edge_mask(case):
    m = 0
    for e, (a, b) in enumerate(EDGES):
        if ((case >> a) & 1) != ((case >> b) & 1):
            m |= 1 << e
    return m


def parse_table(text):
    rows = re.findall(r"\[([-0-9, ]+)\]", text)
    rows = [[int(v) for v in r.split(",")] for r in rows if len(r.split(",")) == 16]
    if len(rows) != 256:
        raise SystemExit("expected 256 rows of 16 entries, got %d" % len(rows))
    return rows


def pack(rows):
    ntri, packed = [], []
    for case, r in enumerate(rows):
        k = next((i for i, v in enumerate(r) if v < 0), 16)
        if k % 3 != 0 or any(v >= 0 for v in r[k:]):
            raise SystemExit("case %d: malformed row" % case)
        em = edge_mask(case)
        word = 0
        for i, e in enumerate(r[:k]):
            if not (0 <= e < 12) or not (em >> e) & 1:
                raise SystemExit("case %d uses edge %d outside its edge mask" % (case, e))
            word |= e << (4 * i)
        ntri.append(k // 3)
        packed.append(word)
    return ntri, packed


def main():
    src = sys.argv[1]
    rows = parse_table(open(src).read())
    ntri, packed = pack(rows)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mc_tri_table.inc")
    with open(out, "w") as f:
        f.write("/* Generated by gen_mc_table.py from the reference crate's src/tri_table.inl\n"
                " * (classic marching-cubes triangle table, Lorensen & Cline 1987 / Bourke 1994;\n"
                " * BSD-3-Clause in the crate).  Re-encoded: 4 bits per edge index, low nibble\n"
                " * first.  Identical data is required for bit-exact triangle connectivity. */\n")
        f.write("#define PR_MC_TABLE_CASES 256\n")
        f.write("PR_MC_TABLE_QUAL unsigned char PR_MC_NTRI[256] = {\n")
        for i in range(0, 256, 32):
            f.write("  " + ",".join(str(v) for v in ntri[i:i + 32]) + ",\n")
        f.write("};\n")
        f.write("PR_MC_TABLE_QUAL unsigned long long PR_MC_TRIS[256] = {\n")
        for i in range(0, 256, 4):
            f.write("  " + ", ".join("0x%015xULL" % v for v in packed[i:i + 4]) + ",\n")
        f.write("};\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
