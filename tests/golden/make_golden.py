"""Writes the known-answer fixtures under tests/golden/.

single_triangle.dat / .bin: the 7-column boundary matrix of a filled triangle
(three vertices, three edges, one triangle) in PHAT ascii form with comments
and blank lines, and in PHAT binary form.  Its persistence pairs are the
reference's known answer, phat-highclear/examples/single_triangle_persistence_pairs.dat
("3 / 1 3 / 2 4 / 5 6"); when the reference tree is present the script checks
the expected file against it.
"""
import os
import struct

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference tree's root comes from SSPP_REFERENCE (checked only when set)
REF_PAIRS = os.path.join(os.environ.get("SSPP_REFERENCE", ""),
                         "phat-highclear/examples/single_triangle_persistence_pairs.dat")

COLUMNS = [(0, []), (0, []), (0, []), (1, [0, 1]), (1, [0, 2]), (1, [1, 2]), (2, [3, 4, 5])]
PAIRS = [(1, 3), (2, 4), (5, 6)]


def main():
    with open(os.path.join(HERE, "single_triangle.dat"), "w") as f:
        f.write("# three vertices\n0\n0\n0\n\n# three edges\n1 0 1\n1 0 2\n1 1 2\n# the triangle\n2 3 4 5\n\n\n")
    with open(os.path.join(HERE, "single_triangle.bin"), "wb") as f:
        f.write(struct.pack("<q", len(COLUMNS)))
        for d, c in COLUMNS:
            f.write(struct.pack("<qq", d, len(c)))
            for x in c:
                f.write(struct.pack("<q", x))
    with open(os.path.join(HERE, "single_triangle_pairs.dat"), "w") as f:
        f.write(f"{len(PAIRS)}\n")
        for b, d in PAIRS:
            f.write(f"{b} {d}\n")
    if os.environ.get("SSPP_REFERENCE") and os.path.exists(REF_PAIRS):
        ref = [ln.split() for ln in open(REF_PAIRS).read().split("\n") if ln.strip()]
        assert int(ref[0][0]) == len(PAIRS)
        assert [(int(a), int(b)) for a, b in ref[1:]] == PAIRS, "fixture disagrees with the reference's answer"


if __name__ == "__main__":
    main()
