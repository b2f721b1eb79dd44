#!/usr/bin/env python3
"""Writes parasail_b200/csrc/matrices_data.inc: the built-in substitution
matrices (BLOSUM30-100, BLOSUMN, PAM10-500, DNAfull, NUC.4.4) as one text
record per matrix: "name alphabet max min v00 v01 ...". The values are the
published NCBI/EMBOSS tables; they must be identical to the reference's
(parasail/matrices/*.h) for drop-in parity, so this one-off generator reads
them from a checkout of the reference given on the command line.

    python parasail_b200/csrc/gen_matrices.py /path/to/parasail > parasail_b200/csrc/matrices_data.inc
"""
import os
import re
import sys


def main(ref):
    mdir = os.path.join(ref, "parasail", "matrices")
    names = sorted(f[:-2] for f in os.listdir(mdir)
                   if f.endswith(".h") and not f.endswith("_map.h"))
    print("/* generated by gen_matrices.py: name alphabet max min values(row-major) */")
    for n in names:
        txt = open(os.path.join(mdir, n + ".h")).read()
        body = re.search(r"static const int parasail_%s_\[\] = \{(.*?)\};" % n, txt, re.S).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        vals = [int(v) for v in re.findall(r"-?\d+", body)]
        tail = re.search(r"parasail_matrix_t parasail_%s = \{(.*?)\};" % n, txt, re.S).group(1)
        tail = re.sub(r"/\*.*?\*/", "", tail, flags=re.S)
        parts = [p.strip() for p in tail.split(",")]
        # name, matrix, mapper, size, max, min, user_matrix, type, length, alphabet, query
        size, mx, mn = int(parts[3]), int(parts[4]), int(parts[5])
        alpha = parts[9].strip('"')
        assert len(vals) == size * size, (n, len(vals), size)
        assert len(alpha) == size, (n, alpha)
        print('"%s %s %d %d %s\\n"' % (n, alpha, mx, mn, " ".join(map(str, vals))))


if __name__ == "__main__":
    main(sys.argv[1])
