#!/usr/bin/env python3
"""Generates include/parasail/matrices/*.h, the public matrix headers of the
drop-in API.

Programs written against the reference include e.g.
<parasail/matrices/blosum62.h> and pass &parasail_blosum62 (a static const
parasail_matrix_t defined in that header; reference
parasail/matrices/blosum62.h:29-69, used by tests/test_basic.c:4-6,22). Each
generated header defines, for one built-in matrix, the same two objects: the
row-major value table `parasail_<name>_` and the matrix object
`parasail_<name>`, with the reference's field values (name, size, max, min,
PARASAIL_MATRIX_TYPE_SQUARE, length, alphabet). The BLOSUM and PAM headers
share a mapper array from blosum_map.h / pam_map.h, as the reference's do;
DNAfull and NUC.4.4 carry their own. Every mapper maps each alphabet letter
(either case) to its index and every other byte to the last index, the rule
of parasail_matrix_create (src/memory.c:376-386).

The values are the published NCBI/EMBOSS tables held in
parasail_b200/csrc/matrices_data.inc (the library's own built-in set), so
&parasail_blosum62 and parasail_matrix_lookup("blosum62") hold equal tables.

Run:  python include/gen_matrix_headers.py
"""
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "..", "parasail_b200", "csrc", "matrices_data.inc")
OUT = os.path.join(HERE, "parasail", "matrices")


def read_data():
    out = []
    for line in open(DATA):
        m = re.match(r'^"(\S+) (\S+) (-?\d+) (-?\d+) (.*)\\n"$', line.strip())
        if m:
            vals = [int(v) for v in m.group(5).split()]
            out.append((m.group(1), m.group(2), int(m.group(3)), int(m.group(4)), vals))
    return out


def mapper(alpha):
    m = [len(alpha) - 1] * 256
    for i, c in enumerate(alpha):
        m[ord(c.upper())] = i
        m[ord(c.lower())] = i
    return m


def c_array(name, vals, per_line):
    rows = [", ".join("%3d" % v for v in vals[k:k + per_line]) for k in range(0, len(vals), per_line)]
    return "static const int %s[%s] = {\n    %s\n};\n" % (name, "" if name.endswith("_") else "256",
                                                         ",\n    ".join(rows))


def guard(name):
    return "PARASAIL_B200_MATRIX_%s_H" % re.sub(r"\W", "_", name).upper()


def header(body_name, includes, body):
    g = guard(body_name)
    return ("/* Generated by include/gen_matrix_headers.py: built-in matrix %s of the\n"
            " * parasail-b200 drop-in API (published NCBI/EMBOSS values). */\n"
            "#ifndef %s\n#define %s\n\n%s\n#ifdef __cplusplus\nextern \"C\" {\n#endif\n\n%s\n"
            "#ifdef __cplusplus\n}\n#endif\n\n#endif\n") % (body_name, g, g, includes, body)


def main():
    os.makedirs(OUT, exist_ok=True)
    mats = read_data()
    protein = "ARNDCQEGHILKMFPSTWYVBZX*"
    for fam in ("blosum", "pam"):
        open(os.path.join(OUT, fam + "_map.h"), "w").write(
            header(fam + "_map", "", c_array("parasail_%s_map" % fam, mapper(protein), 16)))
    for name, alpha, mx, mn, vals in mats:
        size = len(alpha)
        assert len(vals) == size * size, name
        if name.startswith("blosum") or name.startswith("pam"):
            fam = "blosum" if name.startswith("blosum") else "pam"
            assert alpha == protein, name
            inc = '#include "parasail.h"\n#include "%s_map.h"\n' % fam
            map_name = "parasail_%s_map" % fam
            body = ""
        else:
            inc = '#include "parasail.h"\n'
            map_name = "parasail_%s_map_" % name
            body = c_array(map_name, mapper(alpha), 16).replace("%s[]" % map_name, "%s[256]" % map_name) + "\n"
        body += c_array("parasail_%s_" % name, vals, size)
        body += ("\nstatic const parasail_matrix_t parasail_%s = {\n    \"%s\",\n    parasail_%s_,\n    %s,\n"
                 "    %d,\n    %d,\n    %d,\n    NULL,\n    PARASAIL_MATRIX_TYPE_SQUARE,\n    %d,\n    \"%s\",\n"
                 "    NULL\n};\n") % (name, name, name, map_name, size, mx, mn, size, alpha)
        open(os.path.join(OUT, name + ".h"), "w").write(header(name, inc, body))


if __name__ == "__main__":
    main()
