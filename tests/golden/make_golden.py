#!/usr/bin/env python3
"""Generates the golden fixtures in tests/golden/ from the reference itself.

Needs oracle/_ref/libparasail_ref.so, the reference (jeffdaily/parasail
v2.6.2) compiled from its sources by oracle/Makefile. Writes:

  matrices.json        BLOSUM62 / BLOSUM50 / PAM50 / NUC.4.4 as the reference
                       library reports them (values, mapper, alphabet, max, min)
  serial_golden.json   outputs of the reference's serial functions
                       (parasail_{alg}[_stats]) and parasail_nw_banded
  vector_golden.json   outputs of the reference's AVX2 striped/scan profile
                       kernels at 8/16/32 bits and of the 8->16->32 chains,
                       flags included, on short pairs chosen to straddle the
                       narrow widths' saturation limits

    python tests/golden/make_golden.py
"""
import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402

AA = "ARNDCQEGHILKMFPSTWYV"
DNA = "ACGT"
ALGS = ["sw", "nw", "sg", "sg_qb", "sg_qe", "sg_qx", "sg_db", "sg_de", "sg_dx",
        "sg_qb_de", "sg_qe_db", "sg_qb_db", "sg_qe_de"]


def rs(rng, n, a):
    return "".join(rng.choice(a) for _ in range(n))


def mut(rng, s, a, sub, indel):
    out = []
    for c in s:
        r = rng.random()
        if r < indel / 2:
            continue
        if r < indel:
            out.append(rng.choice(a))
        out.append(rng.choice(a) if rng.random() < sub else c)
    return "".join(out) or a[0]


def pair(rng, kind, lo, hi):
    a = AA if kind == "aa" else DNA
    q = rs(rng, rng.randint(lo, hi), a)
    r = rng.random()
    if r < 0.4:
        t = mut(rng, q, a, rng.uniform(0.0, 0.4), rng.uniform(0.0, 0.08))
    elif r < 0.5:
        t = q
    else:
        t = rs(rng, rng.randint(lo, hi), a)
    return q, t


def main():
    if O.ref() is None:
        sys.exit("reference library not built: make -C oracle")
    mats = {}
    for name in ("blosum62", "blosum50", "pam50", "nuc44"):
        m = O.ref_matrix(name)
        mats[name] = {"values": m.values.tolist(), "mapper": m.mapper.tolist(),
                      "alphabet": m.alphabet, "max": m.max, "min": m.min}
    json.dump(mats, open(os.path.join(HERE, "matrices.json"), "w"))

    rng = random.Random(20261203)
    settings = [("aa", "blosum62", 10, 1), ("aa", "blosum62", 11, 1), ("aa", "blosum62", 3, 1),
                ("dna", ["ACGT", 2, -3], 5, 2), ("dna", ["ACGT", 1, -2], 4, 1)]
    serial = []
    for alg in ALGS:
        for stats in (0, 1):
            for k in range(8):
                kind, mk, op, gp = settings[k % len(settings)]
                q, t = pair(rng, kind, 1, 80)
                exp = O.ref_serial(alg, stats, q, t, op, gp, mk if isinstance(mk, str) else tuple(mk))
                serial.append({"alg": alg, "stats": stats, "q": q, "t": t, "open": op, "gap": gp,
                               "matrix": mk, "expect": exp})
    for k in range(40):
        q, t = pair(rng, "dna", 1, 90)
        band = rng.randint(1, 30)
        exp = O.ref_nw_banded(q, t, 5, 2, band, ("ACGT", 2, -3))
        serial.append({"alg": "nw_banded", "stats": 0, "q": q, "t": t, "open": 5, "gap": 2,
                       "k": band, "matrix": ["ACGT", 2, -3], "expect": exp})
    json.dump({"cases": serial}, open(os.path.join(HERE, "serial_golden.json"), "w"))

    vector = []
    for alg in ALGS:
        for stats in (0, 1):
            for scheme in ("striped", "scan"):
                for width in ("8", "16", "32", "sat"):
                    for k in range(5):
                        kind, mk, op, gp = settings[(k + len(alg)) % len(settings)]
                        q, t = pair(rng, kind, 2, 140)
                        exp = O.ref_vector(alg, stats, scheme, width, q, t, op, gp,
                                           mk if isinstance(mk, str) else tuple(mk))
                        vector.append({"alg": alg, "stats": stats, "scheme": scheme, "width": width,
                                       "q": q, "t": t, "open": op, "gap": gp, "matrix": mk,
                                       "expect": exp})
    json.dump({"cases": vector}, open(os.path.join(HERE, "vector_golden.json"), "w"))
    print("serial", len(serial), "vector", len(vector))


if __name__ == "__main__":
    main()
