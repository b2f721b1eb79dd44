"""The lane-exact restatement of the reference's 8/16-bit striped kernels
(parasail_b200/csrc/pb_lane.cuh), built for the host with the lane-loop
policy of tests/lane_host.cpp, against the reference's own AVX2 kernels
compiled from source (oracle/_ref): score, ends, statistics and the
saturation flag, on random pairs chosen so that many runs saturate.

The SW statistics case follows the FASTSTATS wrapper
(util/templates/sw_stats_striped_bias.c:644-730): the score pass is exact
when it does not saturate, and the emulated kernel runs on the prefix."""
import ctypes
import json
import os
import random
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import AA, DNA, rand_seq, mutate

HERE = os.path.dirname(__file__)
CSRC = os.path.join(HERE, "..", "parasail_b200", "csrc")
ALGS = ["nw", "sg", "sg_qb", "sg_qe", "sg_qx", "sg_db", "sg_de", "sg_dx", "sg_qb_de", "sg_qe_db", "sg_qb_db",
        "sg_qe_de"]


@pytest.fixture(scope="module")
def lanelib(tmp_path_factory):
    if O.ref() is None:
        pytest.skip("reference library not built")
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    out = str(tmp_path_factory.mktemp("lane") / "liblanehost.so")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", CSRC, "-o", out,
                           os.path.join(HERE, "lane_host.cpp")])
    lib = ctypes.CDLL(out)
    lib.lane_host_run.argtypes = [ctypes.c_int] * 2 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                       ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                       ctypes.c_int] + [ctypes.c_int] * 4 + [ctypes.c_void_p] * 2
    return lib


def _matrix(key):
    if isinstance(key, str):
        g = json.load(open(os.path.join(HERE, "golden", "matrices.json")))[key]
        return O.Matrix(g["values"], g["mapper"], g["alphabet"], g["max"], g["min"], key)
    return O.Matrix.simple(*key)


def _emulate(lib, kind, bits, m, q, t, op, gp, sg, qlen=None, tlen=None):
    qc = m.codes(q).astype(np.uint8)
    tc = m.codes(t).astype(np.uint8)
    lp = len(qc) + 64
    prof = np.zeros((m.size, lp), np.int32)
    prof[:, :len(qc)] = m.values[:, qc]
    qpad = np.zeros(lp, np.uint8)
    qpad[:len(qc)] = qc
    out = np.zeros(7, np.int32)
    sga = np.array(sg, np.int32)
    assert lib.lane_host_run(kind, bits, prof.ctypes.data, m.size, lp, qpad.ctypes.data, qlen or len(qc),
                             tc.ctypes.data, tlen or len(tc), op, gp, m.max, m.min, sga.ctypes.data,
                             out.ctypes.data) == 0
    return out


@pytest.mark.parametrize("seed", [1, 2])
def test_lane_emulation_vs_reference_kernels(lanelib, seed):
    rng = random.Random(seed)
    bad, total, nsat = [], 0, 0
    for it in range(8):
        for bits in (8, 16):
            for stats in (0, 1):
                for name in ALGS + ["sw"]:
                    if name == "sw" and not stats:
                        continue
                    if it % 2:
                        key, a = "blosum62", AA
                        op, gp = rng.choice([(11, 1), (10, 2), (3, 1), (40, 2), (127, 5), (200, 1)])
                    else:
                        key, a = ("ACGT", 2, -3), DNA
                        op, gp = rng.choice([(5, 2), (4, 1), (2, 1), (60, 3), (130, 0)])
                    hi = rng.randint(300, 1500) if (bits == 16 and rng.random() < 0.6) else rng.randint(1, 300)
                    q = rand_seq(rng, rng.randint(1, hi), a)
                    t = mutate(rng, q, a, 0.2, 0.04) if it % 3 == 0 else rand_seq(rng, rng.randint(1, hi), a)
                    m = _matrix(key)
                    sg = [0, 0, 0, 0]
                    if name.startswith("sg"):
                        f = O.SG_CASES[name]
                        sg = [int(bool(f & O.S1_BEG)), int(bool(f & O.S1_END)), int(bool(f & O.S2_BEG)),
                              int(bool(f & O.S2_END))]
                    exp = O.ref_vector(name, stats, "striped", str(bits), q, t, op, gp, key)
                    if name == "sw":
                        if op <= gp or op >= (128 if bits == 8 else 32768):
                            continue   # the score pass itself departs from the exact DP there
                        ex = O.align(O.SW, 0, 0, q, t, op, gp, m)
                        maxp = (127 if bits == 8 else 32767) - (m.max + 1) - (-128 if bits == 8 else -32768)
                        if ex["score"] > maxp:
                            continue   # score pass saturated: no statistics kernel runs
                        o = _emulate(lanelib, 2, bits, m, q, t, op, gp, sg, ex["end_query"] + 1, ex["end_ref"] + 1)
                        got = {"score": int(o[0]), "end_query": ex["end_query"], "end_ref": ex["end_ref"],
                               "matches": int(o[3]), "similar": int(o[4]), "length": int(o[5])}
                    else:
                        o = _emulate(lanelib, 1 if stats else 0, bits, m, q, t, op, gp, sg)
                        got = {"score": int(o[0]), "end_query": int(o[1]), "end_ref": int(o[2])}
                        if stats:
                            got.update(matches=int(o[3]), similar=int(o[4]), length=int(o[5]))
                    total += 1
                    nsat += int(o[6])
                    e = dict(exp)
                    esat = int(bool(e.pop("flag") & 64))
                    if esat != int(o[6]) or any(got.get(k) != v for k, v in e.items()):
                        bad.append((name, bits, stats, key, op, gp, q, t, exp, got))
    assert total > 300 and nsat > 50
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:2])


@pytest.mark.parametrize("seed", [3, 4])
def test_lane_emulation_linear_and_wrapped_penalties(lanelib, seed):
    """open <= gap (the score-only kernels' lazy-F loop stops on ties there)
    and penalties that wrap in the lane width, at 8, 16 and 32 bits, for the
    score-only nw/sg kernels (src/nw_striped_avx2_256_16.c), the statistics
    nw/sg kernels and the score-only SW kernels (util/templates/
    sw_striped_bias.c, util/templates/sw_striped.c)."""
    rng = random.Random(seed)
    bad, total = [], 0
    cases = (("sw", 3), ("nw", 0), ("sg", 0), ("sg_qx", 0), ("sg_de", 0), ("sg_qb_db", 0), ("nw", 1),
             ("sg_qe_db", 1))
    for it in range(6):
        for bits in (8, 16, 32):
            for name, kind in cases:
                stats = kind == 1
                if it % 2:
                    key, a = "blosum62", AA
                    op, gp = rng.choice([(1, 1), (3, 3), (0, 1), (1, 2), (2, 2), (200, 1), (5, 5)])
                else:
                    key, a = ("ACGT", 2, -3), DNA
                    op, gp = rng.choice([(1, 1), (2, 2), (0, 1), (1, 3), (130, 2), (3, 3)])
                hi = rng.randint(1, 250)
                q = rand_seq(rng, rng.randint(1, hi), a)
                t = mutate(rng, q, a, 0.2, 0.04) if it % 3 == 0 else rand_seq(rng, rng.randint(1, hi), a)
                m = _matrix(key)
                sg = [0, 0, 0, 0]
                if name.startswith("sg"):
                    f = O.SG_CASES[name]
                    sg = [int(bool(f & O.S1_BEG)), int(bool(f & O.S1_END)), int(bool(f & O.S2_BEG)),
                          int(bool(f & O.S2_END))]
                exp = O.ref_vector(name, stats, "striped", str(bits), q, t, op, gp, key)
                o = _emulate(lanelib, kind, bits, m, q, t, op, gp, sg)
                got = {"score": int(o[0]), "end_query": int(o[1]), "end_ref": int(o[2])}
                if stats:
                    got.update(matches=int(o[3]), similar=int(o[4]), length=int(o[5]))
                total += 1
                e = dict(exp)
                esat = int(bool(e.pop("flag") & 64))
                if esat != int(o[6]) or any(got.get(k) != v for k, v in e.items()):
                    bad.append((name, kind, bits, key, op, gp, q, t, exp, got))
    assert total == 6 * 3 * len(cases)
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:2])


def _ref_trace_flag(name, scheme, bits, q, t, op, gp, key):
    """Saturation flag and score of the reference's AVX2 trace kernel
    parasail_{name}_trace_{scheme}_avx2_256_{bits}."""
    import ctypes
    r = O.ref()
    fn = getattr(r, "parasail_%s_trace_%s_avx2_256_%d" % (name, scheme, bits))
    fn.restype = ctypes.POINTER(O.PResult)
    fn.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.POINTER(O.PMatrix)]
    rp = fn(q.encode(), len(q), t.encode(), len(t), op, gp, O.ref_matrix_ptr(key))
    out = (int(bool(rp.contents.flag & 64)), rp.contents.score)
    r.parasail_result_free(rp)
    return out


@pytest.mark.parametrize("seed", [5, 6])
def test_trace_kernel_saturation_emulation(lanelib, seed):
    """The 8/16-bit nw/sg trace kernels (util/templates/{nw,sg}_trace_striped.c:
    the score-only passes with the lazy-F loop continuing on ties;
    {nw,sg}_trace_scan.c: E, H, F and the SG gap ramp checked): the
    emulation's saturation flag equals the reference kernel's, and the
    striped emulation's score equals the reference's when not saturated,
    over penalties with open > gap, open == gap, open < gap and wrapped
    values, and lengths around the 8- and 16-bit limits."""
    rng = random.Random(seed)
    bad, total, nsat = [], 0, 0
    for it in range(6):
        for bits in (8, 16):
            for scheme, kind in (("striped", 4), ("scan", 5)):
                for name in ALGS:
                    if it % 2:
                        key, a = "blosum62", AA
                        op, gp = rng.choice([(11, 1), (10, 2), (3, 1), (40, 2), (127, 5), (200, 1), (1, 1), (0, 1),
                                             (1, 3), (5, 5)])
                    else:
                        key, a = ("ACGT", 2, -3), DNA
                        op, gp = rng.choice([(5, 2), (4, 1), (2, 1), (60, 3), (130, 0), (1, 1), (0, 2), (3, 3)])
                    hi = rng.randint(300, 1500) if (bits == 16 and rng.random() < 0.6) else rng.randint(1, 300)
                    q = rand_seq(rng, rng.randint(1, hi), a)
                    t = mutate(rng, q, a, 0.2, 0.04) if it % 3 == 0 else rand_seq(rng, rng.randint(1, hi), a)
                    m = _matrix(key)
                    sg = [0, 0, 0, 0]
                    if name.startswith("sg"):
                        f = O.SG_CASES[name]
                        sg = [int(bool(f & O.S1_BEG)), int(bool(f & O.S1_END)), int(bool(f & O.S2_BEG)),
                              int(bool(f & O.S2_END))]
                    esat, escore = _ref_trace_flag(name, scheme, bits, q, t, op, gp, key)
                    o = _emulate(lanelib, kind, bits, m, q, t, op, gp, sg)
                    total += 1
                    nsat += esat
                    if int(o[6]) != esat or (kind == 4 and not esat and int(o[0]) != escore):
                        bad.append((name, scheme, bits, key, op, gp, q, t, esat, escore, list(o)))
    assert total == 6 * 2 * 2 * len(ALGS) and 60 < nsat < total - 60
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:2])


@pytest.mark.parametrize("seed", [7, 8])
def test_scan_kernel_emulation(lanelib, seed):
    """The score-only scan kernels (util/templates/nw_scan.c, sg_scan.c,
    sw_scan.c) restated lane by lane: score, ends and the saturation flag
    equal the reference's AVX2 kernels at 8, 16 and 32 bits, including open
    < gap (where their prefix scan of F departs from the exact DP) and
    penalties that wrap in the lane."""
    rng = random.Random(seed)
    bad, total, differs = [], 0, 0
    for it in range(5):
        for bits in (8, 16, 32):
            for name in ALGS + ["sw"]:
                if it % 2:
                    key, a = "blosum62", AA
                    op, gp = rng.choice([(11, 1), (10, 2), (1, 3), (0, 2), (2, 5), (200, 1), (1, 1), (3, 4)])
                else:
                    key, a = ("ACGT", 2, -3), DNA
                    op, gp = rng.choice([(5, 2), (0, 1), (1, 3), (2, 4), (130, 2), (1, 1)])
                hi = rng.randint(1, 260)
                q = rand_seq(rng, rng.randint(1, hi), a)
                t = mutate(rng, q, a, 0.2, 0.04) if it % 3 == 0 else rand_seq(rng, rng.randint(1, hi), a)
                m = _matrix(key)
                sg = [0, 0, 0, 0]
                if name.startswith("sg"):
                    f = O.SG_CASES[name]
                    sg = [int(bool(f & O.S1_BEG)), int(bool(f & O.S1_END)), int(bool(f & O.S2_BEG)),
                          int(bool(f & O.S2_END))]
                exp = O.ref_vector(name, 0, "scan", str(bits), q, t, op, gp, key)
                o = _emulate(lanelib, 7 if name == "sw" else 6, bits, m, q, t, op, gp, sg)
                got = {"score": int(o[0]), "end_query": int(o[1]), "end_ref": int(o[2])}
                total += 1
                e = dict(exp)
                esat = int(bool(e.pop("flag") & 64))
                if not esat and op < gp:
                    ex = O.align(O.alg_of(name)[0], O.alg_of(name)[1], 0, q, t, op, gp, m)
                    differs += (ex["score"], ex["end_query"], ex["end_ref"]) != (e["score"], e["end_query"],
                                                                             e["end_ref"])
                if esat != int(o[6]) or any(got.get(k) != v for k, v in e.items()):
                    bad.append((name, bits, key, op, gp, q, t, exp, got))
    assert total == 5 * 3 * (len(ALGS) + 1) and differs > 5
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:2])


@pytest.mark.parametrize("seed", [9, 10])
def test_stats_scan_kernel_emulation(lanelib, seed):
    """The statistics scan kernels (util/templates/nw_stats_scan.c,
    sg_stats_scan.c, sw_stats_scan.c) restated lane by lane: score, ends,
    matches, similar, length and the saturation flag equal the reference's
    AVX2 kernels at 8, 16 and 32 bits, including open < gap (where their
    prefix scan of F departs from the exact DP) and penalties that wrap in
    the lane."""
    rng = random.Random(seed)
    bad, total, differs, nsat = [], 0, 0, 0
    for it in range(4):
        for bits in (8, 16, 32):
            for name in ALGS + ["sw"]:
                if it % 2:
                    key, a = "blosum62", AA
                    op, gp = rng.choice([(11, 1), (10, 2), (1, 3), (0, 2), (2, 5), (200, 1), (1, 1), (3, 4)])
                else:
                    key, a = ("ACGT", 2, -3), DNA
                    op, gp = rng.choice([(5, 2), (0, 1), (1, 3), (2, 4), (130, 2), (1, 1)])
                hi = rng.randint(1, 220)
                q = rand_seq(rng, rng.randint(1, hi), a)
                t = mutate(rng, q, a, 0.2, 0.04) if it % 3 == 0 else rand_seq(rng, rng.randint(1, hi), a)
                m = _matrix(key)
                sg = [0, 0, 0, 0]
                if name.startswith("sg"):
                    f = O.SG_CASES[name]
                    sg = [int(bool(f & O.S1_BEG)), int(bool(f & O.S1_END)), int(bool(f & O.S2_BEG)),
                          int(bool(f & O.S2_END))]
                exp = O.ref_vector(name, 1, "scan", str(bits), q, t, op, gp, key)
                o = _emulate(lanelib, 9 if name == "sw" else 8, bits, m, q, t, op, gp, sg)
                got = {"score": int(o[0]), "end_query": int(o[1]), "end_ref": int(o[2]),
                       "matches": int(o[3]), "similar": int(o[4]), "length": int(o[5])}
                total += 1
                e = dict(exp)
                esat = int(bool(e.pop("flag") & 64))
                nsat += esat
                if not esat and op < gp:
                    ex = O.align(O.alg_of(name)[0], O.alg_of(name)[1], 1, q, t, op, gp, m)
                    differs += any(ex[k] != e[k] for k in got)
                if esat != int(o[6]) or any(got.get(k) != v for k, v in e.items() if k in got):
                    bad.append((name, bits, key, op, gp, q, t, exp, got))
    assert total == 4 * 3 * (len(ALGS) + 1) and differs > 3 and nsat > 3
    assert not bad, "%d mismatches, first: %r" % (len(bad), bad[:2])
