"""Long global alignments, the banded DP, the exactness certificate and the
learned band (MLP on k-mer diagonal histograms), through the C ABI.

* the one-warp-per-pair global kernel against the oracle's serial NW;
* the banded kernel against the oracle's banded DP, and the certificate's
  soundness: every certified banded score equals the full-DP score;
* the MLP's GPU gradients against a NumPy float64 restatement of the same
  network (same BF16-rounded weights), and its input features against a
  NumPy restatement of the histogram;
* training on GPU, the learned band's scores equal full DP on every pair,
  and the gain over the method without the network (a fixed band).
"""
import random

import numpy as np
import pytest

import oracle as O
from conftest import AA, DNA, rand_seq, mutate

pb = pytest.importorskip("parasail_b200")
from parasail_b200 import synth  # noqa: E402

pytestmark = pytest.mark.gpu

OPEN, GAP = 4, 1


def _pack(seqs):
    return pb.pack(seqs)


def _dna_pairs(rng, n, lo, hi, div=0.1):
    qs, ts = [], []
    for _ in range(n):
        q = rand_seq(rng, rng.randint(lo, hi), DNA)
        t = mutate(rng, q, DNA, div, div / 3) if rng.random() < 0.8 else rand_seq(rng, rng.randint(lo, hi), DNA)
        qs.append(q)
        ts.append(t)
    return qs, ts


def test_nw_long_vs_oracle_dna_and_protein():
    rng = random.Random(1)
    dna = pb.matrix_create("ACGT", 1, -2)
    om = O.Matrix.simple("ACGT", 1, -2)
    qs, ts = _dna_pairs(rng, 120, 1, 700)
    qs += [rand_seq(rng, 3000, DNA)]
    ts += [mutate(rng, qs[-1], DNA, 0.1, 0.03)]
    got = pb.nw_long(dna, *_pack(qs), *_pack(ts), OPEN, GAP)
    exp = [O.align(O.NW, 0, 0, q, t, OPEN, GAP, om)["score"] for q, t in zip(qs, ts)]
    assert got.tolist() == exp
    b62 = pb.matrix_lookup("blosum62")
    ob = O.Matrix.from_struct(b62)
    ps = [rand_seq(rng, rng.randint(1, 400), AA) for _ in range(40)]
    pt = [mutate(rng, p, AA, 0.3, 0.05) for p in ps]
    got = pb.nw_long(b62, *_pack(ps), *_pack(pt), 11, 1)
    assert got.tolist() == [O.align(O.NW, 0, 0, q, t, 11, 1, ob)["score"] for q, t in zip(ps, pt)]
    # open < gap takes the kernel's general F recurrence
    got = pb.nw_long(dna, *_pack(qs[:40]), *_pack(ts[:40]), 1, 3)
    assert got.tolist() == [O.align(O.NW, 0, 0, q, t, 1, 3, om)["score"] for q, t in zip(qs[:40], ts[:40])]
    # open >= gap with scores + open past int8: the unbiased one-operation chain
    got = pb.nw_long(b62, *_pack(ps), *_pack(pt), 120, 2)
    assert got.tolist() == [O.align(O.NW, 0, 0, q, t, 120, 2, ob)["score"] for q, t in zip(ps, pt)]


def test_banded_vs_oracle_and_certificate_soundness():
    rng = random.Random(2)
    dna = pb.matrix_create("ACGT", 1, -2)
    om = O.Matrix.simple("ACGT", 1, -2)
    qs, ts = _dna_pairs(rng, 150, 50, 900, div=0.08)
    lo, hi = [], []
    for q, t in zip(qs, ts):
        d_end = len(q) - len(t)
        w = rng.choice([0, 3, 20, 80, 300, 2000])
        c = d_end // 2 + rng.randint(-10, 10)
        lo.append(min(c - w, min(0, d_end)))
        hi.append(max(c + w, max(0, d_end)))
    sc, cert = pb.nw_banded_certified(dna, *_pack(qs), *_pack(ts), OPEN, GAP, lo, hi)
    full = pb.nw_long(dna, *_pack(qs), *_pack(ts), OPEN, GAP)
    ncert = 0
    for k, (q, t) in enumerate(zip(qs, ts)):
        assert sc[k] == O.nw_band(q, t, OPEN, GAP, lo[k], hi[k], om), k
        assert sc[k] <= full[k]
        if cert[k]:
            ncert += 1
            assert sc[k] == full[k], k
    assert 0 < ncert < len(qs)


def test_banded_pass_edges_vs_oracle():
    """Banded pairs whose lengths sit at the 256-row pass and 8-row lane
    boundaries, with narrow and wide bands, for open > gap, open < gap (the
    kernel's general F recurrence) and a protein matrix (scores from the
    shared-memory table rather than the byte permute)."""
    rng = random.Random(5)
    dna = pb.matrix_create("ACGT", 1, -2)
    om = O.Matrix.simple("ACGT", 1, -2)
    b62 = pb.matrix_lookup("blosum62")
    ob = O.Matrix.from_struct(b62)
    lens = [255, 256, 257, 263, 264, 511, 512, 513, 520, 767, 768, 769]
    for mat, omat, alpha, op, gp in ((dna, om, DNA, OPEN, GAP), (dna, om, DNA, 1, 3), (b62, ob, AA, 11, 1)):
        qs, ts, lo, hi = [], [], [], []
        for L in lens:
            for w in (0, 5, 40, 400):
                q = rand_seq(rng, L, alpha)
                t = mutate(rng, q, alpha, 0.06, 0.02) if rng.random() < 0.7 else \
                    rand_seq(rng, L + rng.randint(-30, 30), alpha)
                d_end = len(q) - len(t)
                c = d_end // 2 + rng.randint(-5, 5)
                qs.append(q)
                ts.append(t)
                lo.append(min(c - w, min(0, d_end)))
                hi.append(max(c + w, max(0, d_end)))
        sc, _ = pb.nw_banded_certified(mat, *_pack(qs), *_pack(ts), op, gp, lo, hi)
        for k, (q, t) in enumerate(zip(qs, ts)):
            assert sc[k] == O.nw_band(q, t, op, gp, lo[k], hi[k], omat), (k, len(q), len(t), lo[k], hi[k], op, gp)


def _bf16(x):
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def _numpy_grads(w, b, x, t, tau, nin=258, nh=128, no=2):
    """float64 forward/backward of the band MLP (the CPU oracle of the GPU
    kernels): squared error on output 0, pinball loss on output 1."""
    w = _bf16(w).astype(np.float64)
    b = b.astype(np.float64)
    n1, n2 = nh * nin, nh * nh
    W1 = w[:n1].reshape(nh, nin)
    W2 = w[n1:n1 + n2].reshape(nh, nh)
    W3 = w[n1 + n2:].reshape(no, nh)
    b1, b2, b3 = b[:nh], b[nh:2 * nh], b[2 * nh:]
    x = x.astype(np.float64)
    B = len(x)
    h1 = np.maximum(x @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    y = h2 @ W3.T + b3
    ec = y[:, 0] - t[:, 0]
    ew = t[:, 1] - y[:, 1]
    dy = np.stack([2 * ec / B, np.where(ew > 0, -tau, 1 - tau) / B], axis=1)
    d2 = (dy @ W3) * (h2 > 0)
    d1 = (d2 @ W2) * (h1 > 0)
    gw = np.concatenate([(d1.T @ x).ravel(), (d2.T @ h1).ravel(), (dy.T @ h2).ravel()])
    gb = np.concatenate([d1.sum(0), d2.sum(0), dy.sum(0)])
    loss = np.mean(ec ** 2 + np.where(ew > 0, tau * ew, (tau - 1) * ew))
    return gw, gb, loss


def test_mlp_gradients_vs_cpu_oracle():
    m = pb.BandModel(seed=3)
    rng = np.random.default_rng(0)
    x = rng.random((64, m.n_in)).astype(np.float32)
    t = np.stack([rng.normal(0, 0.05, 64), rng.uniform(0.01, 0.3, 64)], axis=1).astype(np.float32)
    w, b = m.get()
    gw, gb, loss = m.gradients(x, t, 0.9)
    ew, eb, eloss = _numpy_grads(w, b, x, t, 0.9)
    assert np.allclose(gw, ew, rtol=2e-3, atol=1e-6)
    assert np.allclose(gb, eb, rtol=2e-3, atol=1e-6)
    assert abs(loss - eloss) < 1e-4 * max(1.0, abs(eloss))
    m.close()


def _numpy_features(a, b):
    """Restatement of the k = 8 diagonal-offset histogram feature."""
    n, m = len(a), len(b)
    first = {}
    for i in range(n - 7):
        k = a[i:i + 8]
        if all(c < 4 for c in k):
            first.setdefault(bytes(k), i)
    hist = np.zeros(256, np.float64)
    nk = 0
    L = np.float32(max(n, m))
    mid = np.float32(0.5) * np.float32(n - m)
    scale = np.float32(256) / (np.float32(0.5) * L)
    for j in range(m - 7):
        k = b[j:j + 8]
        if not all(c < 4 for c in k):
            continue
        nk += 1
        i = first.get(bytes(k))
        if i is None:
            continue
        d = np.float32(i - j) - mid
        bn = int(np.floor(np.float32(d * scale))) + 128
        hist[min(max(bn, 0), 255)] += 1
    f = np.zeros(258, np.float32)
    f[:256] = (hist * np.float32(1.0 / max(1, nk)) * 16).astype(np.float32)
    f[256] = np.float32(np.log(np.float32(n)) / 11)
    f[257] = np.float32(np.log(np.float32(m)) / 11)
    return f


def test_features_vs_numpy():
    a, ao, al, b, bo, bl, _ = synth.dna_long_pairs(seed=9, n_pairs=6, lo=500, hi=3000)
    dna = pb.matrix_create("ACGT", 1, -2)
    # the API takes characters; the generator gives ACGT bytes
    f = pb.band_features(dna, a, ao, al, b, bo, bl)
    amap = {ord(c): i for i, c in enumerate("ACGT")}
    for k in range(6):
        A = [amap[c] for c in a[ao[k]:ao[k] + al[k]].tolist()]
        B = [amap[c] for c in b[bo[k]:bo[k] + bl[k]].tolist()]
        e = _numpy_features(A, B)
        assert np.allclose(f[k], e, rtol=1e-5, atol=1e-6), k


def test_learned_band_trains_certifies_and_beats_fixed_band():
    dna = pb.matrix_create("ACGT", 1, -2)
    tr = synth.dna_long_pairs(seed=11, n_pairs=600, lo=1000, hi=4000)
    te = synth.dna_long_pairs(seed=12, n_pairs=120, lo=1000, hi=4000)
    m = pb.BandModel(seed=1)
    l0 = m.train(dna, *tr[:6], OPEN, GAP, epochs=1, batch=128, lr=2e-3)
    l1 = m.train(dna, *tr[:6], OPEN, GAP, epochs=60, batch=128, lr=2e-3)
    assert l1 < l0
    widen, slack = m.scaling()                     # tuned on the held-out tenth
    assert 1.0 <= widen <= 3.0 and slack == 32
    full = pb.nw_long(dna, *te[:6], OPEN, GAP)
    sc, lo, hi, st = m.align(dna, *te[:6], OPEN, GAP, widen=0.0, slack=-1)
    assert (sc == full).all()                      # every reported score equals full DP
    assert st.pairs == 120 and st.certified + st.fallback == 120
    assert st.certified >= 0.8 * 120
    # the method without the network: one fixed band for all pairs, wide
    # enough for the largest divergence of the distribution
    qlen, tlen = te[2], te[5]
    L = np.maximum(qlen, tlen)
    half = (0.25 * L).astype(np.int64)
    d_end = qlen.astype(np.int64) - tlen
    flo = np.minimum(d_end // 2 - half, np.minimum(0, d_end))
    fhi = np.maximum(d_end // 2 + half, np.maximum(0, d_end))
    fsc, fcert = pb.nw_banded_certified(dna, *te[:6], OPEN, GAP, flo, fhi)

    def cells(lo_, hi_):
        tot = 0
        for n, mm, l_, h_ in zip(qlen.tolist(), tlen.tolist(), lo_.tolist(), hi_.tolist()):
            for d in range(max(l_, -(mm - 1)), min(h_, n - 1) + 1):
                tot += min(n - 1 - d, mm - 1) - max(0, -d) + 1
        return tot

    full_cells = qlen.astype(np.int64) * tlen
    learned_cells = st.band_cells                 # every DP cell the learned path ran, reruns included
    # the fixed band, too, must fall back to full DP where it does not certify
    assert (fsc[fcert == 1] == full[fcert == 1]).all()
    fixed_cells = cells(flo, fhi) + float(full_cells[fcert == 0].sum())
    assert learned_cells < fixed_cells
    m.close()


def test_doubling_band_equals_full_dp():
    """The model-free certified band (doubling on certificate failure)
    returns the full-DP score of every pair, including pairs whose first
    band is far too narrow and short pairs whose band covers the matrix."""
    a, ao, al, b, bo, bl, _ = synth.dna_long_pairs(seed=31, n_pairs=40, lo=200, hi=4000)
    dna = pb.matrix_create("ACGT", 1, -2)
    full = pb.nw_long(dna, a, ao, al, b, bo, bl, 4, 1)
    for w0 in (1, 16, 5000):
        sc, st = pb.nw_doubling_band(dna, a, ao, al, b, bo, bl, 4, 1, w0)
        assert (sc == full).all(), w0
        assert st.pairs == 40
    _, st1 = pb.nw_doubling_band(dna, a, ao, al, b, bo, bl, 4, 1, 1)
    assert st1.fallback > 0        # a one-diagonal start fails the certificate somewhere
