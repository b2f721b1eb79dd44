"""Seeded synthetic workloads shaped like the reference's benchmark configs.

No public dataset is available offline, so each generator draws i.i.d.
residues at published background frequencies and plants homologs with a
stated identity and indel rate. All generators are vectorised numpy and
deterministic for a given seed.
"""
import numpy as np

AA = "ARNDCQEGHILKMFPSTWYV"
# Amino-acid background frequencies of Robinson & Robinson (1991), the
# composition NCBI BLAST uses for protein statistics.
AA_FREQ = np.array([0.07805, 0.05129, 0.04487, 0.05364, 0.01925, 0.04264, 0.06295, 0.07377,
                    0.02199, 0.05142, 0.09019, 0.05744, 0.02243, 0.03856, 0.05203, 0.07120,
                    0.05841, 0.01330, 0.03216, 0.06441])
AA_FREQ = AA_FREQ / AA_FREQ.sum()
AA_BYTES = np.frombuffer(AA.encode(), dtype=np.uint8)
DNA_BYTES = np.frombuffer(b"ACGT", dtype=np.uint8)


def _residues(rng, n, protein=True):
    if protein:
        return AA_BYTES[rng.choice(20, size=n, p=AA_FREQ)]
    return DNA_BYTES[rng.integers(0, 4, size=n)]


def mutate(rng, seq, identity, indel, protein=True, geom_p=None):
    """seq: uint8 array. Keeps each residue with probability `identity`
    (else a background draw), inserts/deletes at total rate `indel` (half
    each); indel lengths geometric(geom_p) when given, else 1."""
    n = len(seq)
    keep = rng.random(n) < identity
    out = np.where(keep, seq, _residues(rng, n, protein))
    ev = rng.random(n)
    pieces = []
    i = 0
    ins_pos = np.nonzero(ev < indel / 2)[0]
    del_pos = np.nonzero((ev >= indel / 2) & (ev < indel))[0]
    events = sorted([(p, 0) for p in ins_pos] + [(p, 1) for p in del_pos])
    for p, kind in events:
        if p < i:
            continue
        pieces.append(out[i:p])
        ln = 1 if geom_p is None else int(rng.geometric(geom_p))
        if kind == 0:
            pieces.append(_residues(rng, ln, protein))
            i = p
        else:
            i = min(n, p + ln)
    pieces.append(out[i:])
    res = np.concatenate(pieces) if pieces else out
    return res if len(res) else seq[:1].copy()


def protein_db_search(seed=2, n_targets=200_000, query_lengths=(100, 250, 500, 1000, 2000),
                      median=270.0, sigma=0.72, lo=20, hi=5000, homolog_frac=0.01,
                      homolog_identity=0.30, homolog_indel=0.02):
    """Protein database search: queries of the given lengths against
    log-normal-length targets (median 270, sigma 0.72 -> mean about 350,
    clipped to [20, 5000]); homolog_frac of the targets are homologs of a
    random query. Returns (queries: list[bytes], targets buffer, offsets, lengths)."""
    rng = np.random.default_rng(seed)
    queries = [_residues(rng, L).tobytes() for L in query_lengths]
    lens = np.clip(np.rint(rng.lognormal(np.log(median), sigma, n_targets)), lo, hi).astype(np.int64)
    homolog = rng.random(n_targets) < homolog_frac
    which = rng.integers(0, len(queries), n_targets)
    seqs = []
    pool = _residues(rng, int(lens.sum()))
    off = 0
    for k in range(n_targets):
        L = int(lens[k])
        if homolog[k]:
            q = np.frombuffer(queries[which[k]], dtype=np.uint8)
            seqs.append(mutate(rng, q, homolog_identity, homolog_indel))
        else:
            seqs.append(pool[off:off + L])
        off += L
    lengths = np.array([len(s) for s in seqs], dtype=np.int32)
    offsets = np.zeros(n_targets, dtype=np.int64)
    offsets[1:] = np.cumsum(lengths, dtype=np.int64)[:-1]
    buf = np.concatenate(seqs).astype(np.uint8)
    return queries, buf, offsets, lengths


def protein_query_vs_targets(seed=1, qlen=300, n_targets=1000, lo=100, hi=500):
    """One query of length qlen vs n_targets with lengths uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    q = _residues(rng, qlen).tobytes()
    lens = rng.integers(lo, hi + 1, n_targets).astype(np.int32)
    buf = _residues(rng, int(lens.sum()))
    offsets = np.zeros(n_targets, dtype=np.int64)
    offsets[1:] = np.cumsum(lens, dtype=np.int64)[:-1]
    return q, buf, offsets, lens


def dna_read_windows(seed=3, n_pairs=1_000_000, lo=100, hi=300, flank=32, sub=0.05, ins=0.005, dele=0.005):
    """DNA reads vs their reference windows: window = uniform ACGT of length
    read+flank; read = the window's first read-length bases mutated with
    5% substitutions and 0.5% insertions / 0.5% deletions (lengths geometric
    p=0.5). Returns (reads buf, offs, lens, windows buf, offs, lens)."""
    rng = np.random.default_rng(seed)
    rl = rng.integers(lo, hi + 1, n_pairs).astype(np.int64)
    wl = rl + flank
    wbuf = DNA_BYTES[rng.integers(0, 4, int(wl.sum()))]
    woff = np.zeros(n_pairs, dtype=np.int64)
    woff[1:] = np.cumsum(wl)[:-1]
    reads = []
    for k in range(n_pairs):
        base = wbuf[woff[k]:woff[k] + rl[k]]
        reads.append(mutate(rng, base, 1.0 - sub * 4 / 3, ins + dele, protein=False, geom_p=0.5))
    rlen = np.array([len(r) for r in reads], dtype=np.int32)
    roff = np.zeros(n_pairs, dtype=np.int64)
    roff[1:] = np.cumsum(rlen, dtype=np.int64)[:-1]
    return np.concatenate(reads), roff, rlen, wbuf, woff, wl.astype(np.int32)


def dna_long_pairs(seed=5, n_pairs=20_000, lo=5_000, hi=50_000, div_lo=0.01, div_hi=0.15,
                   indel_share=0.30, indel_mean=3.0, big_frac=0.30, big_lo=50, big_hi=500):
    """Long DNA pairs: A uniform ACGT of length U[lo, hi]; B = A with a
    per-pair divergence d ~ U[div_lo, div_hi] split 70/30 between
    substitutions and indels (indel lengths geometric with the given mean),
    plus one large insertion or deletion of U[big_lo, big_hi] bp in big_frac
    of the pairs. Returns (A buf, offs, lens, B buf, offs, lens, divergences)."""
    rng = np.random.default_rng(seed)
    la = rng.integers(lo, hi + 1, n_pairs)
    div = rng.uniform(div_lo, div_hi, n_pairs)
    a_all = DNA_BYTES[rng.integers(0, 4, int(la.sum()))]
    aoff = np.zeros(n_pairs, dtype=np.int64)
    aoff[1:] = np.cumsum(la)[:-1]
    bs = []
    gp = 1.0 / indel_mean
    for k in range(n_pairs):
        a = a_all[aoff[k]:aoff[k] + la[k]]
        sub = div[k] * (1.0 - indel_share)
        # indel events: each costs on average indel_mean bases of divergence
        ind = div[k] * indel_share / indel_mean
        b = mutate(rng, a, 1.0 - sub * 4.0 / 3.0, 2.0 * ind, protein=False, geom_p=gp)
        if rng.random() < big_frac:
            L = int(rng.integers(big_lo, big_hi + 1))
            p = int(rng.integers(0, max(1, len(b) - L)))
            if rng.random() < 0.5:
                b = np.concatenate([b[:p], DNA_BYTES[rng.integers(0, 4, L)], b[p:]])
            else:
                b = np.concatenate([b[:p], b[p + L:]]) if len(b) > L + 1 else b
        bs.append(b)
    lb = np.array([len(b) for b in bs], dtype=np.int32)
    boff = np.zeros(n_pairs, dtype=np.int64)
    boff[1:] = np.cumsum(lb, dtype=np.int64)[:-1]
    return a_all, aoff, la.astype(np.int32), np.concatenate(bs), boff, lb, div
