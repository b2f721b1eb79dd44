"""Seeded synthetic workloads shaped like the reference's benchmark configs.

No public dataset is available offline, so each generator draws i.i.d.
residues at published background frequencies and plants homologs with a
stated identity and indel rate. All generators are vectorised numpy
(mutations of many sequences at once, no per-sequence Python loop) and
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
_AA_CDF = np.cumsum(AA_FREQ)


def _residues(rng, n, protein=True):
    if protein:
        idx = np.searchsorted(_AA_CDF, rng.random(n), side="right")
        return AA_BYTES[np.minimum(idx, 19)]
    return DNA_BYTES[rng.integers(0, 4, size=n, dtype=np.uint8)]


def offsets_of(lens):
    offs = np.zeros(len(lens), dtype=np.int64)
    if len(lens):
        offs[1:] = np.cumsum(np.asarray(lens, dtype=np.int64))[:-1]
    return offs


def mutate_many(rng, buf, offs, lens, identity, indel, protein=True, geom_p=None,
                extra_pos=None, extra_len=None, extra_ins=None):
    """Mutates many sequences at once. Sequence k (buf[offs[k]:offs[k]+lens[k]])
    keeps each residue with probability identity[k] (else a background draw);
    at rate indel[k] per residue an insertion (half) or deletion (half)
    event starts, of length geometric(geom_p) (1 when geom_p is None);
    insertions put random residues before the residue, deletions remove
    it and the following ones (within the sequence). identity and indel
    are scalars or per-sequence arrays. Optionally one extra event per
    sequence: extra_pos[k] >= 0 is its position (relative to the sequence),
    extra_len[k] its length and extra_ins[k] whether it inserts. A sequence
    that would become empty keeps its first residue. Returns (buf, offs,
    lens) of the mutated sequences."""
    lens = np.asarray(lens, dtype=np.int64)
    offs = np.asarray(offs, dtype=np.int64)
    n_seq = len(lens)
    total = int(lens.sum())
    src = np.concatenate([buf[o:o + l] for o, l in zip(offs, lens)]) if n_seq and \
        not (len(buf) == total and (offs == offsets_of(lens)).all()) else np.asarray(buf[:total])
    ident = np.broadcast_to(np.asarray(identity, dtype=np.float32), (n_seq,))
    ind = np.broadcast_to(np.asarray(indel, dtype=np.float32), (n_seq,))
    res = np.array(src, dtype=np.uint8, copy=True)
    change = rng.random(total, dtype=np.float32) >= np.repeat(ident, lens)
    res[change] = _residues(rng, int(change.sum()), protein)
    ev = rng.random(total, dtype=np.float32)
    ind_r = np.repeat(ind, lens)
    is_ins = ev < ind_r * 0.5
    is_del = (ev >= ind_r * 0.5) & (ev < ind_r)
    del ev, ind_r, change
    glen = (lambda m: rng.geometric(geom_p, m)) if geom_p is not None else (lambda m: np.ones(m, np.int64))
    ins_len = np.zeros(total, dtype=np.int32)
    ins_len[is_ins] = glen(int(is_ins.sum()))
    seq_start = offsets_of(lens)
    seq_end = seq_start + lens
    dpos = np.nonzero(is_del)[0]
    dlen = glen(len(dpos))
    if extra_pos is not None:
        extra_pos = np.asarray(extra_pos, dtype=np.int64)
        sel = np.nonzero(extra_pos >= 0)[0]
        p = seq_start[sel] + np.minimum(extra_pos[sel], np.maximum(lens[sel] - 1, 0))
        ins_k = np.asarray(extra_ins, dtype=bool)[sel]
        np.add.at(ins_len, p[ins_k], np.asarray(extra_len, dtype=np.int64)[sel][ins_k])
        dpos = np.concatenate([dpos, p[~ins_k]])
        dlen = np.concatenate([dlen, np.asarray(extra_len, dtype=np.int64)[sel][~ins_k]])
    # deleted spans: a difference array clipped at each sequence's end
    diff = np.zeros(total + 1, dtype=np.int32)
    owner = np.searchsorted(seq_start, dpos, side="right") - 1
    np.add.at(diff, dpos, 1)
    np.add.at(diff, np.minimum(dpos + dlen, seq_end[owner]), -1)
    kept = np.cumsum(diff[:-1], dtype=np.int32) == 0
    del diff

    def per_seq(counts):
        c = np.concatenate([np.zeros(1, np.int64), np.cumsum(counts, dtype=np.int64)])
        return c[seq_end] - c[seq_start]

    counts = ins_len + kept
    out_len = per_seq(counts)
    empty = np.nonzero((out_len == 0) & (lens > 0))[0]
    if len(empty):
        kept[seq_start[empty]] = True
        counts = ins_len + kept
        out_len = per_seq(counts)
    out_total = int(counts.sum())
    starts = np.cumsum(counts, dtype=np.int64) - counts
    is_src = np.zeros(out_total, dtype=bool)
    slot = (starts + ins_len)[kept]
    is_src[slot] = True
    out = np.empty(out_total, dtype=np.uint8)
    out[slot] = res[kept]
    out[~is_src] = _residues(rng, out_total - len(slot), protein)
    return out, offsets_of(out_len), out_len.astype(np.int32)


def mutate(rng, seq, identity, indel, protein=True, geom_p=None):
    """One sequence (uint8 array): mutate_many on a single sequence."""
    out, _, _ = mutate_many(rng, seq, np.zeros(1, np.int64), np.array([len(seq)]), identity, indel,
                            protein, geom_p)
    return out


def _random_lengths_buffer(rng, lens, protein=True):
    lens = np.asarray(lens, dtype=np.int64)
    return _residues(rng, int(lens.sum()), protein), offsets_of(lens), lens.astype(np.int32)


def protein_db_search(seed=2, n_targets=200_000, query_lengths=(100, 250, 500, 1000, 2000),
                      median=270.0, sigma=0.72, lo=20, hi=5000, homolog_frac=0.01,
                      homolog_identity=0.30, homolog_indel=0.02):
    """Protein database search: queries of the given lengths against
    log-normal-length targets (median 270, sigma 0.72 -> mean about 350,
    clipped to [20, 5000]); homolog_frac of the targets are homologs of a
    random query (homolog_identity identity, homolog_indel indels). Returns
    (queries: list[bytes], targets buffer, offsets, lengths)."""
    rng = np.random.default_rng(seed)
    queries = [_residues(rng, L).tobytes() for L in query_lengths]
    lens = np.clip(np.rint(rng.lognormal(np.log(median), sigma, n_targets)), lo, hi).astype(np.int64)
    homolog = rng.random(n_targets) < homolog_frac
    which = rng.integers(0, len(queries), n_targets)
    hk = np.nonzero(homolog)[0]
    qb = [np.frombuffer(q, dtype=np.uint8) for q in queries]
    if len(hk):
        src = np.concatenate([qb[w] for w in which[hk]])
        sl = np.array([len(qb[w]) for w in which[hk]], dtype=np.int64)
        hb, _, hl = mutate_many(rng, src, offsets_of(sl), sl, homolog_identity, homolog_indel)
        lens[hk] = hl
    else:
        hb = np.zeros(0, np.uint8)
    buf = _residues(rng, int(lens.sum()))
    offsets = offsets_of(lens)
    # homolog sequences replace the random residues of their slots
    if len(hk):
        hoff = offsets_of(lens[hk])
        dst = np.concatenate([np.arange(offsets[k], offsets[k] + lens[k]) for k in hk])
        srcix = np.concatenate([np.arange(o, o + l) for o, l in zip(hoff, lens[hk])])
        buf[dst] = hb[srcix]
    return queries, buf, offsets, lens.astype(np.int32)


def protein_query_vs_targets(seed=1, qlen=300, n_targets=1000, lo=100, hi=500):
    """One query of length qlen vs n_targets with lengths uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    q = _residues(rng, qlen).tobytes()
    lens = rng.integers(lo, hi + 1, n_targets).astype(np.int32)
    buf = _residues(rng, int(lens.sum()))
    return q, buf, offsets_of(lens), lens


def dna_read_windows(seed=3, n_pairs=1_000_000, lo=100, hi=300, flank=32, sub=0.05, ins=0.005, dele=0.005):
    """DNA reads vs their reference windows: window = uniform ACGT of length
    read+flank; read = the window's first read-length bases mutated with
    5% substitutions and 0.5% insertions / 0.5% deletions (lengths geometric
    p=0.5). Returns (reads buf, offs, lens, windows buf, offs, lens)."""
    rng = np.random.default_rng(seed)
    rl = rng.integers(lo, hi + 1, n_pairs).astype(np.int64)
    wl = rl + flank
    wbuf = DNA_BYTES[rng.integers(0, 4, int(wl.sum()))]
    woff = offsets_of(wl)
    # the first rl[k] bases of every window, then the mutations of all reads at once
    roff0 = offsets_of(rl)
    base = wbuf[np.repeat(woff - roff0, rl) + np.arange(int(rl.sum()))]
    rbuf, roff, rlen = mutate_many(rng, base, offsets_of(rl), rl, 1.0 - sub * 4 / 3, ins + dele,
                                   protein=False, geom_p=0.5)
    return rbuf, roff, rlen, wbuf, woff, wl.astype(np.int32)


def protein_all_vs_all(seed=4, n_seqs=4096, lo=50, hi=1500, family_frac=0.20, n_families=64,
                       identity=0.40, indel=0.03):
    """Protein all-vs-all set: n_seqs sequences with lengths uniform in
    [lo, hi] and residues at background frequencies; family_frac of them are
    members of n_families planted families (each a mutated copy of its
    family's ancestor, `identity` identity and `indel` indels; ancestor
    lengths uniform in [lo, hi]). Returns (buf, offs, lens)."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(lo, hi + 1, n_seqs).astype(np.int64)
    member = rng.random(n_seqs) < family_frac
    fam = rng.integers(0, n_families, n_seqs)
    anc_len = rng.integers(lo, hi + 1, n_families).astype(np.int64)
    anc_buf, anc_off, _ = _random_lengths_buffer(rng, anc_len)
    mk = np.nonzero(member)[0]
    if len(mk):
        src = np.concatenate([anc_buf[anc_off[f]:anc_off[f] + anc_len[f]] for f in fam[mk]])
        sl = anc_len[fam[mk]]
        mb, moff, ml = mutate_many(rng, src, offsets_of(sl), sl, identity, indel)
        lens[mk] = ml
    buf = _residues(rng, int(lens.sum()))
    offs = offsets_of(lens)
    for t, k in enumerate(mk):
        buf[offs[k]:offs[k] + lens[k]] = mb[moff[t]:moff[t] + ml[t]]
    return buf, offs, lens.astype(np.int32)


def all_pairs_count(n):
    """Pairs of the upper triangle (i < j) of n sequences."""
    return n * (n - 1) // 2


def dna_long_pairs(seed=5, n_pairs=20_000, lo=5_000, hi=50_000, div_lo=0.01, div_hi=0.15,
                   indel_share=0.30, indel_mean=3.0, big_frac=0.30, big_lo=50, big_hi=500, chunk=4000):
    """Long DNA pairs: A uniform ACGT of length U[lo, hi]; B = A with a
    per-pair divergence d ~ U[div_lo, div_hi] split 70/30 between
    substitutions and indels (indel lengths geometric with the given mean),
    plus one large insertion or deletion of U[big_lo, big_hi] bp in big_frac
    of the pairs. Generated `chunk` pairs at a time. Returns (A buf, offs,
    lens, B buf, offs, lens, divergences)."""
    rng = np.random.default_rng(seed)
    la = rng.integers(lo, hi + 1, n_pairs).astype(np.int64)
    div = rng.uniform(div_lo, div_hi, n_pairs)
    big = rng.random(n_pairs) < big_frac
    big_len = rng.integers(big_lo, big_hi + 1, n_pairs)
    big_ins = rng.random(n_pairs) < 0.5
    big_at = rng.random(n_pairs)
    a_all = DNA_BYTES[rng.integers(0, 4, int(la.sum()))]
    aoff = offsets_of(la)
    sub = div * (1.0 - indel_share)
    # indel events: each costs on average indel_mean bases of divergence
    ev = 2.0 * div * indel_share / indel_mean
    gp = 1.0 / indel_mean
    bs, bl = [], []
    for c0 in range(0, n_pairs, chunk):
        c1 = min(n_pairs, c0 + chunk)
        seg = a_all[aoff[c0]:aoff[c1 - 1] + la[c1 - 1]]
        pos = np.where(big[c0:c1], (big_at[c0:c1] * la[c0:c1]).astype(np.int64), -1)
        b, _, l = mutate_many(rng, seg, aoff[c0:c1] - aoff[c0], la[c0:c1], 1.0 - sub[c0:c1] * 4.0 / 3.0,
                              ev[c0:c1], protein=False, geom_p=gp, extra_pos=pos, extra_len=big_len[c0:c1],
                              extra_ins=big_ins[c0:c1])
        bs.append(b)
        bl.append(l)
    lb = np.concatenate(bl).astype(np.int32)
    return a_all, aoff, la.astype(np.int32), np.concatenate(bs), offsets_of(lb), lb, div
