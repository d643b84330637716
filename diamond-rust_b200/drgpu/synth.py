"""Seeded synthetic protein data with the shapes of the benchmark workloads.

Databases and queries are drawn as the workload definitions describe:
  * residues iid from the BLOSUM62 background frequencies (NCBI order, the
    table the reference ships in matrix.rs:16-19), normalised;
  * lengths lognormal with sigma 0.57 in log space (mu = ln(mean) - sigma^2/2)
    and clipped to a range -- sigma 0.57 reproduces a median/mean of 245/288;
  * a fraction of database sequences carry a 10-30 residue homopolymer run;
  * planted homologs: a query segment mutated with BLOSUM62 target
    frequencies q_ij = p_i p_j exp(lambda_u s_ij) to a target identity, with
    indels at 0.02 per site of geometric length (mean 3), embedded in random
    flanks.
Everything is driven by numpy's PCG64 with a fixed seed, so the same call
returns the same data on every machine.
"""
from __future__ import annotations

import numpy as np

AA = "ARNDCQEGHILKMFPSTWYVBJZX*"
BACKGROUND = np.array([0.074, 0.052, 0.045, 0.054, 0.025, 0.034, 0.054, 0.074, 0.026, 0.068, 0.099, 0.058, 0.025,
                       0.047, 0.039, 0.057, 0.051, 0.013, 0.032, 0.073])
BACKGROUND = BACKGROUND / BACKGROUND.sum()
SIGMA = 0.57

def _blosum62_from_tables():
    """The 20x20 canonical block of BLOSUM62 from the package's score tables."""
    import os
    import re
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "csrc", "host",
                        "score_tables.inc")
    text = open(path).read()
    m = re.search(r'\{"BLOSUM62",[^\n]*\n\s*\{([-0-9,]+)\}', text)
    vals = np.array([int(v) for v in m.group(1).split(",")], dtype=np.float64).reshape(25, 25)
    return vals[:20, :20]


B62 = _blosum62_from_tables()


def _lambda_u():
    lo, hi = 1e-6, 2.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        f = (BACKGROUND[:, None] * BACKGROUND[None, :] * np.exp(mid * B62)).sum() - 1.0
        if f > 0:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


LAMBDA_U = _lambda_u()
_Q = BACKGROUND[:, None] * BACKGROUND[None, :] * np.exp(LAMBDA_U * B62)
_Q = _Q / _Q.sum()
# substitution distribution given the original residue, excluding identity
_SUB = _Q.copy()
np.fill_diagonal(_SUB, 0.0)
_SUB = _SUB / _SUB.sum(axis=1, keepdims=True)
_SUB_CDF = np.cumsum(_SUB, axis=1)


def lognormal_lengths(rng, n, mean, lo, hi):
    mu = np.log(mean) - SIGMA * SIGMA / 2.0
    return np.clip(np.round(rng.lognormal(mu, SIGMA, size=n)), lo, hi).astype(np.int64)


def random_protein(rng, n):
    return rng.choice(20, size=int(n), p=BACKGROUND).astype(np.uint8)


def mutate(rng, seq, identity, indel_rate=0.02, indel_mean=3.0):
    """Substitutions toward `identity` by target frequencies, plus indels."""
    seq = np.asarray(seq, dtype=np.uint8)
    keep = rng.random(len(seq)) < identity
    u = rng.random(len(seq))
    # ambiguous letters (B/J/Z/X/*) are replaced by a background residue
    subs = np.array([np.searchsorted(_SUB_CDF[a], x) if a < 20 else np.searchsorted(np.cumsum(BACKGROUND), x)
                     for a, x in zip(seq, u)], dtype=np.int64)
    subs = np.minimum(subs, 19).astype(np.uint8)
    out = np.where(keep, seq, subs).astype(np.uint8)
    res = []
    i = 0
    p_geom = 1.0 / indel_mean
    while i < len(out):
        if rng.random() < indel_rate:
            L = int(rng.geometric(p_geom))
            if rng.random() < 0.5:
                res.extend(random_protein(rng, L).tolist())  # insertion
            else:
                i += L  # deletion
                continue
        res.append(int(out[i]))
        i += 1
    return np.array(res, dtype=np.uint8)


def planted_homolog(rng, query, seg_lo, seg_hi, id_lo, id_hi, total_len):
    """A DB sequence holding a mutated copy of a query segment in random flanks."""
    qlen = len(query)
    seg = int(rng.integers(min(seg_lo, qlen), min(seg_hi, qlen) + 1))
    start = int(rng.integers(0, qlen - seg + 1))
    core = mutate(rng, query[start:start + seg], float(rng.uniform(id_lo, id_hi)))
    flank = max(0, int(total_len) - len(core))
    left = int(rng.integers(0, flank + 1))
    return np.concatenate([random_protein(rng, left), core, random_protein(rng, flank - left)]).astype(np.uint8)


def make_db(rng, n_seqs, mean=288, lo=30, hi=5000, homopolymer_frac=0.02):
    lens = lognormal_lengths(rng, n_seqs, mean, lo, hi)
    seqs = [random_protein(rng, L) for L in lens]
    for i in np.nonzero(rng.random(n_seqs) < homopolymer_frac)[0]:
        s = seqs[i]
        run = int(rng.integers(10, 31))
        if len(s) > run:
            at = int(rng.integers(0, len(s) - run + 1))
            s[at:at + run] = rng.integers(0, 20)
    return seqs


class Workload:
    """Database and queries (lists of uint8 residue arrays) with FASTA ids."""

    def __init__(self, db, queries, name):
        self.db = db
        self.queries = queries
        self.name = name
        self.db_ids = [f"S{i}" for i in range(len(db))]
        self.query_ids = [f"Q{i}" for i in range(len(queries))]

    @property
    def db_letters(self):
        return int(sum(len(s) for s in self.db))

    @property
    def query_letters(self):
        return int(sum(len(s) for s in self.queries))

    def write_fasta(self, db_path, query_path):
        for path, seqs, ids in ((db_path, self.db, self.db_ids), (query_path, self.queries, self.query_ids)):
            with open(path, "w") as f:
                for i, s in zip(ids, seqs):
                    f.write(f">{i} synthetic\n")
                    txt = "".join(AA[c] for c in s)
                    for k in range(0, len(txt), 80):
                        f.write(txt[k:k + 80] + "\n")


def workload(config_id: int, scale: float = 1.0, n_queries=None, n_db=None, seed_offset=0) -> Workload:
    """Synthetic inputs of a benchmark configuration.

    1: 7,860-sequence DB, one 497-aa query with 7 planted homologs.
    2: 7,860-sequence DB, 1,000 queries (mean 350, 50-1500 aa), 5 homologs each.
    scale shrinks the counts for quick tests; n_queries / n_db override them.
    """
    rng = np.random.Generator(np.random.PCG64(20261203 + config_id + seed_offset))
    if config_id == 1:
        ndb = n_db or max(8, int(7860 * scale))
        db = make_db(rng, ndb)
        q = random_protein(rng, 497)
        slots = rng.choice(ndb, size=min(7, ndb), replace=False)
        for s in slots:
            db[s] = planted_homolog(rng, q, 200, 497, 0.30, 0.70, len(db[s]) + 200)
        return Workload(db, [q], "config1")
    if config_id == 2:
        ndb = n_db or max(8, int(7860 * scale))
        nq = n_queries or max(1, int(1000 * scale))
        queries = [random_protein(rng, L) for L in lognormal_lengths(rng, nq, 350, 50, 1500)]
        db = make_db(rng, ndb)
        n_plant = min(ndb, 5 * nq)
        slots = rng.choice(ndb, size=n_plant, replace=False)
        for k, s in enumerate(slots):
            q = queries[k // 5]
            db[s] = planted_homolog(rng, q, 30, len(q), 0.25, 0.70, max(len(db[s]), 40))
        return Workload(db, queries, "config2")
    if config_id == 3:
        ndb = n_db or max(8, int(2_000_000 * scale))
        nq = n_queries or max(1, int(50_000 * scale))
        queries = [random_protein(rng, L) for L in lognormal_lengths(rng, nq, 350, 20, 2000)]
        db = make_db(rng, ndb)
        with_homologs = rng.random(nq) < 0.10
        slot = 0
        order = rng.permutation(ndb)
        for qi in np.nonzero(with_homologs)[0]:
            q = queries[qi]
            for _ in range(int(rng.integers(1, 21))):
                if slot >= ndb:
                    break
                s = order[slot]
                slot += 1
                db[s] = planted_homolog(rng, q, min(30, len(q)), len(q), 0.25, 0.70, max(len(db[s]), 40))
        return Workload(db, queries, "config3")
    raise ValueError(f"unknown workload {config_id}")


# The standard genetic code, codons in T, C, A, G base order.
CODON_TABLE = "FFLLSSSSYY**CC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG"
_BASES = "TCAG"
_SYNONYMS = {}
for _i, _aa in enumerate(CODON_TABLE):
    _SYNONYMS.setdefault(_aa, []).append(_BASES[_i // 16] + _BASES[(_i // 4) % 4] + _BASES[_i % 4])
_COMPLEMENT = str.maketrans("ACGT", "TGCA")


def reverse_translate(rng, protein, sub_rate=0.01):
    """Nucleotides coding for `protein` (uniform synonymous codons), with substitutions."""
    nt = []
    for c in protein:
        aa = AA[c] if c < 20 else "*"
        cod = _SYNONYMS.get(aa) or _SYNONYMS["*"]
        nt.append(cod[int(rng.integers(0, len(cod)))])
    s = list("".join(nt))
    for k in np.nonzero(rng.random(len(s)) < sub_rate)[0]:
        s[k] = "ACGT"[int(rng.integers(0, 4))]
    return "".join(s)


class ReadWorkload:
    """blastx input: a protein DB and nucleotide reads (strings)."""

    def __init__(self, db, reads, name):
        self.db = db
        self.reads = reads
        self.name = name
        self.db_ids = [f"S{i}" for i in range(len(db))]
        self.read_ids = [f"R{i}" for i in range(len(reads))]

    def write_fasta(self, db_path, read_path):
        with open(db_path, "w") as f:
            for i, s in zip(self.db_ids, self.db):
                f.write(f">{i} synthetic\n" + "".join(AA[c] for c in s) + "\n")
        with open(read_path, "w") as f:
            for i, r in zip(self.read_ids, self.reads):
                f.write(f">{i} read\n{r}\n")


def read_workload(scale: float = 1.0, n_reads=None, n_db=None, seed_offset=0) -> ReadWorkload:
    """blastx configuration: reads of 150-300 nt against the 2M-sequence protein DB
    generator; 30 % of the reads are reverse-translated fragments of DB proteins
    (random strand and frame, 1 % substitutions), the rest random ACGT at 50 % GC."""
    rng = np.random.Generator(np.random.PCG64(20261203 + 4 + seed_offset))
    ndb = n_db or max(8, int(2_000_000 * scale))
    nr = n_reads or max(1, int(500_000 * scale))
    db = make_db(rng, ndb)
    reads = []
    for _ in range(nr):
        L = int(rng.integers(150, 301))
        if rng.random() < 0.30:
            p = db[int(rng.integers(0, ndb))]
            n_aa = L // 3 + 2
            if len(p) > n_aa:
                a = int(rng.integers(0, len(p) - n_aa + 1))
                p = p[a:a + n_aa]
            nt = reverse_translate(rng, p)
            off = int(rng.integers(0, 3))
            nt = (nt[off:] + "".join("ACGT"[int(x)] for x in rng.integers(0, 4, 3)))[:L]
            if rng.random() < 0.5:
                nt = nt.translate(_COMPLEMENT)[::-1]
            reads.append(nt)
        else:
            reads.append("".join("ACGT"[int(x)] for x in rng.integers(0, 4, L)))
    return ReadWorkload(db, reads, "config4")
