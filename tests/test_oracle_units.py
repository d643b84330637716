"""The oracle against the reference crate's own unit-test vectors (CPU only).

Each test restates one `#[test]` of diamond-rust (file:line of the test
module given in the docstring) and checks the C++ oracle gives the same
answer.  These vectors pin the oracle before it is trusted as the checker of
the CUDA path.
"""
import math

import numpy as np
import pytest

import pyoracle as orc


def enc(s):
    return orc.encode(s)


# ---- alphabet.rs:95-121 -----------------------------------------------------
def test_alphabet_ncbi_order_roundtrip():
    """alphabet.rs tests: NCBI order, lower case, U -> C slot, unknown -> X."""
    symbols = "ARNDCQEGHILKMFPSTWYVBJZX*"
    for i, c in enumerate(symbols):
        assert list(enc(c)) == [i], c
    assert list(enc("a")) == [0]
    assert list(enc("U")) == [4]
    assert list(enc("?")) == [23]
    assert orc.decode(enc(symbols)) == symbols


def test_alphabet_strips_layout_characters():
    assert list(enc("AC-DE\nFG")) == [0, 4, 3, 6, 13, 7]


def test_alphabet_header_id():
    assert orc.seq_id(">sp|P1|ABC description here") == "sp|P1|ABC"
    assert orc.seq_id(">  lone") == "lone"


# ---- reduction.rs:86-116 ------------------------------------------------------
def test_murphy10_groups():
    b = lambda c: orc.bucket("murphy10", int(enc(c)[0]))[0]
    assert orc.bucket("murphy10", 0)[1] == 10
    assert b("A") == 0
    assert b("K") == 1
    assert b("R") == 1
    assert b("L") == b("M")


def test_no_reduction_is_bijective():
    for i in range(20):
        bk, size = orc.bucket("none", i)
        assert size == 20 and bk == i


def test_sensitivity_presets_pick_reduction():
    assert orc.reduction_size_for("default") == 10
    assert orc.reduction_size_for("sensitive") == 10
    assert orc.reduction_size_for("very-sensitive") == 9
    assert orc.reduction_size_for("ultra-sensitive") == 10


# ---- shape.rs:231-299 -------------------------------------------------------
def test_contiguous_seed_key():
    seq = enc("MKWV")
    assert orc.shape_packed(seq, 0, "111", 2) == 12 * 400 + 11 * 20 + 17
    assert orc.shape_packed(seq, 2, "111", 2) is None


def test_spaced_seed_uses_only_ones():
    assert orc.shape_packed(enc("ACD"), 0, "101", 2) == 3


def test_reduced_seed_merges_similar_residues():
    assert orc.shape_packed(enc("LI"), 0, "11", 0) == orc.shape_packed(enc("LL"), 0, "11", 0)


def test_shape_presets():
    s = orc.shapes_for("default")
    assert s == ["111101110111", "111011010010111"]
    assert all(c.count("1") == 10 for c in s)
    sens = orc.shapes_for("sensitive")
    assert len(sens) == 16
    assert orc.shapes_for("more-sensitive") == sens
    vs = orc.shapes_for("very-sensitive")
    assert len(vs) == 16 and vs[0] == "11110111" and vs[0].count("1") == 7


# ---- seed.rs:175-216 ---------------------------------------------------------
def test_identical_sequences_share_seeds():
    cut = 0.8 * math.log(2) * 4
    a = enc("MKWVTFGCPD")
    q = orc.seed_build([a], "1111", 0, base=0, cut=cut)
    r = orc.seed_build([a], "1111", 0, base=7, cut=cut)
    assert len(q) == 7 and len(r) == 7
    hits = orc.seed_join(q, r, 1)
    on7 = sorted([h for h in hits if h[2] == 7], key=lambda h: h[1])
    assert len(on7) == 7
    assert (on7[0][1], on7[0][3]) == (0, 0)


def test_low_complexity_seeds_are_filtered():
    cut = 0.8 * math.log(2) * 8
    assert not orc.seed_is_complex(enc("AAAAAAAAAA"), "11111111", 0, cut)
    assert orc.seed_is_complex(enc("MKWVTFGCPD"), "11111111", 0, cut)
    assert not orc.seed_is_complex(enc("AAAAAACC"), "11111111", 0, cut)
    assert orc.seed_is_complex(enc("AAAAAACC"), "11111111", 0, 0.8)


def test_chunking_covers_everything():
    assert orc.chunks(10, 4) == [(0, 3), (3, 6), (6, 8), (8, 10)]
    assert sum(b - a for a, b in orc.chunks(10, 4)) == 10
    assert orc.chunks(0, 4) == []


def test_ln_factorial_is_a_sequential_sum():
    """seed.rs:29-38: lnfact[n] = sum of ln(k), k = 2..n, in order (33 entries)."""
    acc = 0.0
    assert orc.ln_factorial(0) == 0.0 and orc.ln_factorial(1) == 0.0
    for n in range(2, 33):
        acc += math.log(n)
        assert orc.ln_factorial(n) == acc


# ---- ungapped.rs:99-129 -------------------------------------------------------

def _self_score(seq):
    return sum(orc.xdrop(seq[i:i + 1], seq[i:i + 1], 0, 0, xd=1000)[3] for i in range(len(seq)))


def test_identical_region_extends_over_the_whole_seed():
    q = enc("MKWVTFISLLFLFSSAYSR")
    qs, ss, ln, sc = orc.xdrop(q, q, 0, 0, xd=40)
    assert qs == 0 and ln == len(q)
    assert sc == _self_score(q)


def test_stops_at_the_xdrop_boundary():
    q = enc("WWWWWWWWWWCCCCCCCCCC")
    s = enc("WWWWWWWWWWDDDDDDDDDD")
    _, _, ln, sc = orc.xdrop(q, s, 0, 0, xd=5)
    assert ln == 10 and sc == 110


def test_coordinates_are_clipped_at_the_sequence_start():
    q = enc("AAAAAA")
    qs, ss, ln, _ = orc.xdrop(q, q, 0, 0, xd=30)
    assert (qs, ss) == (0, 0) and ln == 6


# ---- gapped.rs:299-338 ---------------------------------------------------------
def _extend(q, s, band):
    """gapped::extend with anchor (0, 0): extend_span over diagonals [-band, band]."""
    return orc.extend_span(q, s, -band, band)[0]


def test_identical_sequences_align_end_to_end():
    q = enc("MKWVTFISLLFLFSSAYSR")
    a = _extend(q, q, 30)
    score, qb, qe, sb, se, ident, pos, mism, gapo, gaps, length, ops = a
    assert score == _self_score(q)
    assert (qb, sb) == (0, 0) and (qe, se) == (len(q), len(q))
    assert ident == len(q) and mism == 0 and gaps == 0


def test_gaps_are_placed_in_the_shorter_sequence():
    q = enc("MKWVTFISLLFLFSSAYSR")
    s = enc("MKWVTFISLLLFSSAYSR")
    a = _extend(q, s, 30)
    assert a[9] > 0
    assert a[5] == len(s)
    assert a[0] < _self_score(s)


def test_unrelated_sequences_give_no_alignment():
    assert _extend(enc("WWWWWWWWWW"), enc("AAAAAAAAAA"), 15) is None


def test_band_widths():
    assert [orc.band_for(n) for n in (10, 50, 120, 400, 900)] == [12, 16, 30, 64, 64]


# ---- search.rs:410-454 ----------------------------------------------------------
@pytest.mark.parametrize("name,cut", [("faster", 0.9), ("fast", 0.9), ("default", 0.8), ("mid-sensitive", 1.0),
                                      ("sensitive", 1.0), ("more-sensitive", 1.0), ("very-sensitive", 1.0),
                                      ("ultra-sensitive", 1.0)])
def test_seed_cut_follows_the_sensitivity_preset(name, cut):
    assert orc.seed_cut_for(name) == cut


def test_explicit_seed_cut_overrides_the_preset():
    assert orc.seed_cut_for("very-sensitive", 0.5) == 0.5


@pytest.mark.parametrize("name,n", [("faster", 4), ("fast", 4), ("default", 4), ("mid-sensitive", 4),
                                    ("sensitive", 4), ("more-sensitive", 4), ("very-sensitive", 1),
                                    ("ultra-sensitive", 1)])
def test_index_chunks_follow_the_sensitivity_preset(name, n):
    assert orc.index_chunks_for(name) == n
    assert orc.index_chunks_for(name, 7) == 7


# ---- matrix.rs:278-321 ----------------------------------------------------------
def test_blosum62_defaults():
    A, W = 0, 17
    assert orc.xdrop([A], [A], 0, 0, xd=100)[3] == 4
    assert orc.xdrop([W], [W], 0, 0, xd=100)[3] == 11
    assert orc.extend_span(np.array([A], np.uint8), np.array([W], np.uint8), 0, 0)[0] is None  # A/W = -3


def test_bit_scores_are_blast_compatible():
    b = orc.bit_score(100)
    assert abs(b - 43.1) < 0.1
    assert orc.raw_score(b) == 100


def test_evalues_match_diamond_alp_statistics():
    got = orc.evalue(198, 497, 601, 2_263_996)
    assert abs(got / 7.60e-17 - 1.0) < 0.01


def test_blast_evalues_match_the_formula():
    expected = 0.041 * 100.0 * 1e6 * math.exp(-0.267 * 100.0)
    got = orc.evalue_blast(100, 100, 1_000_000)
    assert abs(got / expected - 1.0) < 1e-12


def test_unsupported_gap_costs_and_unknown_matrix_are_rejected():
    assert orc.matrix_ok("BLOSUM62")
    assert not orc.matrix_ok("BLOSUM62", 42, 7)
    assert not orc.matrix_ok("NOPE")


# ---- alp.rs:387-418 ----------------------------------------------------------------
def test_log_erfc_matches_reference_values():
    assert orc.log_erfc(0.0) == 0.0
    assert abs(orc.log_erfc(1.0) - (-1.8496055099332485)) < 1e-12
    assert abs(orc.log_erfc(4.0) - (-17.987778312103007)) < 1e-11
    assert abs(orc.log_erfc(5.0) - (-27.200889545537436)) < 1e-11
    assert abs(orc.log_erfc(-5.0) - 0.6931471805591766) < 1e-12
    assert abs(orc.log_erfc(-20.0) - math.log(2)) < 1e-15


@pytest.mark.parametrize("raw,slen,expected", [(818, 454, 3.21e-105), (262, 456, 3.89e-25), (198, 601, 7.60e-17)])
def test_alp_evalues_match_diamond(raw, slen, expected):
    got = orc.evalue(raw, 497, slen, 2_263_996)
    assert abs(got / expected - 1.0) < 0.01


def test_weak_hits_stay_blast_like():
    e = orc.evalue(60, 300, 300, 1_000_000)
    blast = orc.evalue_blast(60, 300, 1_000_000)
    assert e > 0 and math.isfinite(e)
    assert abs(math.log(e / blast)) < 3.0


# ---- output.rs:257-296 ------------------------------------------------------------
def test_outfmt_fields():
    f = orc.parse_outfmt(["6"])
    assert len(f) == 12 and f[0] == "qseqid" and f[11] == "bitscore"
    assert orc.parse_outfmt(["6", "qseqid", "qframe", "btop"]) == ["qseqid", "qframe", "btop"]
    assert orc.parse_outfmt(["6", "nope"]) is None
    assert orc.parse_outfmt(["7"]) is None


def test_evalues_are_formatted_like_diamond():
    assert orc.fmt_evalue(0.0) == "0.0"
    assert orc.fmt_evalue(0.001) == "1.00e-3"
    assert orc.fmt_evalue(4.7e-45) == "4.70e-45"
    assert orc.fmt_evalue(3.21e-105) == "3.21e-105"


def test_doubles_are_formatted_like_diamond():
    assert orc.fmt_double(319.7) == "319"
    assert orc.fmt_double(105.49) == "105"
    assert orc.fmt_double(80.87) == "80.9"
    assert orc.fmt_double(22.581) == "22.6"


# ---- hsp.rs:115-160 ------------------------------------------------------------------
def test_frames_follow_diamond_numbering():
    assert [orc.q_frame(f) for f in range(6)] == [1, 2, 3, -1, -2, -3]


def test_reverse_frame_maps_back_to_forward_strand():
    assert orc.nt_range(3, 2, 5, 30) == (30 - 15, 30 - 6)


# ---- translate.rs:140-187 ---------------------------------------------------------------
def test_standard_code_is_used():
    assert list(orc.translate_frame("ATGGCCTAA", 0)) == list(enc("MA*"))
    assert list(orc.translate_frame("TTTTTCCTT", 0)) == list(enc("FFL"))
    assert list(orc.translate_frame("atgaaa", 0)) == list(enc("MK"))


def test_ambiguous_codons_become_x():
    assert list(orc.translate_frame("ATGNNTAAA", 0)) == list(enc("MXK"))
    assert list(orc.translate_frame("ATGTAA", 0)) == list(enc("M*"))


def test_reverse_frames_read_the_complement():
    f = orc.six_frames("ATGAAATTT")
    assert list(f[0]) == list(enc("MKF"))
    assert list(f[3]) == list(enc("KFH"))


def test_short_orfs_are_masked():
    assert list(orc.mask_short_orfs(enc("MK*MKF*WWWW"), 3)) == list(enc("XX*MKF*WWWW"))
    assert orc.min_orf_len(20) == 1 and orc.min_orf_len(50) == 20 and orc.min_orf_len(150) == 40
    assert orc.min_orf_len(150, 7) == 7
