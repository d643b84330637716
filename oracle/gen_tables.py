#!/usr/bin/env python3
"""Generate the scoring-matrix and erfc-coefficient tables as a C include.

The numbers are data that must be identical to the reference for E-values and
alignment scores to agree bit for bit: the NCBI BLOSUM/PAM score tables with
their published gapped (lambda, K, alpha, alpha_v, sigma) rows, and GSL's
Chebyshev coefficients for erfc.  They are read from the reference sources
(src/matrix_data.rs and src/alp.rs) and written, unchanged in value, to

  oracle/score_tables.inc                       (the CPU oracle's copy)
  diamond-rust_b200/csrc/host/score_tables.inc  (the product's copy)

Usage: python oracle/gen_tables.py REFERENCE_ROOT   (the diamond-rust source tree)
"""
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit(__doc__)
ref = sys.argv[1]
here = os.path.dirname(os.path.abspath(__file__))
repo = os.path.dirname(here)


def num(tok):
    return tok.replace("_", "")


def parse_matrices(text):
    out = []
    for block in re.split(r"StdMatrix \{", text)[1:]:
        m = re.search(r'name:\s*"([^"]+)"', block)
        if m is None:  # the struct definition itself
            continue
        name = m.group(1)
        gap = re.search(r"default_gap:\s*\((-?\d+),\s*(-?\d+)\)", block)
        ung = re.search(r"ungapped:\s*\(([-\d._eE]+),\s*([-\d._eE]+)\)", block)
        sc = re.search(r"scores:\s*\[(.*?)\],\s*params:", block, re.S).group(1)
        vals = [int(v) for v in re.findall(r"-?\d+", sc)]
        assert len(vals) == 625, (name, len(vals))
        pr = re.search(r"params:\s*&\[(.*?)\],\s*\}", block, re.S).group(1)
        rows = re.findall(r"\(([^)]*)\)", pr)
        params = []
        for r in rows:
            t = [x.strip() for x in r.split(",") if x.strip()]
            assert len(t) == 7
            params.append((int(t[0]), int(t[1])) + tuple(num(x) for x in t[2:]))
        out.append((name, (int(gap.group(1)), int(gap.group(2))), (num(ung.group(1)), num(ung.group(2))), vals, params))
    return out


def parse_array(text, name):
    m = re.search(r"const %s: \[f64; (\d+)\] = \[(.*?)\];" % name, text, re.S)
    n = int(m.group(1))
    vals = [num(v) for v in re.findall(r"-?[\d_]+\.[\d_]+(?:e-?\d+)?", m.group(2))]
    assert len(vals) == n, (name, n, len(vals))
    return vals


def main():
    mtext = open(os.path.join(ref, "src/matrix_data.rs")).read()
    atext = open(os.path.join(ref, "src/alp.rs")).read()
    mats = parse_matrices(mtext)
    lines = ["// Generated by oracle/gen_tables.py -- do not edit.",
             "// NCBI score tables with their gapped Gumbel parameter rows, and GSL erfc",
             "// Chebyshev coefficients (values identical to the reference's tables).",
             "#pragma once", ""]
    lines.append("struct StdParamRow { int go, ge; double lambda, k, alpha, alpha_v, sigma; };")
    lines.append("struct StdMatrixDef { const char* name; int default_go, default_ge; double u_alpha, u_alpha_v;"
                 " signed char scores[625]; int n_params; StdParamRow params[16]; };")
    lines.append("static const StdMatrixDef kStdMatrices[] = {")
    for name, gap, ung, vals, params in mats:
        lines.append('  {"%s", %d, %d, %s, %s,' % (name, gap[0], gap[1], ung[0], ung[1]))
        lines.append("   {" + ",".join(str(v) for v in vals) + "},")
        lines.append("   %d, {" % len(params))
        for p in params:
            lines.append("     {%d, %d, %s, %s, %s, %s, %s}," % p)
        lines.append("   }},")
    lines.append("};")
    lines.append("static const int kNumStdMatrices = %d;" % len(mats))
    for arr in ("ERFC_XLT1", "ERFC_X15", "ERFC_X510"):
        v = parse_array(atext, arr)
        lines.append("static const double k%s[%d] = {%s};" % (arr.title().replace("_", ""), len(v), ", ".join(v)))
    m = re.search(r"fn erfc8_sum.*?const P: \[f64; 6\] = \[(.*?)\];.*?const Q: \[f64; 7\] = \[(.*?)\];", atext, re.S)
    p = [num(x) for x in re.findall(r"-?[\d_]+\.[\d_]+", m.group(1))]
    q = [num(x) for x in re.findall(r"-?[\d_]+\.[\d_]+", m.group(2))]
    assert len(p) == 6 and len(q) == 7
    lines.append("static const double kErfc8P[6] = {%s};" % ", ".join(p))
    lines.append("static const double kErfc8Q[7] = {%s};" % ", ".join(q))
    m = re.search(r"fn log_erfc.*?if x \* x < 10\.0 \* ROOT6_EPS \{(.*?)let mut series", atext, re.S)
    cs = re.findall(r"const (C\d+): f64 = (-?[\d_.]+);", m.group(1))
    names = [c[0] for c in cs]
    assert names == ["C5", "C6", "C7", "C8", "C9", "C10", "C11", "C12", "C13", "C14"], names
    lines.append("static const double kLogErfcSeries[10] = {%s};  // C5..C14" % ", ".join(num(c[1]) for c in cs))
    body = "\n".join(lines) + "\n"
    for dst in (os.path.join(here, "score_tables.inc"),
                os.path.join(repo, "diamond-rust_b200", "csrc", "host", "score_tables.inc")):
        with open(dst, "w") as f:
            f.write(body)
        print("wrote", dst)


if __name__ == "__main__":
    main()
