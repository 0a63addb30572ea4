"""Generate tests/golden/sdpa_reader.json: what the reference's SDPA reader (read_sdpa,
problem.c:426) makes of a corpus of small files covering its rules (comment lines, the separators
",{}()=", header lines with trailing text, Fortran exponents, number forms, text after the last
entry, an incomplete last entry, zero values, LP blocks) and its errors (non-integer or
out-of-range indices, non-finite values, non-numeric tokens, bad block sizes, short headers).

Runs oracle/_ref/brisk_ref (the reference compiled from its sources by oracle/Makefile) on each
file with the presolves off (the elimination of split free variables too) and BRISK_WRITEFR set: the reference then writes the problem as read
(entries sorted, i <= j, duplicates summed, values at %.17g so every double survives) and exits
before solving.  Records per case: the file's text, the exit code, the reader's messages (lines
starting "brisk:"; the file's path replaced by <path>) and, for a file read, m, the block sizes, c
and the entries as written.

usage: python tests/golden/make_sdpa_golden.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(ROOT, "oracle", "_ref", "brisk_ref")
OUT = os.path.join(ROOT, "tests", "golden", "sdpa_reader.json")
AS_GIVEN = ["-sym", "none", "-symalg", "0", "-chordal", "0", "-nofr", "-deprows", "0", "-freeelim", "0"]

# the base problem: m = 3, blocks of order 3 and 2; every entry below is one of its entries
BASE_ENTRIES = """0 1 1 1 1.0
0 1 1 2 0.25
0 1 3 3 2.0
0 2 1 2 -0.5
1 1 1 1 1.0
1 1 2 2 1.0
1 2 1 1 1.0
2 1 2 3 0.75
2 1 3 3 1.5
2 2 2 2 2.0
3 1 1 3 -1.25
3 2 1 1 0.5
3 2 2 2 0.5
"""
BASE = "3\n2\n3 2\n1.0 2.0 0.5\n" + BASE_ENTRIES

CASES = {
    "plain": BASE,
    "sdplib_style": ('"a comment line before the header\n* and another\n   3 =mdim\n   2 =nblocks\n'
                     "{3, 2}\n{1.0, 2.0, 0.5}\n" + BASE_ENTRIES.replace("0 1 1 2 0.25", "(0, 1, 1, 2) = 0.25")),
    "comments_in_data": BASE.replace("1 1 1 1 1.0\n", '1 1 1 1 1.0\n" a comment between entries 7 7 7 7 7\n'
                                     "   * another 1 2 3 4 5\n"),
    "fortran_exponents": BASE.replace("0.25", "2.5D-1").replace("1.5\n", "1.5d+00\n").replace("2.0\n", "2D0\n")
                             .replace("-1.25", "-.125D1").replace("0.75", "75.D-2"),
    "number_forms": BASE.replace("0.25", "+0.25").replace("-0.5", "-0x1p-1").replace("0.75", ".75")
                        .replace("1.5\n", "1.50000000000000000000000000001\n")
                        .replace("2 2 2 2 2.0", "2 2 2 2 2000000000000000000000000000000e-30")
                        .replace("3 2 1 1 0.5", "3 2 1 1 2.2250738585072011e-308")
                        .replace("3 2 2 2 0.5", "3 2 2 2 4.9e-324")
                        .replace("1 2 1 1 1.0", "+1 2 1 1 1.7976931348623157e308"),
    "lower_triangle_and_duplicates": BASE.replace("2 1 2 3 0.75", "2 1 3 2 0.75\n2 1 2 3 0.125")
                                         .replace("0 1 1 2 0.25", "0 1 2 1 0.25"),
    "layout": "3\n2\n3 2 1.0\t2.0\n0.5 0 1 1 1 1.0 0 1 1\n2 0.25\n" + BASE_ENTRIES.split("\n", 2)[2].replace("\n", "\t"),
    "err_header_line_rest_skipped": "3 2 3 2\n1.0\t2.0 0.5 0 1 1 1 1.0 0 1 1\n2 0.25\n" + BASE_ENTRIES.split("\n", 2)[2],
    "crlf": BASE.replace("\n", "\r\n"),
    "no_final_newline": BASE.rstrip("\n"),
    "zero_values": BASE + "1 1 3 3 0.0\n2 2 1 1 -0\n3 1 2 2 0e5\n",
    "negative_zero_index": BASE.replace("0 2 1 2 -0.5", "-0 2 1 2 -0.5"),
    "lp_block": "3\n3\n3 2 -2\n1.0 2.0 0.5\n" + BASE_ENTRIES + "1 3 1 1 1.0\n2 3 2 2 1.0\n0 3 2 2 -1.0\n",
    "text_after_last_entry": BASE + "BEGIN.COMMENT\nthese words end the data\n1 2 3\nEND.COMMENT\n",
    "incomplete_last_entry": BASE + "1 1 3\n",
    "err_text_then_entries": BASE + "note:\n1 1 1 1 1.0\n",
    "err_non_numeric_token": BASE.replace("2 1 3 3 1.5", "2 1 3 3 abc 1.5"),
    "err_glued_number": BASE.replace("2 1 3 3 1.5", "2 1 3 3 1.5x"),
    "err_non_integer_index": BASE.replace("2 1 3 3 1.5", "2 1 2.5 3 1.5"),
    "err_huge_index": BASE.replace("2 1 3 3 1.5", "2 1 3000000000 3 1.5"),
    "err_inf_value": BASE.replace("2 1 3 3 1.5", "2 1 3 3 inf"),
    "err_nan_value": BASE.replace("2 1 3 3 1.5", "2 1 3 3 nan"),
    "err_block_out_of_range": BASE.replace("2 1 3 3 1.5", "2 3 1 1 1.5"),
    "err_index_out_of_block": BASE.replace("2 2 2 2 2.0", "2 2 3 3 2.0"),
    "err_matrix_out_of_range": BASE.replace("2 1 3 3 1.5", "4 1 3 3 1.5"),
    "err_lp_off_diagonal": "3\n3\n3 2 -2\n1.0 2.0 0.5\n" + BASE_ENTRIES + "1 3 1 2 1.0\n",
    "err_block_size_zero": BASE.replace("3 2\n", "3 0\n", 1),
    "err_block_size_fraction": BASE.replace("3 2\n", "3 2.5\n", 1),
    "err_short_c": "3\n2\n3 2\n1.0 2.0\n",
    "err_no_nblk": "3\n",
    "err_fraction_nblk": BASE.replace("3\n2\n", "3\n2.5\n", 1),
    "err_first_fault_wins": BASE.replace("2 1 3 3 1.5", "2 1 3 3 1.5\n2 9 1 1 1.0").replace(
        "3 2 2 2 0.5", "3 2 2.5 2 0.5"),
}


def reference_read(text):
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "case.dat-s")
        with open(path, "w", newline="") as f:
            f.write(text)
        out = os.path.join(d, "read.dat-s")
        env = dict(os.environ, BRISK_NOBUSY="1", BRISK_WRITEFR=out)
        r = subprocess.run([REF, path, "-threads", "1", "-nohsd"] + AS_GIVEN, capture_output=True, text=True,
                           env=env, timeout=120)
        msgs = [ln.replace(path, "<path>") for ln in (r.stdout + r.stderr).splitlines() if ln.startswith("brisk:")]
        rec = {"text": text, "rc": r.returncode, "messages": msgs}
        if os.path.exists(out):
            tok = open(out).read().split()
            m, nblk = int(tok[0]), int(tok[1])
            bs = [int(x) for x in tok[2:2 + nblk]]
            c = [float(x) for x in tok[2 + nblk:2 + nblk + m]]
            rest = tok[2 + nblk + m:]
            ents = [[int(rest[q]), int(rest[q + 1]), int(rest[q + 2]), int(rest[q + 3]), float(rest[q + 4])]
                    for q in range(0, len(rest), 5)]
            rec["read"] = {"m": m, "bs": bs, "c": c, "entries": ents}
        return rec


def main():
    if not os.path.exists(REF):
        sys.exit(f"{REF} is missing: build it with `make -C oracle`")
    res = {name: reference_read(text) for name, text in CASES.items()}
    with open(OUT, "w") as f:
        json.dump(res, f, indent=1)
    for name, rec in res.items():
        print(f"{name:32s} rc {rec['rc']}  {'read' if 'read' in rec else '-':4s}  {rec['messages'][:2]}")


if __name__ == "__main__":
    main()
