"""The SDPA reader (brisk_b200/csrc/sdpa.cpp through bgpu_sdpa_read) against the reference's own
reader (read_sdpa, problem.c:426): tests/golden/sdpa_reader.json holds what oracle/_ref/brisk_ref
read from each file of a corpus of the format's rules and errors (made by
tests/golden/make_sdpa_golden.py: the problem as read, written back at %.17g, or the messages of a
refused file).  Then the reader's parallel form of the data section against its serial form, on
files large enough to be cut into several pieces, and its numbers against Python's float (both
correctly rounded, as strtod)."""
import json
import os

import numpy as np
import pytest

import brisk_b200
from refdir import REF_DIR

GOLD = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sdpa_reader.json")))
# the messages of read_sdpa itself (others in the reference's output come from later stages)
READER = ("non-numeric token", "non-integer index", "non-finite value", "bad entry", "off-diagonal entry in LP block",
          "invalid size", "malformed SDPA file", "line(s) of text after the last entry", "incomplete last entry")


def canonical(d):
    """The entries as the reference writes the problem it read: i <= j, duplicates summed, zero
    values left out, sorted by (block, matrix, i, j)."""
    acc = {}
    for mat, blk, i, j, v in zip(d.mat.tolist(), d.blk.tolist(), d.i.tolist(), d.j.tolist(), d.v.tolist()):
        key = (blk, mat, min(i, j), max(i, j))
        acc[key] = acc.get(key, 0.0) + v
    return [(k[1], k[0], k[2], k[3], float(acc[k]).hex()) for k in sorted(acc) if acc[k] != 0]


def ref_canonical(ents):
    return [(e[0], e[1], e[2], e[3], float(e[4]).hex()) for e in sorted(ents, key=lambda e: (e[1], e[0], e[2], e[3]))]


def write(path, text):
    with open(path, "w", newline="") as f:
        f.write(text)


@pytest.mark.parametrize("name", sorted(GOLD))
def test_reader_matches_reference(tmp_path, name):
    rec = GOLD[name]
    path = str(tmp_path / "case.dat-s")
    write(path, rec["text"])
    ref_msgs = [m.replace("<path>", path) for m in rec["messages"] if any(k in m for k in READER)]
    if rec["rc"] == 0:
        d, log = brisk_b200.read_sdpa_file(path)
        r = rec["read"]
        assert d.m == r["m"] and d.bs.tolist() == r["bs"]
        assert [float(x).hex() for x in d.c] == [float(x).hex() for x in r["c"]]
        assert canonical(d) == ref_canonical(r["entries"])
        for m in ref_msgs:
            assert m in log, (m, log)
    else:
        assert rec["rc"] == 2
        with pytest.raises(ValueError) as ei:
            brisk_b200.read_sdpa_file(path)
        log = str(ei.value)
        specific = [m for m in ref_msgs if "malformed SDPA file" not in m]
        if specific:
            assert specific[0] in log, (specific[0], log)
        else:
            assert "malformed SDPA file " + path in log, log


def big_text(seed, n_entries, fmt):
    """A one-block problem of order 60 with n_entries entries and values printed by fmt."""
    rng = np.random.default_rng(seed)
    m, n = 50, 60
    mat = rng.integers(0, m + 1, n_entries)
    i = rng.integers(1, n + 1, n_entries)
    j = rng.integers(1, n + 1, n_entries)
    v = rng.standard_normal(n_entries) * 10.0 ** rng.integers(-20, 20, n_entries)
    head = f"{m}\n1\n{n}\n" + " ".join(repr(float(x)) for x in rng.standard_normal(m)) + "\n"
    body = "".join(f"{a} 1 {b} {c} {fmt(x)}\n" for a, b, c, x in zip(mat.tolist(), i.tolist(), j.tolist(), v.tolist()))
    return head, body, (mat, i, j, v)


def arrays(d):
    return d.mat, d.blk, d.i, d.j, d.v


def test_parallel_parse_matches_serial_and_float(tmp_path):
    """About 13 MB (several 4 MB pieces): the parallel parse gives the serial parse's arrays (the
    same file with words after the last entry goes the serial way), and every value is Python's
    float of its text (repr: shortest round trip; %.25e: 26 significant digits)."""
    for fmt in (repr, lambda x: "%.25e" % x):
        head, body, (mat, i, j, v) = big_text(3, 400000, fmt)
        p1, p2 = str(tmp_path / "a.dat-s"), str(tmp_path / "b.dat-s")
        write(p1, head + body)
        write(p2, head + body + "END OF DATA\n")
        d1, log1 = brisk_b200.read_sdpa_file(p1)
        d2, log2 = brisk_b200.read_sdpa_file(p2)
        assert "text after the last entry" in log2 and log1 == ""
        for a, b in zip(arrays(d1), arrays(d2)):
            np.testing.assert_array_equal(a, b)
        keep = v != 0
        np.testing.assert_array_equal(d1.mat, mat[keep])
        np.testing.assert_array_equal(d1.i, i[keep])
        np.testing.assert_array_equal(d1.j, j[keep])
        want = np.array([float(fmt(x)) for x in v[keep].tolist()])
        assert d1.v.tobytes() == want.tobytes()


def test_fortran_exponents_across_piece_boundaries(tmp_path):
    """Every value written with a 'D' exponent: read as with 'e' wherever the pieces are cut (the
    header is padded so that the cuts move through the 13-character lines)."""
    head, body, _ = big_text(5, 700000, lambda x: "%.3e" % x)
    ref, _ = brisk_b200.read_sdpa_file(_w(tmp_path, "e.dat-s", head + body))
    dbody = body.replace("e+", "D+").replace("e-", "d-")
    for pad in range(0, 26, 5):
        d, _ = brisk_b200.read_sdpa_file(_w(tmp_path, "d.dat-s", head.replace("\n", " " * pad + "\n", 1) + dbody))
        for a, b in zip(arrays(ref), arrays(d)):
            np.testing.assert_array_equal(a, b)


def _w(tmp_path, name, text):
    p = str(tmp_path / name)
    write(p, text)
    return p


def test_first_fault_in_file_order_across_pieces(tmp_path):
    """Two bad entries far apart in a large file: the reference stops at the first in file order,
    so the parallel check reports that one."""
    head, body, _ = big_text(7, 500000, repr)
    lines = body.splitlines(keepends=True)
    lines[100000] = "1 1 61 1 1.0\n"        # index beyond the block: bad entry
    lines[400000] = "1 1 2.5 1 1.0\n"       # non-integer index, later in the file
    with pytest.raises(ValueError, match="bad entry 1 1 61 1"):
        brisk_b200.read_sdpa_file(_w(tmp_path, "f.dat-s", head + "".join(lines)))


def test_solve_file_reads_with_the_library_reader(tmp_path):
    """brisk_solve_file refuses a malformed file with exit code 2 before any GPU work (on a host
    without a GPU too)."""
    p = _w(tmp_path, "bad.dat-s", GOLD["err_non_integer_index"]["text"])
    res = brisk_b200.solve_file(p, verbose=False)
    assert res.exit_code == 2
    assert "non-integer index in entry 2 1 2.5 3 1.5" in res.log


REF_EXAMPLES = os.path.join(REF_DIR, "examples")
REF_BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "brisk_ref")


def _ref_examples():
    if not os.path.isdir(REF_EXAMPLES):
        return []
    return sorted(f for f in os.listdir(REF_EXAMPLES) if f.endswith(".dat-s"))


@pytest.mark.skipif(not os.path.exists(REF_BIN) or not _ref_examples(), reason="reference tree or oracle/_ref absent")
@pytest.mark.parametrize("fname", _ref_examples() or ["-"])
def test_reader_matches_reference_on_its_example_files(tmp_path, fname):
    """The reference's own example files (SDPLIB-style headers, braces and commas, LP blocks,
    comment lines): the reader's numbers equal what oracle/_ref/brisk_ref writes back with
    BRISK_WRITEFR (presolves off, the elimination of split free variables too), bit for bit after
    its canonical form."""
    import subprocess
    path = os.path.join(REF_EXAMPLES, fname)
    out = str(tmp_path / "read.dat-s")
    env = dict(os.environ, BRISK_NOBUSY="1", BRISK_WRITEFR=out)
    subprocess.run([REF_BIN, path, "-threads", "1", "-nohsd", "-sym", "none", "-symalg", "0", "-chordal", "0",
                    "-nofr", "-deprows", "0", "-freeelim", "0"], capture_output=True, env=env, timeout=300)
    assert os.path.exists(out)
    tok = open(out).read().split()
    m, nblk = int(tok[0]), int(tok[1])
    bs = [int(x) for x in tok[2:2 + nblk]]
    c = [float(x) for x in tok[2 + nblk:2 + nblk + m]]
    rest = tok[2 + nblk + m:]
    ents = [[int(rest[q]), int(rest[q + 1]), int(rest[q + 2]), int(rest[q + 3]), float(rest[q + 4])]
            for q in range(0, len(rest), 5)]
    d, _ = brisk_b200.read_sdpa_file(path)
    assert d.m == m and d.bs.tolist() == bs
    assert [float(x).hex() for x in d.c] == [float(x).hex() for x in c]
    assert canonical(d) == ref_canonical(ents)


def test_reader_takes_a_pipe(tmp_path):
    """A file that is not a regular one (a named pipe: no size to split by) is read to its end on
    one thread, with the same result as the regular file."""
    import threading
    text = GOLD["sdplib_style"]["text"]
    reg = _w(tmp_path, "reg.dat-s", text)
    fifo = str(tmp_path / "pipe.dat-s")
    os.mkfifo(fifo)

    def feed():
        with open(fifo, "w", newline="") as f:
            f.write(text)

    th = threading.Thread(target=feed)
    th.start()
    d_pipe, _ = brisk_b200.read_sdpa_file(fifo)
    th.join(timeout=30)
    d_reg, _ = brisk_b200.read_sdpa_file(reg)
    for a, b in zip(arrays(d_pipe), arrays(d_reg)):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(d_pipe.c, d_reg.c)
    assert d_pipe.bs.tolist() == d_reg.bs.tolist()


def test_reader_refuses_a_directory_and_a_missing_file(tmp_path):
    with pytest.raises(ValueError, match="is a directory"):
        brisk_b200.read_sdpa_file(str(tmp_path))
    with pytest.raises(ValueError, match="cannot open"):
        brisk_b200.read_sdpa_file(str(tmp_path / "absent.dat-s"))
