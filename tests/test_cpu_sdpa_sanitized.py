"""The SDPA reader (brisk_b200/csrc/sdpa.cpp, host C++) under AddressSanitizer and
UndefinedBehaviorSanitizer: compiled here with g++ and a small driver, then run on seeded mutations
of the reader corpus (tests/golden/sdpa_reader.json: bytes replaced, inserted or removed, files cut
short, NULs, separators, Fortran exponents, out-of-range numbers) and on a multi-piece file with
mutations, read by several threads.  Every file must end in a result or a clean error, with no
sanitizer report."""
import json
import os
import random
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "brisk_b200", "csrc")

DRIVER = r"""
#include "solver.h"
#include <cstdarg>
#include <cstdio>
namespace bsolve {
void log_printf(int, const char *fmt, ...) { va_list ap; va_start(ap, fmt); vfprintf(stderr, fmt, ap); va_end(ap); }
}
int main(int argc, char **argv) {
    int ok = 0, bad = 0;
    for (int a = 1; a < argc; a++) {
        bsolve::InputData in;
        std::string err;
        if (bsolve::read_sdpa_file(argv[a], in, err) == 0) ok++; else bad++;
    }
    printf("ok %d bad %d\n", ok, bad);
    return 0;
}
"""

ALPHABET = list("0123456789 \t\n\r.,{}()=+-eEdDx*\"abcinf\0") + ["1e308", "1e-400", "-0", "2147483648", "99999999999",
                                                                 "nan"]


def mutate(rng, text, rounds):
    t = list(text)
    for _ in range(rounds):
        op, pos = rng.random(), rng.randrange(len(t) + 1)
        if op < 0.4 and t:
            t[min(pos, len(t) - 1)] = rng.choice(ALPHABET)
        elif op < 0.7:
            t.insert(pos, rng.choice(ALPHABET))
        elif op < 0.85 and t:
            del t[min(pos, len(t) - 1)]
        else:
            t = t[:pos]
    return "".join(t)


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ absent")
def test_reader_is_clean_under_address_and_ub_sanitizers(tmp_path):
    drv = tmp_path / "drv.cpp"
    drv.write_text(DRIVER)
    exe = str(tmp_path / "rd")
    subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
                    "-fno-omit-frame-pointer", "-I" + CSRC, os.path.join(CSRC, "sdpa.cpp"), str(drv), "-o", exe,
                    "-pthread"], check=True, capture_output=True, timeout=300)
    gold = json.load(open(os.path.join(ROOT, "tests", "golden", "sdpa_reader.json")))
    texts = [v["text"] for v in gold.values()]
    rng = random.Random(2026)
    files = []
    for q in range(400):
        p = tmp_path / f"f{q}.dat-s"
        with open(p, "w", newline="") as f:
            f.write(mutate(rng, rng.choice(texts), rng.randint(1, 8)))
        files.append(str(p))
    # a multi-piece file (about 13 MB: several reader threads), a few mutations in it
    lines = ["50\n1\n60\n" + " ".join(str(1.0 + t) for t in range(50)) + "\n"]
    for q in range(500000):
        lines.append(f"{q % 51} 1 {q % 60 + 1} {(q * 7) % 60 + 1} {((q * 2654435761) % 1000003) / 1000.0}\n")
    big = "".join(lines)
    for q in range(3):
        p = tmp_path / f"big{q}.dat-s"
        with open(p, "w", newline="") as f:
            f.write(big if q == 0 else mutate(rng, big, 3))
        files.append(str(p))
    r = subprocess.run([exe] + files, capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0"))
    assert r.returncode == 0, r.stderr[-3000:]
    assert "ERROR: AddressSanitizer" not in r.stderr and "runtime error" not in r.stderr, r.stderr[-3000:]
    ok, bad = (int(x) for x in r.stdout.split()[1::2])
    assert ok + bad == len(files) and ok >= 1
