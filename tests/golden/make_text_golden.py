"""Golden outputs of the reference's own fileConvert (converters/convert.cpp, built
unmodified by oracle/Makefile into oracle/_ref/fileConvert) on the seeded text files of
tests/text_cases.py: for every case the converted graph's vertex and entry counts and
SHA-256 digests of its rowptr, tails and weights (equal (row, tail) entries, whose
order std::sort leaves unspecified, sorted by weight), or the fact that the reference
stopped (its SNAP reader fails an assertion in processGraphData on every file).

Needs the reference build (this container only):
    python tests/golden/make_text_golden.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))
from oracle import vite_oracle as vo  # noqa: E402
import text_cases as tc  # noqa: E402
from make_golden import graph_digest  # noqa: E402


def main() -> None:
    out = {"generator": "oracle/_ref/fileConvert (unmodified reference converters)", "cases": {}}
    with tempfile.TemporaryDirectory() as tmp:
        for name in tc.CASES:
            src = os.path.join(tmp, name + ".txt")
            dst = os.path.join(tmp, name + ".bin")
            fmt, wmode, one_based = tc.write_case(name, src)
            flags = tc.convert_flags(fmt, wmode, one_based)
            res = subprocess.run([vo.FILE_CONVERT, "-f", src, "-o", dst, *flags],
                                 capture_output=True, text=True)
            if res.returncode != 0:
                tailmsg = (res.stderr.strip().splitlines() or ["?"])[-1]
                if "Assertion" in tailmsg:  # keep the failed condition, not the build's paths
                    tailmsg = "Assertion" + tailmsg.split("Assertion", 1)[1]
                out["cases"][name] = {"flags": flags, "reference_failed": tailmsg[-200:]}
                continue
            g = vo.read_vite_binary(dst)
            # equal (row, tail) entries: std::sort leaves their order unspecified, so the
            # weight digest is taken over the runs sorted by weight bits
            g = vo.Graph(g.rowptr, g.tail, vo.canonical_ties(g))
            out["cases"][name] = {"flags": flags, **graph_digest(g)}
    with open(os.path.join(HERE, "text_golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
