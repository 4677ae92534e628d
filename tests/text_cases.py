"""Seeded text edge lists for the converter tests: plain lists (fileConvert -s), SNAP
files (-n) and Matrix Market files (-m) with the features their readers handle --
comment lines, one-based ids, weights written as integers, decimals and exponents
(negative too), CRLF line ends, a missing final newline, symmetric and general
matrices, pattern and complex fields, diagonal entries and repeated pairs.

CASES maps a name to (format, weight mode, one-based, builder); a builder returns the
file's bytes. Weight modes are 'abs' (default), 'orig' (-i), 'one' (-w), 'random' (-r).
"""
from __future__ import annotations

import numpy as np

FLAGS = {"simple": "-s", "snap": "-n", "mm": "-m"}
WFLAGS = {"abs": [], "orig": ["-i"], "one": ["-w"], "random": ["-r"]}


def _weight_text(rng, k: int) -> str:
    kind = k % 5
    if kind == 0:
        return str(int(rng.integers(-5, 20)))
    if kind == 1:
        return f"{rng.uniform(-1, 1):.6f}"
    if kind == 2:
        return f"{rng.uniform(0, 1e4):.3e}"
    if kind == 3:
        return f"{rng.uniform(0, 1):.17g}"   # 17 digits: converted on the host
    return f"{rng.uniform(0, 100):.2f}"


def simple_list(seed: int, n: int, m: int, one_based: bool = False, weights: bool = True,
                final_newline: bool = True, crlf: bool = False, comments: bool = True) -> bytes:
    rng = np.random.default_rng(seed)
    base = 1 if one_based else 0
    out = []
    if comments:
        out.append("# a plain edge list")
        out.append("% another comment")
    for k in range(m):
        u, v = int(rng.integers(0, n)), int(rng.integers(0, n))
        line = f"{u + base} {v + base}"
        if k % 7 == 3:
            line = f"{u + base}\t{v + base}"
        if weights:
            line += " " + _weight_text(rng, k)
        out.append(line)
        if comments and k == m // 2:
            out.append("# a comment in the middle")
    nl = "\r\n" if crlf else "\n"
    text = nl.join(out)
    if final_newline:
        text += nl
    return text.encode()


def snap_file(seed: int, n: int, m: int) -> bytes:
    rng = np.random.default_rng(seed)
    ids = rng.choice(10 * n, size=n, replace=False) + 1000  # arbitrary, non-contiguous
    lines = ["# Undirected graph: synthetic", f"# Nodes: {n} Edges: {m}", "# FromNodeId\tToNodeId"]
    for _ in range(m):
        u, v = ids[int(rng.integers(0, n))], ids[int(rng.integers(0, n))]
        lines.append(f"{u}\t{v}")
    return ("\n".join(lines) + "\n").encode()


def mm_file(seed: int, n: int, m: int, field: str = "real", symmetry: str = "symmetric") -> bytes:
    rng = np.random.default_rng(seed)
    lines = [f"%%MatrixMarket matrix coordinate {field} {symmetry}", "% generated", "%"]
    lines.append(f"{n} {n} {m}")
    for k in range(m):
        u, v = int(rng.integers(1, n + 1)), int(rng.integers(1, n + 1))
        if symmetry == "symmetric" and u < v:
            u, v = v, u  # lower triangle, diagonal included
        if field == "pattern":
            lines.append(f"{u} {v}")
        elif field == "integer":
            lines.append(f"{u} {v} {int(rng.integers(-9, 10))}")
        elif field == "complex":
            lines.append(f"{u} {v} {rng.uniform(-1, 1):.5f} {rng.uniform(-1, 1):.5f}")
        else:
            lines.append(f"{u} {v} {_weight_text(rng, k)}")
    return ("\n".join(lines) + "\n").encode()


CASES = {
    "simple_abs": ("simple", "abs", False, lambda: simple_list(1, 300, 2000)),
    "simple_orig": ("simple", "orig", False, lambda: simple_list(1, 300, 2000)),
    "simple_one": ("simple", "one", False, lambda: simple_list(2, 300, 2000)),
    "simple_random": ("simple", "random", False, lambda: simple_list(3, 300, 2000)),
    "simple_z_nonl": ("simple", "orig", True,
                      lambda: simple_list(4, 200, 900, one_based=True, final_newline=False)),
    "simple_crlf": ("simple", "abs", False, lambda: simple_list(5, 150, 700, crlf=True)),
    "simple_unweighted": ("simple", "one", False,
                          lambda: simple_list(6, 500, 3000, weights=False, comments=False)),
    "mm_sym_real": ("mm", "abs", False, lambda: mm_file(7, 250, 1500)),
    "mm_sym_orig": ("mm", "orig", False, lambda: mm_file(7, 250, 1500)),
    "mm_gen_int": ("mm", "abs", False, lambda: mm_file(8, 250, 1500, "integer", "general")),
    "mm_pattern": ("mm", "abs", False, lambda: mm_file(9, 250, 1500, "pattern")),
    "mm_complex": ("mm", "orig", False, lambda: mm_file(10, 100, 400, "complex", "general")),
    "mm_random": ("mm", "random", False, lambda: mm_file(11, 250, 1500)),
    "snap": ("snap", "one", False, lambda: snap_file(12, 400, 2500)),
    "snap_random": ("snap", "random", False, lambda: snap_file(13, 400, 2500)),
}


def write_case(name: str, path: str) -> tuple:
    """Writes case `name` to path; returns (format, weight mode, one-based)."""
    fmt, wmode, one_based, build = CASES[name]
    with open(path, "wb") as f:
        f.write(build())
    return fmt, wmode, one_based


def convert_flags(fmt: str, wmode: str, one_based: bool) -> list:
    return [FLAGS[fmt], *WFLAGS[wmode], *(["-z"] if one_based else [])]
