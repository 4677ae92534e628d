"""Generate the golden fixtures in this directory from the REFERENCE itself.

Runs the unmodified reference (compiled by oracle/Makefile into oracle/_ref,
driven by oracle/ref_harness.cpp, one OpenMP thread so every floating-point sum
has one order) on small seeded graphs, and records what it returns: every
level's vertex/edge counts, iteration count, modularity (exact bits), a SHA-256
of the level's community vector, the colors, and the CSR of each level. Small
cases also keep the full arrays in an .npz.

Needs the reference sources (this container only):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import vite_oracle as vo  # noqa: E402


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def graph_digest(g: vo.Graph) -> dict:
    return {"nv": int(g.nv), "ne": int(g.ne),
            "rowptr": digest(g.rowptr.astype("<i8")), "tail": digest(g.tail.astype("<i8")),
            "weight": digest(g.weight.astype("<f8"))}


# name -> (graph source, harness flags, keep full arrays)
CASES = {
    "rgg4k": ("gen:4096", [], True),
    "rgg4k_unit": ("file:rgg4k:unit", [], True),
    "rgg64k": ("gen:65536", [], False),
    "rgg64k_unit": ("file:rgg64k:unit", [], False),
    "rgg4k_c8_t2": ("file:rgg4k", ["-c", "8", "-t", "2", "-a", "0.25"], True),
    "rgg4k_unit_c8": ("file:rgg4k:unit", ["-c", "8"], True),
    "rgg4k_unit_i": ("file:rgg4k:unit", ["-i"], True),
    "ba4k_c8_t2": ("ba:4096:4:7", ["-c", "8", "-t", "2", "-a", "0.25"], True),
    "ba4k_t1": ("ba:4096:4:7", ["-t", "1"], True),
    "ba4k_t3": ("ba:4096:4:7", ["-t", "3"], True),
    "ba4k_t4": ("ba:4096:4:7", ["-t", "4", "-a", "0.5"], True),
    "ba4k_d8": ("ba:4096:4:7", ["-d", "8"], True),
    "ba4k_c8_single": ("ba:4096:4:7", ["-c", "8 true"], True),
    "ba4k_p": ("ba:4096:4:7", ["-p"], True),
    "er4k": ("er:4096:16:3", [], True),
    "rgg16k_extra": ("rggx:16384:1.0:42", [], False),
}


def make_graph(src: str, tmp: str, made: dict) -> tuple[str, vo.Graph | None]:
    kind, *rest = src.split(":")
    if kind == "gen":
        return "", None
    if kind == "file":
        base = made[rest[0]]
        g = vo.read_vite_binary(base)
        if len(rest) > 1 and rest[1] == "unit":
            g = g.unit()
    elif kind == "ba":
        g = vo.ba(int(rest[0]), int(rest[1]), int(rest[2]))
    elif kind == "er":
        g = vo.er(int(rest[0]), float(rest[1]), int(rest[2]))
    elif kind == "rggx":
        g, _ = vo.add_random_edges(vo.rgg(int(rest[0])), float(rest[1]), int(rest[2]))
    else:
        raise ValueError(src)
    path = os.path.join(tmp, f"g{len(made)}_{kind}.bin")
    vo.write_vite_binary(path, g)
    return path, g


def main() -> None:
    if not os.path.exists(vo.HARNESS):
        vo.build(quiet=False)
    index = {}
    with tempfile.TemporaryDirectory() as tmp:
        made: dict[str, str] = {}
        for name, (src, flags, keep) in CASES.items():
            rec_path = os.path.join(tmp, name + ".rec")
            if src.startswith("gen:"):
                n = int(src.split(":")[1])
                saved = os.path.join(tmp, name + ".bin")
                vo.run_harness(["-n", str(n), "-s", saved, "-G", *flags], rec_path)
                made[name] = saved
                graph_src = {"kind": "reference_rgg", "n": n}
            else:
                path, _ = make_graph(src, tmp, made)
                vo.run_harness(["-f", path, "-G", *flags], rec_path)
                graph_src = {"kind": "spec", "spec": src}
            rec = vo.read_record(rec_path)
            levels = []
            for lv in rec.levels:
                levels.append({"level": lv.level, "nv": lv.nv, "ne": lv.ne, "iters": lv.iters,
                               "mod": float(lv.mod).hex(), "num_colors": lv.num_colors,
                               "cvect": digest(lv.cvect.astype("<i8"))})
            graphs = {str(k): graph_digest(g) for k, g in rec.graphs.items()}
            entry = {"source": graph_src, "flags": flags, "levels": levels, "graphs": graphs}
            if rec.colors is not None:
                entry["colors"] = digest(rec.colors.astype("<i8"))
            if keep:
                arrays = {}
                g0 = rec.graphs[0]
                arrays["rowptr"], arrays["tail"], arrays["weight"] = g0.rowptr, g0.tail, g0.weight
                for i, lv in enumerate(rec.levels):
                    arrays[f"cvect{i}"] = lv.cvect
                for k, g in rec.graphs.items():
                    if k == 0:
                        continue
                    arrays[f"g{k}_rowptr"], arrays[f"g{k}_tail"], arrays[f"g{k}_weight"] = (
                        g.rowptr, g.tail, g.weight)
                if rec.colors is not None:
                    arrays["colors"] = rec.colors
                np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
                entry["arrays"] = name + ".npz"
            index[name] = entry
            print(name, [(lv["nv"], lv["iters"], float.fromhex(lv["mod"])) for lv in levels][:3])
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump({"generator": "oracle/_ref/vite_ref_harness, OMP_NUM_THREADS=1",
                   "cases": index}, f, indent=1)


if __name__ == "__main__":
    main()
