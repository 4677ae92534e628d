"""graphClustering (vite_b200/graphClustering, host C++ over the C ABI) against Vite's CLI:
flag checks on the CPU; per-level results and the -o community file on the GPU."""
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import vite_oracle as vo

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "vite_b200", "graphClustering")


def run(binary, args, **kw):
    return subprocess.run([binary, *args], capture_output=True, text=True, timeout=600, **kw)


BAD_FLAGS = [
    (["-t", "7", "-n", "1024"], "early-term-type parameter is between 1-4"),
    (["-t", "2", "-a", "1.5", "-n", "1024"], "early-term-alpha must be between 0 and 1"),
    ([], "Must specify a binary file name with -f"),
    (["-c", "8", "-d", "8", "-n", "1024"], "Cannot turn on both coloring (-c) and vertex ordering (-d)"),
    (["-i", "-p", "-n", "1024"], "Cannot turn on threshold-cycling (-i) with a single phase run (-p)"),
    (["-f", "x.bin", "-e", "1"], "Must specify -n <...> for graph generation first"),
]


@pytest.mark.parametrize("args,msg", BAD_FLAGS)
def test_flag_checks_match_reference(args, msg):
    r = run(CLI, args)
    assert r.returncode == 157 and msg in r.stderr, (r.returncode, r.stderr)
    if os.path.exists(vo.REF_MAIN):  # the reference's own main gives the same answer
        rr = run(vo.REF_MAIN, args)
        assert rr.returncode == 157 and msg in (rr.stderr + rr.stdout)


def levels_from(stdout):
    return [(int(m.group(1)), float(m.group(2)), int(m.group(3)))
            for m in re.finditer(r"Level (\d+), Modularity: ([-\d.e+]+), Clustering time: [-\d.e+]+, "
                                 r"Iterations: (\d+)", stdout)]


@pytest.mark.gpu
def test_cli_generated_rgg_levels(golden):
    r = run(CLI, ["-n", "65536"])
    assert r.returncode == 0, r.stderr
    lv = levels_from(r.stdout)
    ref = golden["rgg64k"]["levels"]
    # main prints accepted levels only, with 6 significant digits and cumulative iterations
    assert len(lv) == len(ref) - 1
    tot = 0
    for (p, mod, it), g in zip(lv, ref):
        tot += g["iters"]
        assert p == g["level"] and it == tot
        assert float(f"{float.fromhex(g['mod']):g}") == mod


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [[], ["-c", "8", "-t", "2", "-a", "0.25"], ["-t", "3"], ["-d", "8"]])
def test_cli_file_input_and_output_match_reference(tmp_path, flags):
    g = vo.ba(4096, 4, 7)
    path = str(tmp_path / "ba.bin")
    vo.write_vite_binary(path, g)
    r = run(CLI, ["-f", path, "-o", *flags])
    assert r.returncode == 0, r.stderr
    ours = np.loadtxt(path + ".communities", dtype=np.int64)
    levels = levels_from(r.stdout)
    ref_levels, _ = vo.run_levels(g, **vo.flags_to_kwargs(flags))
    # graphClustering prints 6 significant digits (std::cout default precision)
    assert [m for _, m, _ in levels] == [float(f"{x.mod:g}") for x in ref_levels[:len(levels)]]
    if os.path.exists(vo.REF_MAIN):
        os.rename(path + ".communities", path + ".ours")
        rr = run(vo.REF_MAIN, ["-f", path, "-o", *flags], env=dict(os.environ, OMP_NUM_THREADS="1"))
        assert rr.returncode == 0
        theirs = np.loadtxt(path + ".communities", dtype=np.int64)
        np.testing.assert_array_equal(ours, theirs)
        assert levels == levels_from(rr.stdout)
