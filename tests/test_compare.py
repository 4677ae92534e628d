"""Ground-truth comparison (compare_communities, compare.cpp:58-318): the oracle's
restatement against what the reference's graphClustering -g prints (CPU), and the
device kernel and graphClustering -g against both (GPU)."""
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import vite_oracle as vo

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "vite_b200", "graphClustering")

STAT_LINES = {
    "nc1": r"#communities in C1 : (\d+)",
    "nc2": r"#communities in C2 : (\d+)",
    "same_same": r"Same-Same \(True positive\)  : (\d+)",
    "same_diff": r"Same-Diff \(False negative\) : (\d+)",
    "diff_same": r"Diff-Same \(False positive\) : (\d+)",
    "precision": r"Precision :  ([-\d.e+naif]+) \(",
    "recall": r"Recall    :  ([-\d.e+naif]+) \(",
    "fscore": r"F-score   :  ([-\d.e+naif]+)",
    "gini1": r"Gini coefficient, C1  :  ([-\d.e+naif]+)",
    "gini2": r"Gini coefficient, C2  :  ([-\d.e+naif]+)",
}


def parse_stats(stdout):
    out = {}
    for k, pat in STAT_LINES.items():
        m = re.search(pat, stdout)
        assert m, (k, stdout[-2000:])
        out[k] = int(m.group(1)) if k in ("nc1", "nc2", "same_same", "same_diff", "diff_same") \
            else float(m.group(1))
    return out


def printed(x):
    # std::cout's default: 6 significant digits
    return float(f"{x:g}")


def assert_matches_print(stats, ref):
    for k, v in ref.items():
        if isinstance(v, int):
            assert stats[k] == v, k
        else:
            assert printed(stats[k]) == v, (k, stats[k], v)


def write_truth(path, labels, zero_based=True):
    with open(path, "w") as f:
        for v, c in enumerate(labels):
            f.write(f"{v} {c + (0 if zero_based else 1)}\n")


def truth_labels(n, kind):
    rng = np.random.default_rng(5)
    if kind == "blocks":
        return np.arange(n) // 64
    if kind == "random":
        return rng.integers(0, 37, n)
    return np.zeros(n, np.int64)


@pytest.mark.skipif(not os.path.exists(vo.REF_MAIN), reason="reference build absent")
@pytest.mark.parametrize("kind", ["blocks", "random", "one"])
def test_oracle_matches_reference_print(tmp_path, kind):
    g = vo.rgg(4096).unit()
    gf = tmp_path / "g.bin"
    vo.write_vite_binary(str(gf), g)
    truth = truth_labels(g.nv, kind)
    tf = tmp_path / "truth.txt"
    write_truth(tf, truth, zero_based=False)
    r = subprocess.run([vo.REF_MAIN, "-f", str(gf), "-g", str(tf), "-z", "-o"], capture_output=True,
                       text=True, timeout=600, env={**os.environ, "OMP_NUM_THREADS": "1"})
    assert r.returncode == 0, r.stderr
    ref = parse_stats(r.stdout)
    found = np.loadtxt(str(gf) + ".communities", dtype=np.int64)
    st = vo.compare(truth, found)
    assert_matches_print(st, ref)
    assert st["same_same"] + st["same_diff"] == sum(c * (c - 1) // 2 for c in np.bincount(truth))


def test_oracle_compare_small_cases():
    st = vo.compare(np.array([0, 0, 1, 1, 2]), np.array([0, 0, 0, 1, 1]))
    assert (st["same_same"], st["same_diff"], st["diff_same"]) == (1, 1, 3)
    assert (st["precision"], st["recall"]) == (0.25, 0.5)
    same = vo.compare(np.array([3, 3, 1, 0]), np.array([3, 3, 1, 0]))
    assert same["fscore"] == 1.0 and same["nc1"] == 4  # the largest label + 1


@pytest.mark.gpu
@pytest.mark.parametrize("n,k1,k2", [(1, 1, 1), (1000, 10, 7), (100000, 1000, 50),
                                     (60000, 5, 60000), (20000, 1, 17)])
def test_device_compare_matches_oracle(ctx, n, k1, k2):
    rng = np.random.default_rng(n + k1)
    a = rng.integers(0, k1, n)
    b = rng.integers(0, k2, n)
    if n > 1:
        b[: n // 3] = a[: n // 3]  # some agreement
    dev = ctx.compare_communities(a, b)
    ref = vo.compare(a, b)
    for key in ("n", "nc1", "nc2", "same_same", "same_diff", "diff_same"):
        assert dev[key] == ref[key], key
    for key in ("precision", "recall", "fscore", "gini1", "gini2"):
        assert (np.isnan(dev[key]) and np.isnan(ref[key])) or dev[key] == ref[key], key


@pytest.mark.gpu
def test_device_compare_rejects_bad_labels(ctx):
    import vite_b200 as vb
    with pytest.raises(vb.VgError, match="community labels"):
        ctx.compare_communities(np.array([0, -1, 2]), np.array([0, 1, 2]))


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(vo.REF_MAIN), reason="reference build absent")
def test_cli_ground_truth_matches_reference(tmp_path):
    g = vo.rgg(4096).unit()  # unit weights: our communities equal the reference's bit for bit
    gf = tmp_path / "g.bin"
    vo.write_vite_binary(str(gf), g)
    tf = tmp_path / "truth.txt"
    write_truth(tf, truth_labels(g.nv, "random"))
    r = subprocess.run([CLI, "-f", str(gf), "-g", str(tf)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    rr = subprocess.run([vo.REF_MAIN, "-f", str(gf), "-g", str(tf)], capture_output=True,
                        text=True, timeout=600, env={**os.environ, "OMP_NUM_THREADS": "1"})
    assert rr.returncode == 0, rr.stderr
    assert parse_stats(r.stdout) == parse_stats(rr.stdout)
    assert "Loaded ground-truth file" in r.stdout
