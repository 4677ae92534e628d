"""fileConvert's text readers (converters/convert.cpp:102-281): the oracle's
restatement against the reference's own outputs (tests/golden/text_golden.json, made by
the unmodified converters), and the device readers (vg_graph_read_text) against the
restatement, bit for bit.
"""
import hashlib
import os
import subprocess

import numpy as np
import pytest

import text_cases as tc
from oracle import vite_oracle as vo

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = __import__("json").load(open(os.path.join(HERE, "golden", "text_golden.json")))["cases"]


def _digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _restate(name, tmp_path):
    path = str(tmp_path / (name + ".txt"))
    fmt, wmode, one_based = tc.write_case(name, path)
    return path, fmt, wmode, one_based, vo.read_text(path, fmt, wmode, one_based)


@pytest.mark.parametrize("name", sorted(tc.CASES))
def test_restatement_matches_reference_golden(name, tmp_path):
    _, fmt, _, _, g = _restate(name, tmp_path)
    gold = GOLDEN[name]
    if "reference_failed" in gold:
        # the reference's SNAP reader prepends 2 x numEdges default entries to its edge
        # list (snap.cpp:123-124) and processGraphData's assertion stops it
        assert fmt == "snap" and "Assertion" in gold["reference_failed"]
        assert g.ne == 2 * int(open(tmp_path / (name + ".txt")).read().split("Edges:")[1].split()[0])
        return
    assert (g.nv, g.ne) == (gold["nv"], gold["ne"])
    assert _digest(g.rowptr.astype("<i8")) == gold["rowptr"]
    assert _digest(g.tail.astype("<i8")) == gold["tail"]
    assert _digest(vo.canonical_ties(g).astype("<f8")) == gold["weight"]


@pytest.mark.skipif(not os.path.exists(vo.FILE_CONVERT), reason="reference build absent")
@pytest.mark.parametrize("name", ["simple_random", "mm_random"])
def test_random_weights_are_the_references(name, tmp_path):
    """-r: the reference's genRandom stream restated (minstd_rand0 + generate_canonical)."""
    path, fmt, wmode, one_based, g = _restate(name, tmp_path)
    out = str(tmp_path / "o.bin")
    subprocess.run([vo.FILE_CONVERT, "-f", path, "-o", out,
                    *tc.convert_flags(fmt, wmode, one_based)], check=True, capture_output=True)
    r = vo.read_vite_binary(out)
    np.testing.assert_array_equal(vo.canonical_ties(r).view(np.int64),
                                  vo.canonical_ties(g).view(np.int64))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(tc.CASES))
def test_device_reader_matches_restatement(ctx, name, tmp_path):
    path, fmt, wmode, one_based, g = _restate(name, tmp_path)
    d = ctx.read_text(path, fmt, wmode, one_based)
    rp, tail, w = d.download()
    assert d.nv == g.nv
    np.testing.assert_array_equal(rp, g.rowptr)
    np.testing.assert_array_equal(tail, g.tail)
    np.testing.assert_array_equal(w.view(np.int64), g.weight.view(np.int64))
    d.free()


@pytest.mark.gpu
def test_device_reader_large_list(ctx, tmp_path):
    """200,000 lines: many blocks, weights of every form, host conversions mixed in."""
    path = str(tmp_path / "big.txt")
    with open(path, "wb") as f:
        f.write(tc.simple_list(77, 50_000, 200_000))
    g = vo.read_text(path, "simple", "orig")
    d = ctx.read_text(path, "simple", "orig")
    rp, tail, w = d.download()
    np.testing.assert_array_equal(rp, g.rowptr)
    np.testing.assert_array_equal(tail, g.tail)
    np.testing.assert_array_equal(w.view(np.int64), g.weight.view(np.int64))
    d.free()


@pytest.mark.gpu
@pytest.mark.parametrize("text,fmt", [
    (b"0 1 1.0\nnot an edge\n2 3 1.0\n", "simple"),
    (b"0 -1 1.0\n", "simple"),
    (b"%%MatrixMarket matrix coordinate real general\n3 3 2\n1 2 1.0\n", "mm"),
    (b"%%MatrixMarket matrix coordinate real general\n3 3 1\n1 4 1.0\n", "mm"),
    (b"%%MatrixMarket matrix array real general\n3 3 1\n1 2 1.0\n", "mm"),
    (b"# Nodes: 2 Edges: 2\n5 6\n7 8\n", "snap"),
    (b"# no header\n5 6\n", "snap"),
    (b"# Nodes: 5 Edges: 2\n5 6\n7 x8\n", "snap"),
])
def test_device_reader_rejects_bad_files(ctx, tmp_path, text, fmt):
    import vite_b200

    path = str(tmp_path / "bad.txt")
    open(path, "wb").write(text)
    with pytest.raises(vite_b200.VgError) as ei:
        ctx.read_text(path, fmt)
    assert ei.value.status == vite_b200.VG_ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["simple_orig", "mm_sym_real", "simple_z_nonl"])
def test_file_convert_cli_writes_the_references_file(name, tmp_path):
    """vite_b200/fileConvert (the reference's flags) writes the file the reference's own
    fileConvert writes (equal (row, tail) entries compared as multisets)."""
    import vite_b200

    path = str(tmp_path / (name + ".txt"))
    fmt, wmode, one_based = tc.write_case(name, path)
    out = str(tmp_path / "ours.bin")
    cli = os.path.join(os.path.dirname(vite_b200.LIB_PATH), "fileConvert")
    subprocess.run([cli, "-f", path, "-o", out, *tc.convert_flags(fmt, wmode, one_based)],
                   check=True, capture_output=True)
    ours = vo.read_vite_binary(out)
    gold = GOLDEN[name]
    assert (ours.nv, ours.ne) == (gold["nv"], gold["ne"])
    assert _digest(ours.rowptr.astype("<i8")) == gold["rowptr"]
    assert _digest(ours.tail.astype("<i8")) == gold["tail"]
    assert _digest(vo.canonical_ties(ours).astype("<f8")) == gold["weight"]
