"""Vite's binary graph file read straight to the device (vg_graph_read_vite) and
written from it (vg_graph_write_vite), against the oracle's reader and writer of
the same format."""
import os

import numpy as np
import pytest

from oracle import vite_oracle as vo
import vite_b200 as vb

pytestmark = pytest.mark.gpu


def host_copy(g):
    rp, tl, w = g.download()
    return vo.Graph(rp, tl, w)


def test_round_trip_two_chunks(ctx, tmp_path):
    # about 5.2e6 edge records: more than one 64 MiB reader chunk
    g = ctx.generate_rgg(1 << 19, 1.0, 17)
    ref = host_copy(g)
    assert ref.ne > (64 << 20) // 16
    path = str(tmp_path / "g.bin")
    vo.write_vite_binary(path, ref)
    h = ctx.read_vite(path)
    got = host_copy(h)
    np.testing.assert_array_equal(got.rowptr, ref.rowptr)
    np.testing.assert_array_equal(got.tail, ref.tail)
    np.testing.assert_array_equal(got.weight.view(np.int64), ref.weight.view(np.int64))
    # and back out: byte for byte the oracle's file
    out = str(tmp_path / "h.bin")
    ctx.write_vite(h, out)
    assert open(out, "rb").read() == open(path, "rb").read()
    # the read graph runs like the generated one
    a, b = ctx.run(g), ctx.run(h)
    assert [s["nv"] for s in a.stats] == [s["nv"] for s in b.stats]
    g.free()
    h.free()


def test_write_from_locality_layout_is_reference_order(ctx, tmp_path):
    g = ctx.generate_rgg(1 << 18, 1.0, 5)
    ref = host_copy(g)
    ctx.reorder(g, 1)
    path = str(tmp_path / "g.bin")
    ctx.write_vite(g, path)
    got = vo.read_vite_binary(path)
    np.testing.assert_array_equal(got.rowptr, ref.rowptr)
    np.testing.assert_array_equal(got.tail, ref.tail)
    np.testing.assert_array_equal(got.weight, ref.weight)
    g.free()


def test_bad_files_are_rejected(ctx, tmp_path):
    ref = vo.rgg(4096)
    good = str(tmp_path / "good.bin")
    vo.write_vite_binary(good, ref)
    data = open(good, "rb").read()
    cases = {
        "missing": None,
        "truncated": data[:-8],
        "short_header": data[:8],
    }
    bad_tail = bytearray(data)
    off = 16 + 8 * (ref.nv + 1)
    bad_tail[off:off + 8] = np.int64(ref.nv).tobytes()  # first tail = nv
    cases["bad_tail"] = bytes(bad_tail)
    bad_rp = bytearray(data)
    bad_rp[16 + 8:16 + 16] = np.int64(10 ** 9).tobytes()  # rowptr[1] far too large
    cases["bad_offsets"] = bytes(bad_rp)
    for name, blob in cases.items():
        path = str(tmp_path / f"{name}.bin")
        if blob is not None:
            open(path, "wb").write(blob)
        with pytest.raises(vb.VgError):
            ctx.read_vite(path)
    # the context is still usable
    h = ctx.read_vite(good)
    assert (h.nv, h.ne) == (ref.nv, ref.ne)
    h.free()
