"""The allocation-free degree entry point (vg_vertex_degree_noalloc) against the
allocating one (vg_vertex_degree), through the C ABI, on two calls in a row.

This path serves callers that cannot allocate device memory while they run (a server
that reserved its memory up front, a framework whose allocator owns the GPU). The
file sorts last so that a run stopping at the first failure has run every other test.
"""
import numpy as np
import pytest

import vite_b200
from oracle import vite_oracle as vo


def test_rejects_sizes_beyond_the_maximum():
    # rejected before any GPU work
    with pytest.raises(vite_b200.VgError) as ei:
        vite_b200.vertex_degree_noalloc(vite_b200.NOALLOC_MAX_VERTICES + 1, 1, 1, 1)
    assert ei.value.status == vite_b200.VG_ERR_ARG
    assert "maximum" in str(ei.value)


@pytest.mark.gpu
@pytest.mark.parametrize("maker", ["rgg_distance", "ba_unit", "ba_real"])
def test_noalloc_matches_vg_vertex_degree(maker):
    """ba_*: hub rows of hundreds to thousands of entries, which the warp folds
    together; with real weights their sums must keep the serial CSR order"""
    import torch

    if maker == "rgg_distance":
        g = vo.rgg(65536)
    elif maker == "ba_unit":
        g = vo.ba(20000, 8, 3)
    else:
        g = vo.reweight(vo.ba(20000, 8, 3), 2, 7)
    with vite_b200.Context(0) as ctx:
        vd_ref, c_ref = ctx.vertex_degree(ctx.upload(g.rowptr, g.tail, g.weight))
    rp = torch.tensor(g.rowptr, dtype=torch.int64, device="cuda")
    w = torch.tensor(g.weight, dtype=torch.float64, device="cuda")
    for k in range(2):  # two calls in a row share the static scratch
        out = torch.full((g.nv,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        c = vite_b200.vertex_degree_noalloc(g.nv, rp.data_ptr(), w.data_ptr(), out.data_ptr(),
                                            torch.cuda.current_stream().cuda_stream)
        if k == 1:  # after the first call has loaded the kernels: no device memory taken
            assert torch.cuda.mem_get_info()[0] == free_before
        vd = out.cpu().numpy()
        # degrees: the same CSR-order row sums, bit for bit
        np.testing.assert_array_equal(vd.view(np.int64), vd_ref.view(np.int64))
        # 1/(2m): the same sum in another reduction order (exact on unit weights)
        if maker == "ba_unit":
            assert c == c_ref
        else:
            assert abs(c - c_ref) <= 1e-12 * abs(c_ref)


@pytest.mark.gpu
def test_null_weights_only_without_entries():
    import torch

    # a CSR without entries: NULL weights are accepted, every degree is zero and
    # 1/(2m) is what vg_vertex_degree gives for the same graph
    nv = 5
    rowptr = np.zeros(nv + 1, np.int64)
    with vite_b200.Context(0) as ctx:
        vd_ref, c_ref = ctx.vertex_degree(ctx.upload(rowptr, np.zeros(0, np.int64), np.zeros(0)))
    rp = torch.tensor(rowptr, device="cuda")
    out = torch.full((nv,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    c = vite_b200.vertex_degree_noalloc(nv, rp.data_ptr(), 0, out.data_ptr(), stream)
    np.testing.assert_array_equal(out.cpu().numpy(), vd_ref)
    assert c == c_ref
    # a CSR with entries and NULL weights: rejected before any kernel runs
    g = vo.rgg(4096)
    rp = torch.tensor(g.rowptr, dtype=torch.int64, device="cuda")
    out = torch.full((g.nv,), float("nan"), dtype=torch.float64, device="cuda")
    with pytest.raises(vite_b200.VgError) as ei:
        vite_b200.vertex_degree_noalloc(g.nv, rp.data_ptr(), 0, out.data_ptr(), stream)
    assert ei.value.status == vite_b200.VG_ERR_ARG
    assert "NULL" in str(ei.value)
    assert torch.isnan(out).all().item()
