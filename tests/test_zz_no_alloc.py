"""The allocation-free match entry point, for callers that cannot call
cudaMalloc where they index patterns (an acquisition callback that must never
block, or a host application that owns all device memory). It must give the
same top-k as the regular entry points with caller-allocated scratch, on
consecutive calls that reuse its fixed device scratch array.

Kept in its own file, named to be collected after every other test file."""

import numpy as np
import pytest
import torch

from oracle import di_oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _rows(n, n_pad, k_pad, p, seed, like=None, noise=0.0):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn((n, p), generator=g, dtype=torch.float64)
    if like is not None:
        x = like[torch.randint(0, like.shape[0], (n,), generator=g)] + noise * x
    x = x - x.mean(dim=1, keepdim=True)
    norm = x.norm(dim=1)
    out = torch.zeros((n_pad, k_pad), dtype=torch.bfloat16)
    out[:n, :p] = (x / norm[:, None]).to(torch.bfloat16)
    return x, out.to(DEV), norm.float().to(DEV)


def _existing_path(lib, q_lp, nq, d_lp, nd, col_scale, k):
    from ebsdtorch_b200 import _capi

    n_cand = 1 << (k - 1).bit_length()
    splits = int(lib.ebsd_match_auto_splits(q_lp.shape[0], d_lp.shape[0]))
    part_val = torch.empty((q_lp.shape[0], splits, n_cand), dtype=torch.float32, device=DEV)
    part_idx = torch.empty((q_lp.shape[0], splits, n_cand), dtype=torch.int32, device=DEV)
    status = torch.zeros(1, dtype=torch.int32, device=DEV)
    s = torch.cuda.current_stream().cuda_stream
    _capi.call("ebsd_match_topk", q_lp.data_ptr(), q_lp.shape[0], d_lp.data_ptr(), d_lp.shape[0], nd,
               q_lp.shape[1], _capi.DT_BF16, col_scale.data_ptr(), n_cand, splits, part_val.data_ptr(),
               part_idx.data_ptr(), splits, 0, 0, status.data_ptr(), s)
    val = torch.empty((nq, k), dtype=torch.float32, device=DEV)
    idx = torch.empty((nq, k), dtype=torch.int64, device=DEV)
    _capi.call("ebsd_merge_rescore", part_val.data_ptr(), part_idx.data_ptr(), nq, splits, n_cand, None, 0, None, 0,
               0, 1, 0, None, None, None, _capi.SIM_DOT, min(n_cand * splits, 128), k, None, None, val.data_ptr(),
               idx.data_ptr(), s)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return idx.cpu().numpy(), val.cpu().numpy()


def _case(nq, nd, p, seed):
    nq_pad, nd_pad, k_pad = -(-nq // 128) * 128, -(-nd // 256) * 256, -(-p // 64) * 64
    d64, d_lp, d_norm = _rows(nd, nd_pad, k_pad, p, seed)
    _, q_lp, _ = _rows(nq, nq_pad, k_pad, p, seed + 1, like=d64, noise=0.5)
    col_scale = torch.zeros(nd_pad, dtype=torch.float32, device=DEV)
    col_scale[:nd] = d_norm
    return dict(nq=nq, nd=nd, nq_pad=nq_pad, nd_pad=nd_pad, k_pad=k_pad, q_lp=q_lp, d_lp=d_lp, col_scale=col_scale)


def _noalloc(lib, c, k):
    from ebsdtorch_b200 import _capi

    val = torch.full((c["nq"], k), float("nan"), dtype=torch.float32, device=DEV)
    idx = torch.full((c["nq"], k), -7, dtype=torch.int64, device=DEV)
    st = torch.full((1,), 123, dtype=torch.int32, device=DEV)
    rc = lib.ebsd_match_topk_noalloc(c["q_lp"].data_ptr(), c["nq"], c["nq_pad"], c["d_lp"].data_ptr(), c["nd_pad"],
                                     c["nd"], c["k_pad"], _capi.DT_BF16, c["col_scale"].data_ptr(), None, k,
                                     val.data_ptr(), idx.data_ptr(), st.data_ptr(),
                                     torch.cuda.current_stream().cuda_stream)
    assert rc == 0, _capi.last_error()
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return idx.cpu().numpy(), val.cpu().numpy()


def _check(got, ref):
    (gi, gv), (ri, rv) = got, ref
    assert (gi == ri).mean() >= 0.999
    assert np.abs(gv - rv).max() <= 1e-5 * np.abs(rv).max()


@pytest.mark.parametrize("nq,nd,p,k", [(1000, 5000, 300, 8), (77, 700, 64, 1)])
def test_noalloc_matches_existing_entry_points(nq, nd, p, k):
    from ebsdtorch_b200 import _capi

    lib = _capi.load()
    c = _case(nq, nd, p, 1)
    ref = _existing_path(lib, c["q_lp"], nq, c["d_lp"], nd, c["col_scale"], k)
    for _ in range(2):  # two calls in a row share the fixed scratch
        _check(_noalloc(lib, c, k), ref)
    # and both agree with the oracle's exact top-k of the same bf16 rows
    q = c["q_lp"][:nq].double().cpu().numpy()
    d = (c["d_lp"][:nd].double() * c["col_scale"][:nd, None].double()).cpu().numpy()
    oi, ov = O.topk_dot(q, d, k)
    gi, gv = ref
    assert (gi[:, 0] == oi[:, 0]).mean() >= 0.999
    assert np.abs(gv - ov).max() <= 1e-5 * np.abs(ov).max()


def test_noalloc_ignores_leftovers_of_larger_calls():
    """Calls of different shapes on one stream: a large one (many padded
    queries, a larger k, more candidate lists), a small one, the large one
    again. Each must match the regular entry points on its own inputs, so
    nothing a larger earlier call left in the shared scratch leaks into a
    smaller later one."""
    from ebsdtorch_b200 import _capi

    lib = _capi.load()
    big, small = _case(3000, 9000, 200, 11), _case(40, 600, 64, 21)
    ref_big = _existing_path(lib, big["q_lp"], big["nq"], big["d_lp"], big["nd"], big["col_scale"], 32)
    ref_small = _existing_path(lib, small["q_lp"], small["nq"], small["d_lp"], small["nd"], small["col_scale"], 3)
    _check(_noalloc(lib, big, 32), ref_big)
    _check(_noalloc(lib, small, 3), ref_small)
    _check(_noalloc(lib, big, 32), ref_big)
    _check(_noalloc(lib, small, 3), ref_small)


def test_noalloc_rejects_oversized_calls():
    from ebsdtorch_b200 import _capi

    lib = _capi.load()
    q = torch.zeros((128, 64), dtype=torch.bfloat16, device=DEV)
    d = torch.zeros((256, 64), dtype=torch.bfloat16, device=DEV)
    out_v = torch.empty((128, 64), dtype=torch.float32, device=DEV)
    out_i = torch.empty((128, 64), dtype=torch.int64, device=DEV)
    too_many = 1 << 20  # padded queries: 2^20 x 64 candidates x 8 B = 512 MiB > 32 MiB
    rc = lib.ebsd_match_topk_noalloc(q.data_ptr(), 128, too_many, d.data_ptr(), 256, 256, 64, _capi.DT_BF16,
                                     None, None, 64, out_v.data_ptr(), out_i.data_ptr(), None,
                                     torch.cuda.current_stream().cuda_stream)
    assert rc == 1
    assert "scratch" in _capi.last_error()
