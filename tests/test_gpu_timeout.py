"""Bounded device waits: a match whose waits run out reports
EBSD_DEVICE_TIMEOUT in its status word and returns, and the context stays
usable for the next call.

The wait limit is set to 1 ns (ebsd_set_wait_limit_ns), so the first wait of
any role that is not satisfied within its short spin gives up. Nothing faults
or hangs: the kernel lets the copies and MMAs it issued complete (under the
default 4 s limit) before it releases TMEM and exits."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _match(lib, q, d, col_scale, k, status):
    from ebsdtorch_b200 import _capi

    n_cand = 1 << (k - 1).bit_length()
    splits = int(lib.ebsd_match_auto_splits(q.shape[0], d.shape[0]))
    pv = torch.empty((q.shape[0], splits, n_cand), dtype=torch.float32, device=DEV)
    pi = torch.empty((q.shape[0], splits, n_cand), dtype=torch.int32, device=DEV)
    _capi.call("ebsd_match_topk", q.data_ptr(), q.shape[0], d.data_ptr(), d.shape[0], d.shape[0], q.shape[1],
               _capi.DT_BF16, col_scale.data_ptr(), n_cand, splits, pv.data_ptr(), pi.data_ptr(), splits, 0, 0,
               status.data_ptr(), torch.cuda.current_stream().cuda_stream)
    val = torch.empty((q.shape[0], k), dtype=torch.float32, device=DEV)
    idx = torch.empty((q.shape[0], k), dtype=torch.int64, device=DEV)
    _capi.call("ebsd_merge_rescore", pv.data_ptr(), pi.data_ptr(), q.shape[0], splits, n_cand, None, 0, None, 0, 0,
               1, 0, None, None, None, _capi.SIM_DOT, min(n_cand * splits, 128), k, None, None, val.data_ptr(),
               idx.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return idx, val


@pytest.mark.parametrize("variant", ["one_tile", "pairs", "dual"])
def test_wait_limit_runs_out_and_the_next_call_succeeds(variant):
    """For each match kernel: the one-tile kernel, CTA pairs (whose even CTA
    drains both CTAs' copies before the cluster barrier) and two query tiles
    per CTA."""
    from ebsdtorch_b200 import _capi, kernels

    lib = _capi.load()
    prev_modes = (kernels.set_match_pairs(variant == "pairs"), kernels.set_match_dual(variant == "dual"))
    try:
        _run_timeout_case(lib)
    finally:
        kernels.set_match_pairs(prev_modes[0])
        kernels.set_match_dual(prev_modes[1])


def _run_timeout_case(lib):
    from ebsdtorch_b200 import _capi

    g = torch.Generator(device=DEV).manual_seed(3)
    # 256 queries x 16,384 rows of 16,384 bf16 values: every accumulator
    # takes far longer than a wait's spin, so a 1 ns limit always runs out
    q = torch.randn((256, 16384), device=DEV, generator=g).bfloat16()
    d = torch.randn((16384, 16384), device=DEV, generator=g).bfloat16()
    col_scale = torch.ones(16384, dtype=torch.float32, device=DEV)
    status = torch.zeros(1, dtype=torch.int32, device=DEV)
    prev = lib.ebsd_set_wait_limit_ns(1)
    try:
        _match(lib, q, d, col_scale, 4, status)
        torch.cuda.synchronize()  # the kernel returned
    finally:
        assert lib.ebsd_set_wait_limit_ns(prev) == 1
    assert int(status.item()) == _capi.DEVICE_TIMEOUT
    # the context is usable: the same match under the default limit succeeds
    # and agrees with an FP32 product of the same bf16 values
    status.zero_()
    idx, val = _match(lib, q, d, col_scale, 4, status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    ref_v, ref_i = torch.topk(q.float() @ d.float().t(), 4, dim=1)
    assert (idx[:, 0] == ref_i[:, 0]).float().mean().item() >= 0.99
    assert np.abs((val - ref_v).cpu().numpy()).max() <= 1e-3 * float(ref_v.abs().max())
