"""Kernel-level parity of the CUDA path (through the C-ABI) against the CPU
oracle and the reference's golden vectors."""

import math

import numpy as np
import pytest
import torch

from oracle import di_oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _sign_invariant_maxdiff(a, b):
    return float(np.minimum(np.abs(a - b).max(-1), np.abs(a + b).max(-1)).max())


# ------------------------------------------------------------------ A1/A2


@pytest.mark.parametrize("laue", range(1, 12))
@pytest.mark.parametrize("res", [15.0, 7.5])
def test_grid_matches_reference_golden(golden, laue, res):
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.s2_and_so3.laue_fz_ori import edge_length_for_resolution

    ref = golden("grid")[f"q_{laue}_{res}"]
    q32, q64 = kernels.grid_fz(laue, edge_length_for_resolution(laue, res), DEV, want_f64=True)
    assert q32.shape[0] == ref.shape[0]
    assert _sign_invariant_maxdiff(q32.cpu().numpy(), ref) < 2e-6
    ora = O.sample_ori_fz_laue_angle(laue, res)
    assert np.abs(q64.cpu().numpy() - ora).max() < 1e-12


def test_grid_config_counts(golden):
    """Dictionary sizes of the benchmark configurations equal the reference's."""
    from ebsdtorch_b200.s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle

    for laue, res, n in golden("grid")["counts"]:
        q = sample_ori_fz_laue_angle(int(laue), float(res), DEV, permute=False)
        assert q.shape[0] == int(n), (laue, res)


def test_grid_large_matches_reference_order(golden):
    from ebsdtorch_b200.s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle

    ref = golden("grid")["q_11_1.0"]
    q = sample_ori_fz_laue_angle(11, 1.0, DEV, permute=False).cpu().numpy()
    assert q.shape == ref.shape
    assert np.abs(q - ref).max() < 2e-6


def test_permutation_convention_matches_reference(golden):
    from ebsdtorch_b200.s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle

    torch.manual_seed(1234)
    q = sample_ori_fz_laue_angle(11, 7.5, DEV, permute=True).cpu().numpy()
    assert np.abs(q - golden("grid")["q_11_7.5_perm_seed1234"]).max() < 2e-6


def test_gather_rows_bounds():
    from ebsdtorch_b200 import kernels

    src = torch.arange(12, dtype=torch.float32, device=DEV).view(3, 4)
    out = kernels.gather_rows(src, torch.tensor([2, 0, 5, -1], device=DEV))
    assert torch.equal(out[0].cpu(), src[2].cpu()) and torch.equal(out[1].cpu(), src[0].cpu())
    assert torch.isnan(out[2:]).all()


# ------------------------------------------------------------------ A3-A7


@pytest.mark.parametrize("b", [1, 2])
def test_projector_matches_reference_golden(golden, b):
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.kernels import RowBuffers

    g = golden("projector")
    mp = torch.from_numpy(g["master_pattern"]).to(DEV)
    if b > 1:
        mp = kernels.avg_pool(mp, b)
    rays = torch.from_numpy(g[f"rays_b{b}"]).t().contiguous().to(DEV)
    quats = torch.from_numpy(g["quats"]).contiguous().to(DEV)
    out = torch.empty((quats.shape[0], rays.shape[1]), dtype=torch.float32, device=DEV)
    kernels.project(mp, rays, quats, RowBuffers(f32=out), subtract_mean=False)
    assert np.abs(out.cpu().numpy() - g[f"sims_b{b}"]).max() < 5e-5


def test_avg_pool_matches_torch():
    from ebsdtorch_b200 import kernels

    x = torch.randn(5, 12, 18, device=DEV)
    for b in (1, 2, 3):
        ref = torch.nn.functional.avg_pool2d(x.unsqueeze(1), b).squeeze(1)
        assert torch.allclose(kernels.avg_pool(x, b), ref, atol=1e-6)


def test_master_pattern_interpolate(golden):
    from ebsdtorch_b200.ebsd.master_pattern import MasterPattern

    g = golden("projector")
    mp = MasterPattern(torch.from_numpy(g["master_pattern"]), laue_group=11).to(DEV)
    rays = torch.from_numpy(g["rays_b1"]).to(DEV)
    q = torch.from_numpy(g["quats"]).to(DEV)
    rot = torch.from_numpy(O.qu_apply(g["quats"][:, None, :].astype(np.float64),
                                      g["rays_b1"][None].astype(np.float64))).float().to(DEV)
    vals = mp.interpolate(rot, normalize_coords=False)
    assert vals.shape == (q.shape[0], rays.shape[0])
    assert np.abs(vals.cpu().numpy() - g["sims_b1"]).max() < 5e-5


@pytest.mark.parametrize("lp", ["bf16", "fp8"])
def test_projector_row_outputs(lp):
    """Zero-mean FP32 rows, norms and the unit low-precision copy."""
    from ebsdtorch_b200 import kernels, synthetic
    from ebsdtorch_b200.kernels import LP_DTYPES, LP_TORCH, RowBuffers, round_up

    mp = synthetic.synthetic_master_pattern(65, seed=3).to(DEV)
    rng = np.random.default_rng(0)
    rays64 = rng.standard_normal((300, 3))
    rays64 /= np.linalg.norm(rays64, axis=1, keepdims=True)
    rays = torch.from_numpy(rays64.T.copy()).float().to(DEV)
    quats = synthetic.random_quaternions(37, 5).to(DEV)
    dt = LP_DTYPES[lp]
    kp = round_up(300, 64 if lp == "bf16" else 128)
    f32 = torch.empty((37, 300), device=DEV)
    low = torch.full((37, kp), 7, dtype=LP_TORCH[dt], device=DEV) if lp == "bf16" else \
        torch.zeros((37, kp), dtype=LP_TORCH[dt], device=DEV)
    norm = torch.empty(37, device=DEV)
    scale = torch.empty(37, device=DEV)
    kernels.project(mp, rays, quats, RowBuffers(f32=f32, lp=low, lp_dtype=dt, norm=norm, lp_scale=scale))
    ref = O.dictionary_rows(mp.cpu().numpy(), rays64, quats.cpu().numpy().astype(np.float64))
    assert np.abs(f32.cpu().numpy() - ref).max() < 5e-5
    assert np.allclose(norm.cpu().numpy(), np.linalg.norm(ref, axis=1), rtol=1e-5)
    unit = low.float()[:, :300] * (scale[:, None] if lp == "fp8" else 1.0)
    tol = 2 ** -8 if lp == "bf16" else 2 ** -3
    exp = ref / np.linalg.norm(ref, axis=1, keepdims=True)
    assert np.abs(unit.cpu().numpy() - exp).max() <= tol * np.abs(exp).max()
    assert torch.all(low.float()[:, 300:] == 0)


@pytest.mark.parametrize("b,masked", [(1, False), (2, True), (3, False)])
def test_prep_patterns_matches_oracle(b, masked):
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.kernels import RowBuffers
    from ebsdtorch_b200.preprocessing.radial_mask import get_radial_mask

    H, W = 24, 30
    x = torch.rand(11, H, W) * 100
    mask = get_radial_mask((H // b, W // b)) if masked else None
    pix = torch.nonzero(mask.reshape(-1)).reshape(-1).int().to(DEV) if masked else None
    n_pix = int(mask.sum()) if masked else (H // b) * (W // b)
    out = torch.empty((11, n_pix), device=DEV)
    norm = torch.empty(11, device=DEV)
    kernels.prep_patterns(x.to(DEV), RowBuffers(f32=out, norm=norm), b, pix, n_pix, True)
    ref = O.prep_patterns(x.numpy(), b, mask.numpy() if masked else None, True)
    assert np.abs(out.cpu().numpy() - ref).max() < 1e-4
    assert np.allclose(norm.cpu().numpy(), np.linalg.norm(ref, axis=1), rtol=1e-5)


# ------------------------------------------------------------------ A9/A10


def _rows(n, p, seed, corr=None):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, p))
    if corr is not None:
        x = x @ corr
    return x - x.mean(axis=1, keepdims=True)


@pytest.mark.parametrize("lp,nq,nd,p,k", [
    ("bf16", 300, 1000, 200, 1),
    ("bf16", 128, 256, 64, 8),
    ("bf16", 517, 3001, 333, 5),
    ("fp8", 260, 2000, 250, 3),
])
def test_match_and_rescore_match_oracle(lp, nq, nd, p, k):
    """Tensor-core candidates + FP32 re-score reproduce the exact top-k."""
    from ebsdtorch_b200.engine import Searcher, SearchConfig

    rng = np.random.default_rng(1)
    mix = np.eye(p) + 0.3 * rng.standard_normal((p, p)) / math.sqrt(p)
    d = _rows(nd, p, 2, mix)
    q = d[rng.integers(0, nd, nq)] + 0.3 * _rows(nq, p, 3)
    q = q - q.mean(axis=1, keepdims=True)
    dt, qt = torch.from_numpy(d).float().to(DEV), torch.from_numpy(q).float().to(DEV)
    from ebsdtorch_b200 import kernels

    def fill_d(d0, d1, bufs):
        kernels.prep_patterns(dt[d0:d1].reshape(d1 - d0, 1, p), bufs, subtract_mean=False)

    def fill_q(q0, q1, bufs):
        kernels.prep_patterns(qt[q0:q1].reshape(q1 - q0, 1, p), bufs, subtract_mean=False)

    s = Searcher(nd, nq, p, k, SearchConfig(precision=lp, rescore_k=32), DEV)
    idx, val = s.run(fill_d, fill_q)
    ref_i, ref_v = O.topk_dot(q.astype(np.float32).astype(np.float64), d.astype(np.float32).astype(np.float64), k)
    idx, val = idx.cpu().numpy(), val.cpu().numpy()
    agree = (idx == ref_i).mean()
    assert agree >= 0.999, agree
    assert np.abs(val - ref_v).max() <= 1e-5 * np.abs(ref_v).max()


@pytest.mark.parametrize("lp,shape", [
    ("bf16", dict(persistent=True, splits=4)),
    ("bf16", dict(persistent=True, splits=2, tile_n=128)),
    ("bf16", dict(tile_n=128)),
    ("bf16", dict(wave_tiles=2, splits=3)),
    ("fp8", dict(persistent=True, splits=8)),
    ("fp8", dict(tile_n=128, splits=5)),
])
def test_match_launch_shapes_give_identical_results(lp, shape):
    """Every launch shape the batch autotuner may pick (128- or 256-row tiles,
    persistent or one-wave launches, any number of dictionary ranges) returns
    exactly the default shape's top-k."""
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.engine import Searcher, SearchConfig

    p, nd, nq, k = 320, 5000, 2300, 6
    d = _rows(nd, p, 11)
    q = d[np.arange(nq) * 2] + 0.4 * _rows(nq, p, 12)
    dt, qt = torch.from_numpy(d).float().to(DEV), torch.from_numpy(q).float().to(DEV)

    def fill_d(d0, d1, bufs):
        kernels.prep_patterns(dt[d0:d1].reshape(d1 - d0, 1, p), bufs, subtract_mean=False)

    def fill_q(q0, q1, bufs):
        kernels.prep_patterns(qt[q0:q1].reshape(q1 - q0, 1, p), bufs, subtract_mean=False)

    base_i, base_v = Searcher(nd, nq, p, k, SearchConfig(precision=lp), DEV).run(fill_d, fill_q)
    i2, v2 = Searcher(nd, nq, p, k, SearchConfig(precision=lp, **shape), DEV).run(fill_d, fill_q)
    assert torch.equal(base_i, i2)
    assert torch.equal(base_v, v2)


@pytest.mark.parametrize("variant", ["pairs", "dual"])
@pytest.mark.parametrize("lp,shape,rescore_k", [
    ("bf16", {}, 0),
    ("bf16", {}, 32),
    ("fp8", {}, 0),
    ("bf16", dict(wave_tiles=4, splits=3), 32),
    ("bf16", dict(wave_tiles=3), 0),
    ("fp8", dict(wave_tiles=6, splits=5), 32),
])
def test_match_pairs_give_identical_results(lp, shape, rescore_k, variant):
    """CTA-pair launches (two query tiles per tcgen05.mma.cta_group::2, half
    of each dictionary tile staged per CTA) and two-tile launches (two MMAs
    per K step sharing one staged dictionary tile) return exactly the
    one-tile kernel's top-k, raw low-precision scores included; launches with
    an odd number of query tiles (wave_tiles=3) fall back to the one-tile
    kernel."""
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.engine import Searcher, SearchConfig

    p, nd, nq, k = 320, 5000, 2300, 6
    d = _rows(nd, p, 21)
    q = d[np.arange(nq) * 2] + 0.4 * _rows(nq, p, 22)
    dt, qt = torch.from_numpy(d).float().to(DEV), torch.from_numpy(q).float().to(DEV)

    def fill_d(d0, d1, bufs):
        kernels.prep_patterns(dt[d0:d1].reshape(d1 - d0, 1, p), bufs, subtract_mean=False)

    def fill_q(q0, q1, bufs):
        kernels.prep_patterns(qt[q0:q1].reshape(q1 - q0, 1, p), bufs, subtract_mean=False)

    cfg = SearchConfig(precision=lp, rescore_k=rescore_k, **shape)
    switch = kernels.set_match_pairs if variant == "pairs" else kernels.set_match_dual
    prev = (kernels.set_match_pairs(False), kernels.set_match_dual(False))
    try:
        base_i, base_v = Searcher(nd, nq, p, k, cfg, DEV).run(fill_d, fill_q)
        switch(True)
        i2, v2 = Searcher(nd, nq, p, k, cfg, DEV).run(fill_d, fill_q)
    finally:
        kernels.set_match_pairs(prev[0])
        kernels.set_match_dual(prev[1])
    torch.cuda.synchronize()
    assert torch.equal(base_i, i2)
    assert torch.equal(base_v, v2)


def test_prep_patterns_integer_counts():
    """uint16 / uint8 / fp16 detector counts prepare to the same rows as the
    same values in float32."""
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.kernels import RowBuffers

    counts = torch.randint(0, 250, (9, 20, 24), dtype=torch.int32)
    ref = torch.empty((9, 480), device=DEV)
    kernels.prep_patterns(counts.float().to(DEV), RowBuffers(f32=ref))
    for dt in (torch.uint16, torch.uint8, torch.float16):
        out = torch.empty((9, 480), device=DEV)
        kernels.prep_patterns(counts.to(dt).to(DEV), RowBuffers(f32=out))
        assert torch.equal(out, ref), dt
    b2 = torch.empty((9, 120), device=DEV)
    r2 = torch.empty((9, 120), device=DEV)
    kernels.prep_patterns(counts.to(torch.uint16).to(DEV), RowBuffers(f32=b2), binning=2)
    kernels.prep_patterns(counts.float().to(DEV), RowBuffers(f32=r2), binning=2)
    assert torch.equal(b2, r2)


def test_match_chunked_dictionary_and_queries():
    """Dictionary chunks with a running merge and several query chunks."""
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.engine import Searcher, SearchConfig

    p, nd, nq, k = 128, 2000, 700, 4
    d = _rows(nd, p, 5)
    q = d[np.arange(nq) * 2] + 0.5 * _rows(nq, p, 6)
    dt, qt = torch.from_numpy(d).float().to(DEV), torch.from_numpy(q).float().to(DEV)

    def fill_d(d0, d1, bufs):
        kernels.prep_patterns(dt[d0:d1].reshape(d1 - d0, 1, p), bufs, subtract_mean=False)

    def fill_q(q0, q1, bufs):
        kernels.prep_patterns(qt[q0:q1].reshape(q1 - q0, 1, p), bufs, subtract_mean=False)

    cfg = SearchConfig(rescore_k=16, dict_chunk=512, query_chunk=256)
    idx, val = Searcher(nd, nq, p, k, cfg, DEV).run(fill_d, fill_q)
    ref_i, ref_v = O.topk_dot(q.astype(np.float32).astype(np.float64), d.astype(np.float32).astype(np.float64), k)
    assert (idx.cpu().numpy() == ref_i).mean() >= 0.999
    assert np.abs(val.cpu().numpy() - ref_v).max() <= 1e-5 * np.abs(ref_v).max()


def test_match_without_rescore_is_close():
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.engine import Searcher, SearchConfig

    p, nd, nq = 256, 1500, 200
    d = _rows(nd, p, 7)
    q = d[np.arange(nq) * 3] + 0.2 * _rows(nq, p, 8)
    dt, qt = torch.from_numpy(d).float().to(DEV), torch.from_numpy(q).float().to(DEV)

    def fill_d(d0, d1, bufs):
        kernels.prep_patterns(dt[d0:d1].reshape(d1 - d0, 1, p), bufs, subtract_mean=False)

    def fill_q(q0, q1, bufs):
        kernels.prep_patterns(qt[q0:q1].reshape(q1 - q0, 1, p), bufs, subtract_mean=False)

    idx, val = Searcher(nd, nq, p, 1, SearchConfig(rescore_k=0), DEV).run(fill_d, fill_q)
    ref_i, ref_v = O.topk_dot(q, d, 1)
    assert (idx.cpu().numpy() == ref_i).mean() >= 0.99
    assert np.abs(val.cpu().numpy() - ref_v).max() <= 2e-2 * np.abs(ref_v).max()


def test_gemm_nt_store_and_split3():
    """Store-epilogue GEMM with the 3-term bf16 split is FP32-class accurate."""
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.kernels import round_up

    rng = np.random.default_rng(9)
    X = torch.from_numpy(rng.standard_normal((300, 200))).float().to(DEV)
    Vt = torch.from_numpy(rng.standard_normal((70, 200))).float().to(DEV)
    seg = round_up(200, 64)
    A3 = kernels.split3(X, 0, False, seg, round_up(300, 128), 3 * seg)
    B3 = kernels.split3(Vt, 1, False, seg, round_up(70, 256), 3 * seg)
    out = torch.empty((300, 70), device=DEV)
    st = kernels.gemm_nt(A3, B3, out, m_valid=300, n_valid=70)
    assert int(st.item()) == 0
    ref = X.double().cpu() @ Vt.double().cpu().T
    assert (out.double().cpu() - ref).abs().max() <= 2e-5 * ref.abs().max()
    # several B tiles streamed by one work unit give the same result
    Wt = torch.from_numpy(rng.standard_normal((1000, 200))).float().to(DEV)
    B4 = kernels.split3(Wt, 1, False, seg, round_up(1000, 256), 3 * seg)
    o1 = torch.empty((300, 1000), device=DEV)
    o2 = torch.empty((300, 1000), device=DEV)
    kernels.gemm_nt(A3, B4, o1, m_valid=300, n_valid=1000)
    assert int(kernels.gemm_nt(A3, B4, o2, m_valid=300, n_valid=1000, splits=2).item()) == 0
    assert torch.equal(o1, o2)
    # transposed split: X^T X with centring
    mu = kernels.col_mean(X)
    segn = round_up(300, 64)
    A = kernels.split3(X, 0, True, segn, round_up(200, 128), 3 * segn, shift=mu)
    B = kernels.split3(X, 1, True, segn, round_up(200, 256), 3 * segn, shift=mu)
    cov = torch.empty((200, 200), device=DEV)
    kernels.gemm_nt(A, B, cov, alpha=1.0 / 299, m_valid=200, n_valid=200)
    ref_cov = np.cov(X.double().cpu().numpy(), rowvar=False)
    assert np.abs(cov.cpu().numpy() - ref_cov).max() <= 2e-5 * np.abs(ref_cov).max()


# ---------------------------------------------------------------------- A14


@pytest.mark.parametrize("laue", [11, 9, 5, 3, 1])
def test_disorientation_matches_reference(golden, laue):
    from ebsdtorch_b200.s2_and_so3.laue_fz_misori import disori_angle_laue

    g = golden("disori")
    a = disori_angle_laue(torch.from_numpy(g[f"q1_{laue}"]).to(DEV), torch.from_numpy(g[f"q2_{laue}"]).to(DEV),
                          laue, laue)
    assert np.abs(a.cpu().numpy() - g[f"ang_{laue}"]).max() < 2e-3  # fp32 acos near 1


@pytest.mark.parametrize("dict_chunk", [None, 512])
def test_host_patterns_prefetch_matches_device_patterns(dict_chunk):
    """Pinned host patterns, copied a query chunk ahead on a side stream while
    the previous chunk is matched (one and several dictionary chunks, a
    ragged last query chunk), give exactly the results of the same patterns
    resident on the device."""
    from ebsdtorch_b200 import kernels
    from ebsdtorch_b200.ebsd.indexing import _query_fill
    from ebsdtorch_b200.engine import Searcher, SearchConfig

    p, nd, nq, k = 16 * 16, 1300, 700, 4
    d = _rows(nd, p, 15)
    pats = (d[np.arange(nq) % nd] + 0.4 * _rows(nq, p, 16)).reshape(nq, 16, 16).astype(np.float32)
    dt = torch.from_numpy(d).float().to(DEV)

    def fill_d(d0, d1, bufs):
        kernels.prep_patterns(dt[d0:d1].reshape(d1 - d0, 1, p), bufs, subtract_mean=True)

    out = []
    for src in (torch.from_numpy(pats).to(DEV), torch.from_numpy(pats).pin_memory()):
        cfg = SearchConfig(rescore_k=16, dict_chunk=dict_chunk, query_chunk=256)
        fill = _query_fill(src, 1, None, p, True, torch.device(DEV))
        out.append(Searcher(nd, nq, p, k, cfg, DEV).run(fill_d, fill))
        if src.device.type == "cpu":
            assert fill.copy_stream is not None and not fill.pending
    assert torch.equal(out[0][0], out[1][0])
    assert torch.equal(out[0][1], out[1][1])
