"""The pattern-centre fitter's tensor-core correlation kernels
(ebsd_pcfit_spectra, ebsd_pcfit_xcorr_max, ebsd_pcfit_fold) against the FFT
formulation the reference uses (fitting.py:413, 484-507), computed here in
float64 with torch.fft; and the fitter's two search paths against each
other."""

import pytest
import torch

from ebsdtorch_b200._capi import call, load, ptr

pytestmark = pytest.mark.gpu

DEV = "cuda"
SIZES = [(78, 78), (23, 22), (14, 13), (16, 16), (120, 120), (127, 64)]


def _tables(hp, wp):
    n = int(load().ebsd_pcfit_xcorr_table_bytes(hp, wp))
    assert n > 0
    t = torch.empty((n,), dtype=torch.uint8, device=DEV)
    call("ebsd_pcfit_xcorr_tables", hp, wp, ptr(t), n, None)
    return t


def _spectra(imgs, tables, hp, wp, status):
    n = imgs.shape[0]
    out = torch.empty((n, 4 * (hp // 2 + 1) * (wp // 2 + 1)), dtype=torch.float32, device=DEV)
    call("ebsd_pcfit_spectra", ptr(imgs), hp * wp, n, hp, wp, ptr(tables), ptr(out), ptr(status), None)
    return out


@pytest.mark.parametrize("hp,wp", SIZES)
def test_spectra_match_fft(hp, wp):
    g = torch.Generator(device="cpu").manual_seed(hp * 1000 + wp)
    imgs = torch.rand((5, hp, wp), generator=g).to(DEV)
    tables = _tables(hp, wp)
    status = torch.zeros(1, dtype=torch.int32, device=DEV)
    spec = _spectra(imgs.reshape(5, -1), tables, hp, wp, status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    h2, wf = hp // 2 + 1, wp // 2 + 1
    sp = spec.double().view(5, 2, 2, h2, wf)
    cc = torch.complex(sp[:, 0, 0], sp[:, 0, 1])
    ss = torch.complex(sp[:, 1, 0], sp[:, 1, 1])
    ref = torch.fft.rfft2(imgs.double())
    ky = torch.arange(h2, device=DEV)
    scale = float(ref.abs().max())
    assert float((cc - 1j * ss - ref[:, ky]).abs().max()) < 2e-5 * scale
    assert float((cc + 1j * ss - ref[:, (-ky) % hp]).abs().max()) < 2e-5 * scale


def _reference_batch_max(sims, pats):
    """max / first argmax over the simulated patterns of
    fftshift(irfft2(rfft2(sim) * conj(rfft2(pat)))), float64."""
    hp, wp = sims.shape[-2:]
    sf = torch.fft.rfft2(sims.double())
    pf = torch.fft.rfft2(pats.double()).conj()
    maps = torch.fft.fftshift(torch.fft.irfft2(sf[:, None] * pf[None], s=(hp, wp)), dim=(-2, -1))  # (n, B, h, w)
    v, i = maps.max(dim=0)
    top2 = maps.topk(2, dim=0).values
    return v, i, top2[0] - top2[1], maps.pow(2).mean().sqrt()


@pytest.mark.parametrize("hp,wp", SIZES)
def test_xcorr_max_matches_fft(hp, wp):
    n, B = 37, 3
    g = torch.Generator(device="cpu").manual_seed(7 + hp + wp)
    sims = torch.rand((n, hp, wp), generator=g).to(DEV)
    pats = torch.zeros((B, hp, wp), device=DEV)
    pats[:, 3:hp - 2, 2:wp - 3] = torch.randn((B, hp - 5, wp - 5), generator=g).to(DEV)
    tables = _tables(hp, wp)
    status = torch.zeros(1, dtype=torch.int32, device=DEV)
    sspec = _spectra(sims.reshape(n, -1), tables, hp, wp, status)
    pspec = _spectra(pats.reshape(B, -1), tables, hp, wp, status)
    terms = torch.empty_like(pspec)
    call("ebsd_pcfit_pattern_terms", ptr(pspec), B, hp, wp, ptr(terms), None)
    keys = torch.zeros((B * hp * wp,), dtype=torch.int64, device=DEV)
    # two launches into one batch's keys: entries [0, 20) and [20, 37)
    call("ebsd_pcfit_xcorr_max", ptr(sspec), 20, ptr(terms), B, hp, wp, ptr(tables), ptr(keys), 0, ptr(status), None)
    call("ebsd_pcfit_xcorr_max", ptr(sspec[20:]), n - 20, ptr(terms), B, hp, wp, ptr(tables), ptr(keys), 20,
         ptr(status), None)
    best = torch.full((B, hp, wp), -1e30, device=DEV)
    best_idx = torch.full((B, hp, wp), -1, dtype=torch.int64, device=DEV)
    call("ebsd_pcfit_fold", ptr(keys), keys.numel(), ptr(best), ptr(best_idx), None)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    assert int(keys.abs().sum()) == 0  # the fold clears the keys
    v, i, gap, rms = _reference_batch_max(sims, pats)
    err = float((best.double() - v).abs().max() / rms)
    assert err < 2e-4, err
    clear = gap > 2e-3 * rms
    assert bool((best_idx == i)[clear].all())
    assert int(clear.sum()) > 0.9 * clear.numel()


def test_fold_keeps_the_running_best_rule():
    """best = max(best, batch max); the index is replaced where they are
    equal (a later batch wins a tie); zero keys leave an entry alone."""
    hp, wp = 14, 13
    tables = _tables(hp, wp)
    status = torch.zeros(1, dtype=torch.int32, device=DEV)
    g = torch.Generator(device="cpu").manual_seed(3)
    sims = torch.rand((6, hp, wp), generator=g).to(DEV)
    pats = torch.randn((1, hp, wp), generator=g).to(DEV)
    sspec = _spectra(sims.reshape(6, -1), tables, hp, wp, status)
    pspec = _spectra(pats.reshape(1, -1), tables, hp, wp, status)
    terms = torch.empty_like(pspec)
    call("ebsd_pcfit_pattern_terms", ptr(pspec), 1, hp, wp, ptr(terms), None)
    keys = torch.zeros((hp * wp,), dtype=torch.int64, device=DEV)
    best = torch.zeros((hp, wp), device=DEV)
    best_idx = torch.zeros((hp, wp), dtype=torch.int64, device=DEV)
    # the same entries twice, as two batches with different index bases
    for base in (0, 100):
        call("ebsd_pcfit_xcorr_max", ptr(sspec), 6, ptr(terms), 1, hp, wp, ptr(tables), ptr(keys), base,
             ptr(status), None)
        call("ebsd_pcfit_fold", ptr(keys), keys.numel(), ptr(best), ptr(best_idx), None)
    torch.cuda.synchronize()
    v, i, _, rms = _reference_batch_max(sims, pats)
    pos, neg = v[0] > 1e-3 * rms, v[0] < -1e-3 * rms
    assert bool(pos.any()) and bool(neg.any())
    # positive maxima: the second batch ties the first and wins
    assert bool((best_idx[pos] >= 100).all())
    # negative maxima never beat the initial 0: index untouched
    assert bool((best_idx[neg] == 0).all()) and bool((best[neg] == 0).all())


def test_fitter_paths_agree(monkeypatch):
    """spatial_fft_pc_fitter through the tensor-core kernels and through
    cuFFT give the same pattern centre and orientations."""
    from ebsdtorch_b200 import synthetic
    from ebsdtorch_b200.ebsd import EBSDGeometry, MasterPattern, spatial_fft_pc_fitter
    from ebsdtorch_b200.ebsd import fitting as F

    mp_t = synthetic.synthetic_master_pattern(257, seed=5, device=DEV)
    geom = EBSDGeometry((40, 40), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.48, 0.52, 0.55))
    q = synthetic.random_quaternions(6, 11).to(DEV)
    pats = synthetic.synthetic_patterns(mp_t, geom, q, mean_counts=300.0, seed=12).view(6, 1, 40, 40)
    mp = MasterPattern(mp_t, laue_group=11)
    kw = dict(pc_x_min=0.4, pc_x_max=0.6, pc_y_min=0.4, pc_y_max=0.6, pc_z_min=0.5, pc_z_max=0.6, pc_z_steps=3,
              dictionary_resolution_deg=6.0, dictionary_indexing_batch_size=256)
    out = {}
    for path in ("dft", "fft"):
        if path == "fft":
            monkeypatch.setattr(F, "xcorr_supported", lambda hp, wp: False)
        torch.manual_seed(1)
        out[path] = spatial_fft_pc_fitter(mp, pats.clone(), **kw)
    (pc_d, q_d), (pc_f, q_f) = out["dft"], out["fft"]
    assert torch.equal(pc_d, pc_f)
    assert torch.equal(q_d, q_f)
