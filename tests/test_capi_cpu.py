"""The C-ABI library builds for sm_100a, loads without a GPU, and exports every
function declared in include/ebsd_b200.h with the binding's signature. CPU only:
no compute entry point is called here."""

import os
import re

from ebsdtorch_b200 import _capi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "ebsd_b200.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ebsd_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = _declared()
    assert "ebsd_match_topk" in names and "ebsd_project_dictionary" in names
    assert len(names) >= 19


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    for name in _declared():
        assert hasattr(lib, name), name


def test_bindings_cover_header():
    assert set(_declared()) == set(_capi.SIGNATURES)


def test_version_and_error_channel():
    lib = _capi.load()
    assert lib.ebsd_version() >= 100
    assert isinstance(_capi.last_error(), str)


def test_argument_errors_need_no_gpu():
    """Argument checks run on the host before any CUDA call."""
    import pytest

    with pytest.raises(ValueError, match="Laue group"):
        _capi.call("ebsd_grid_fz_count", 12, 10, 1, 1 << 20, 1, None)
    with pytest.raises(ValueError, match="n_cand|multiple"):
        _capi.call("ebsd_match_topk", 16, 100, 16, 256, 256, 64, _capi.DT_BF16, None, 8, 1, 16, 16, 1, 0, 0, 16,
                   None)
    assert _capi.load().ebsd_grid_workspace_bytes(199) > 199**3 // 1024 * 12


def test_device_guard_passes_host_calls_through():
    """Without CUDA data the guard runs the call unchanged (host data goes to
    the current device inside the call)."""
    import torch

    from ebsdtorch_b200._device import _find, on_data_device

    @on_data_device
    def f(xs, scale=1.0, device=None):
        return [x * scale for x in xs]

    x = torch.arange(4.0)
    assert torch.equal(f([x], scale=2.0)[0], x * 2.0)
    assert torch.equal(f([x], device="cpu")[0], x)

    class Holder:
        master_pattern = torch.zeros(2)

    assert _find(Holder()) is None and _find([x, (x,)]) is None


def test_preprocessing_and_fitting_argument_errors_need_no_gpu():
    """The preprocessing and pattern-centre-fitting entry points reject bad
    shapes and parameters on the host, before any CUDA call."""
    import pytest

    fake = 256  # never dereferenced: every call below fails its argument check
    with pytest.raises(ValueError, match="mode"):
        _capi.call("ebsd_normalize_patterns", fake, 4, 16, 16, 7, None)
    with pytest.raises(ValueError, match="n_bins"):
        _capi.call("ebsd_clahe", fake, 2, 16, 16, 256, None, 0, 40.0, 1, 4, 4, 0, fake, 256, None)
    with pytest.raises(ValueError, match="bad grid"):
        _capi.call("ebsd_clahe", fake, 2, 4, 4, 16, None, 0, 40.0, 16, 5, 3, 0, fake, 16, None)
    with pytest.raises(ValueError, match="radius"):
        _capi.call("ebsd_nlpar_dists", fake, 8, 8, 64, 64, 8, fake, 0, 9, 9, fake, None)
    with pytest.raises(ValueError, match="offset block"):
        _capi.call("ebsd_nlpar_average", fake, 8, 8, 64, 64, 3, fake, 0, 129, 129, fake, 0, fake, 64, None)
    with pytest.raises(ValueError, match="at least 9"):
        _capi.call("ebsd_nlpar_weights", fake, 8, 8, 64, fake, 4, 0.375, 1e-6, 0.0, fake, 1 << 20, None)
    with pytest.raises(ValueError, match="workspace too small"):
        _capi.call("ebsd_nlpar_weights", fake, 8, 8, 64, fake, 49, 0.375, 1e-6, 0.0, fake, 16, None)
    with pytest.raises(ValueError, match="does not fit"):
        _capi.call("ebsd_pcfit_prep", fake, 2, 16, 16, 20, 20, 5, 0, 1, fake, None)
    with pytest.raises(ValueError, match="bad sizes"):
        _capi.call("ebsd_pcfit_reduce", fake, 0, 4, 8, 8, 0, fake, fake, None)


def test_pcfit_correlation_kernels_size_limits_need_no_gpu():
    """The tensor-core correlation kernels take enlarged detectors of 2..127
    rows and columns; the table size query says which, and every entry point
    rejects other sizes and bad arguments on the host."""
    import pytest

    lib = _capi.load()
    assert lib.ebsd_pcfit_xcorr_table_bytes(78, 78) == 290816  # six matrices, hi and lo images each
    assert lib.ebsd_pcfit_xcorr_table_bytes(127, 127) > 0
    for h, w in ((128, 78), (78, 128), (1, 40), (40, 1), (0, 0)):
        assert lib.ebsd_pcfit_xcorr_table_bytes(h, w) == 0
    fake = 256  # never dereferenced
    with pytest.raises(ValueError, match="not supported"):
        _capi.call("ebsd_pcfit_xcorr_tables", 128, 60, fake, 1 << 20, None)
    with pytest.raises(ValueError, match="needed"):
        _capi.call("ebsd_pcfit_xcorr_tables", 78, 78, fake, 1024, None)
    with pytest.raises(ValueError, match="16-byte aligned"):
        _capi.call("ebsd_pcfit_xcorr_tables", 78, 78, fake + 4, 1 << 20, None)
    with pytest.raises(ValueError, match="not supported"):
        _capi.call("ebsd_pcfit_spectra", fake, 78 * 78, 4, 200, 78, fake, fake, fake, None)
    with pytest.raises(ValueError, match="leading dimension"):
        _capi.call("ebsd_pcfit_spectra", fake, 78, 4, 78, 78, fake, fake, fake, None)
    with pytest.raises(ValueError, match="32 bits"):
        _capi.call("ebsd_pcfit_xcorr_max", fake, 16, fake, 2, 78, 78, fake, fake, (1 << 32) - 4, fake, None)
    with pytest.raises(ValueError, match="null pointer"):
        _capi.call("ebsd_pcfit_fold", None, 10, fake, fake, None)


def test_noalloc_argument_checks_need_no_gpu():
    """ebsd_match_topk_noalloc rejects bad arguments on the host, before any
    CUDA call: k_out outside 1..64, more queries than padded rows, null
    outputs, and padded query counts whose candidate lists would not fit the
    fixed 32 MiB scratch. The rejection message states the largest padded
    query count that fits for that k (32 MiB - 256 B over 8 B per candidate
    slot, rounded to a power-of-two candidate count)."""
    lib = _capi.load()
    fake = 256  # never dereferenced: every call below fails its argument check

    def call(nq, nq_pad, k, out_val=fake, out_idx=fake):
        return lib.ebsd_match_topk_noalloc(fake, nq, nq_pad, fake, 256, 256, 64, _capi.DT_BF16, None, None, k,
                                           out_val, out_idx, None, None)

    for k in (0, 65, -1):
        assert call(128, 128, k) == 1 and "k_out" in _capi.last_error()
    assert call(129, 128, 8) == 1 and "n_queries" in _capi.last_error()
    assert call(0, 128, 8) == 1 and "n_queries" in _capi.last_error()
    assert call(128, 128, 8, out_val=None) == 1 and "null output" in _capi.last_error()
    assert call(128, 128, 8, out_idx=None) == 1 and "null output" in _capi.last_error()
    cap = (32 << 20) - 256
    for k, n_cand in ((1, 1), (64, 64), (5, 8)):
        most = cap // (8 * n_cand)
        assert call(128, most + 1, k) == 1
        msg = _capi.last_error()
        assert "scratch" in msg and f"at most {most} padded queries" in msg, msg


def test_check_build_query_without_checks_needs_no_gpu():
    """The normal build reports that it carries no device checks (-1)."""
    if _capi.LIB_PATH.endswith("_check.so"):
        return
    assert _capi.debug_check() == (-1, "")


def test_match_variant_switches_need_no_gpu():
    """The match-variant switches: CTA pairs off and two query tiles per CTA
    for e4m3 rows by default; a negative argument only reads the mode; the
    setters return the previous mode."""
    from ebsdtorch_b200 import kernels

    lib = _capi.load()
    pairs0, dual0 = lib.ebsd_set_match_pairs(-1), lib.ebsd_set_match_dual(-1)
    if os.environ.get("EBSD_MATCH_PAIRS") is None:
        assert pairs0 == 0
    if os.environ.get("EBSD_MATCH_DUAL") is None:
        assert dual0 == 2
    try:
        assert lib.ebsd_set_match_pairs(1) == pairs0 and lib.ebsd_set_match_pairs(-1) == 1
        assert kernels.takes_tile_pairs(_capi.DT_BF16) and kernels.takes_tile_pairs(_capi.DT_E4M3)
        lib.ebsd_set_match_pairs(0)
        for mode, bf16, e4m3 in ((0, False, False), (1, True, True), (2, False, True)):
            kernels.set_match_dual(mode)
            assert kernels.match_dual() == mode
            assert kernels.takes_tile_pairs(_capi.DT_BF16) == bf16
            assert kernels.takes_tile_pairs(_capi.DT_E4M3) == e4m3
        assert kernels.set_match_dual(True) == 2 and kernels.match_dual() == 1
    finally:
        lib.ebsd_set_match_pairs(pairs0)
        lib.ebsd_set_match_dual(dual0)
