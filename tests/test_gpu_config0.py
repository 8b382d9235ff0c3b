"""Plain DI at the small configuration against the reference's own output.

tests/golden/config0.npz holds what the reference's dictionary_index_orientations
(indexing.py:14-211, float32 matching) returned for 4,096 patterns of 60 x 60 px
against the m-3m 1.0 deg dictionary (36,829 rows), top-4; the inputs are rebuilt
by tests/golden/config0_inputs.py and checked against the committed SHA-256.

Tolerances: the top-1 dictionary entry is identical wherever the reference's
own top-1 / top-2 metric gap exceeds 1e-5 of the metric (FP32 dots of 3,600
terms summed in different orders differ by ~1e-6 relative), and on at least
99.9 % of all patterns; each of the four ranks is identical wherever both of
the reference's gaps around it exceed 1e-5; metrics of identical entries agree
to 1e-4 relative.
"""

import os
import sys

import numpy as np
import pytest
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import config0_inputs as C  # noqa: E402

pytestmark = pytest.mark.gpu

GAP = 1e-5


@pytest.fixture(scope="module")
def case(golden):
    d = golden("config0")
    inp = C.make_inputs(C.CASE)
    assert inp["sha256_master_pattern"] == str(d["sha256_master_pattern"]), "master pattern differs from the golden's"
    assert inp["sha256_counts"] == str(d["sha256_counts"]), "rebuilt patterns differ from the golden's"
    return d, inp


def _run(inp, precision, small_plan, monkeypatch):
    from ebsdtorch_b200 import engine
    from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, MasterPattern, dictionary_index_orientations

    c = C.CASE
    mp = MasterPattern(torch.from_numpy(inp["master_pattern"]), laue_group=11).to("cuda")
    geom = EBSDGeometry(c["det"], tilts_degrees=c["tilts"], proj_center=c["pc"]).to("cuda")
    exp = ExperimentPatterns(torch.from_numpy(inp["counts"].astype(np.float32)).to("cuda"))
    kw = {}
    if small_plan:
        # dictionary in chunks of ~6,900 rows merged into a running top-k, and
        # match launches of 8 query tiles (4 launches per query chunk)
        kw["workspace_bytes"] = 300 << 20
        monkeypatch.setattr(engine, "wave_query_tiles", lambda dev, row_bytes=0: 8)
    torch.manual_seed(c["perm_seed"])
    dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=c["res"], top_k_matches=c["k"],
                                  dictionary_chunk_size=c["dictionary_chunk_size"],
                                  experiment_chunk_size=c["experiment_chunk_size"], match_dtype=torch.float32,
                                  precision=precision, **kw)
    return exp


@pytest.mark.parametrize("precision,small_plan", [("bf16", False), ("fp8", False), ("bf16", True)])
def test_config0_matches_reference(case, precision, small_plan, monkeypatch):
    d, inp = case
    exp = _run(inp, precision, small_plan, monkeypatch)
    assert exp.dictionaries[0].shape[0] == int(d["n_dictionary"][0])
    idx = exp.raw_indexing_indices[0].cpu().numpy()
    val = exp.raw_indexing_results[0][1].float().cpu().numpy()
    ref_i, ref_m = d["indices"].astype(np.int64), d["metrics"]
    scale = np.abs(ref_m[:, :1])
    gaps = (ref_m[:, :-1] - ref_m[:, 1:]) / scale  # (Q, 3): gap below rank j
    clear1 = gaps[:, 0] > GAP
    same1 = idx[:, 0] == ref_i[:, 0]
    assert same1[clear1].all(), f"{(~same1[clear1]).sum()} clear top-1 mismatches"
    assert same1.mean() >= 0.999
    for j in range(ref_i.shape[1]):
        above = gaps[:, j - 1] > GAP if j > 0 else np.ones(len(idx), bool)
        below = gaps[:, j] > GAP if j < gaps.shape[1] else np.ones(len(idx), bool)
        clear = above & below
        assert (idx[clear, j] == ref_i[clear, j]).all(), f"rank {j}: clear mismatches"
    same = idx == ref_i
    rel = np.abs(val - ref_m) / scale
    assert rel[same].max() <= 1e-4
    # the metrics come out sorted, like retrieve_topk's (knn.py:268-287)
    assert (np.diff(val, axis=1) <= 0).all()
