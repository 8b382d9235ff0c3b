"""The margin-gated FP32 re-score gives exactly the results of re-scoring all
candidates, while reading fewer FP32 rows (ebsd_merge_rescore_gated)."""

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("similarity,precision", [("dot", "bf16"), ("cosine", "bf16"), ("dot", "fp8")])
def test_gate_keeps_results_and_skips_rows(monkeypatch, similarity, precision):
    from ebsdtorch_b200 import engine, kernels, synthetic
    from ebsdtorch_b200.ebsd import dictionary_index_orientations

    mp, geom, exp, _ = synthetic.make_case(257, (64, 64), 3000, seed=41, mean_counts=150.0)
    kw = dict(dictionary_resolution_degrees=1.5, top_k_matches=8, match_dtype=torch.float32, rescore_k=32,
              similarity=similarity, precision=precision)
    runs = {}
    for gated in (True, False):
        if not gated:
            monkeypatch.setattr(kernels, "rescore_gate", lambda *a: 0.0)
        counter = torch.zeros(1, dtype=torch.int64, device="cuda")
        monkeypatch.setattr(engine, "RESCORE_COUNTER", counter)
        torch.manual_seed(3)
        dictionary_index_orientations(mp, geom, exp, **kw)
        runs[gated] = (exp.raw_indexing_indices[0].clone(), exp.raw_indexing_results[0][1].clone(),
                       int(counter.item()))
    (gi, gv, gn), (fi, fv, fn) = runs[True], runs[False]
    assert torch.equal(gi, fi)
    assert torch.equal(gv, fv)
    assert fn == 3000 * 32
    if precision == "bf16":
        assert 3000 * 8 <= gn < fn  # the gate re-scores at least k and fewer than all
    else:
        assert gn == fn  # no gate for e4m3 (its rounding bound is too wide)
    print({"rescored_per_query_gated": gn / 3000, "ungated": fn / 3000})
