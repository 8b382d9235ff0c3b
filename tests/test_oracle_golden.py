"""Pins the CPU oracle against golden vectors produced by the reference
ebsdtorch itself (tests/golden/make_golden.py). CPU only."""

import os

import numpy as np
import pytest

from oracle import di_oracle as O


def _sign_invariant_maxdiff(a, b):
    return float(np.minimum(np.abs(a - b).max(-1), np.abs(a + b).max(-1)).max())


@pytest.mark.parametrize("laue", range(1, 12))
@pytest.mark.parametrize("res", [15.0, 7.5])
def test_grid_sets_match_reference(golden, laue, res):
    ref = golden("grid")[f"q_{laue}_{res}"]
    mine = O.sample_ori_fz_laue_angle(laue, res)
    assert mine.shape == ref.shape
    # same order; q and -q are the same rotation (matters only at w == 0)
    assert _sign_invariant_maxdiff(mine.astype(np.float32), ref) < 2e-6


def test_grid_counts_match_reference(golden):
    counts = golden("grid")["counts"]
    for laue, res, n in counts:
        if n > 100000:  # large grids are checked on the GPU
            continue
        assert O.sample_ori_fz_laue_angle(int(laue), float(res)).shape[0] == int(n)


def test_grid_edge_length_rule(golden):
    # 0.5 deg m-3m: edge 199 -> 328,720 FZ points (count checked on the GPU)
    assert O.grid_edge_length(11, 0.5) == 199
    assert O.grid_edge_length(11, 1.0) == 96


def test_cu2qu_matches_reference(golden):
    g = golden("cu2qu")
    q = O.qu_std(O.cu2qu(g["cu64"]))
    ref = O.qu_std(g["qu64"])
    # reference float64 uses a 10-term polynomial (error ~5e-10 in cos(w/2))
    assert _sign_invariant_maxdiff(q, ref) < 5e-7
    q32 = O.qu_std(O.cu2qu(g["cu"].astype(np.float64)))
    assert _sign_invariant_maxdiff(q32, O.qu_std(g["qu"])) < 3e-6


def test_cu2qu_fp32_poly_mode(golden):
    g = golden("cu2qu")
    q = O.qu_std(O.cu2qu(g["cu"], mode="fp32poly"))
    assert _sign_invariant_maxdiff(q, O.qu_std(g["qu"])) < 3e-6


@pytest.mark.parametrize("name", ["d60", "d60b2", "d5", "d40x32", "d128"])
def test_detector_rays_match_reference(golden, name):
    r = golden("rays")
    m = r[name + "_meta"]
    shape, pc, tilts, b = (int(m[0]), int(m[1])), m[2:5], m[5:8], int(m[8])
    mine = O.detector_coords_sample_frame(shape, pc, tilts, (b, b))
    ref = r[name]
    assert np.abs(mine - ref).max() <= 2e-7 * np.abs(ref).max() * 10


def test_lambert_matches_reference(golden):
    g = golden("lambert")
    uv = O.rosca_lambert_side_by_side(g["xyz"].astype(np.float64))
    assert np.abs(uv - g["uv"]).max() < 5e-7


@pytest.mark.parametrize("b", [1, 2])
def test_projector_matches_reference(golden, b):
    g = golden("projector")
    mp = O.avg_pool(g["master_pattern"].astype(np.float64), b)
    sims = O.project_patterns(mp, g[f"rays_b{b}"].astype(np.float64), g["quats"].astype(np.float64))
    assert np.abs(sims - g[f"sims_b{b}"]).max() < 5e-5


@pytest.mark.parametrize("case", ["di_a", "di_b", "di_c"])
def test_dictionary_index_matches_reference(golden, case):
    d = golden(case)
    m = d["meta"]
    det, pc, res, k, b = (int(m[0]), int(m[1])), m[2:5], m[5], int(m[7]), int(m[8])
    mask = d["mask"] if d["mask"].size else None
    oq, ov, oi, _ = O.dictionary_index(d["master_pattern"], 11, d["patterns"], det, pc, (0, 70, 0), res, top_k=k,
                                       mask=mask, binning=b, dictionary=d["dictionary"].astype(np.float64))
    assert np.abs(oq - d["quats"]).max() < 1e-6  # identical dictionary entries, same order
    assert np.abs(ov - d["metrics"]).max() <= 1e-5 * np.abs(d["metrics"]).max()


def test_permuted_dictionary_matches_reference(golden):
    """The reference dictionary of each DI case equals the oracle grid under
    the permutation torch.randperm draws from the seeded CPU generator."""
    import torch

    d = golden("di_a")
    seed = int(d["meta"][-1])
    base = O.sample_ori_fz_laue_angle(11, float(d["meta"][5]))
    torch.manual_seed(seed)
    perm = torch.randperm(base.shape[0]).numpy()
    assert np.abs(base[perm] - d["dictionary"]).max() < 2e-6


def test_covariance_matches_reference(golden):
    g = golden("covariance")
    x = g["x"].astype(np.float64)
    cov = O.covariance_chan((x[i:i + 64] for i in range(0, x.shape[0], 64)), x.shape[1])
    assert np.abs(cov - g["cov"]).max() <= 1e-4 * np.abs(g["cov"]).max()


def test_pca_shipped_slice_semantics():
    """indexing.py:355 keeps [:, -n : -n + 300]: none for P >= 300 and n < 300."""
    rng = np.random.default_rng(0)
    a = rng.standard_normal((400, 400))
    cov = a @ a.T
    assert O.pca_components(cov, 100, "reference").shape[1] == 0
    assert O.pca_components(cov, 350, "reference").shape[1] == 300
    assert O.pca_components(cov, 100, "top").shape[1] == 100
    small = a[:25, :25] @ a[:25, :25].T
    assert O.pca_components(small, 100, "reference").shape[1] == 25


@pytest.mark.parametrize("laue", [11, 9, 5, 3, 1])
def test_disorientation_matches_reference(golden, laue):
    g = golden("disori")
    ang = O.disori_angle(g[f"q1_{laue}"], g[f"q2_{laue}"], laue)
    assert np.abs(ang - g[f"ang_{laue}"]).max() < 1e-6


@pytest.mark.parametrize("laue", range(1, 12))
def test_laue_groups_are_groups(laue):
    g = O.laue_elements(laue)
    assert g.shape[0] == O.laue_mult(laue) // 2
    assert np.allclose(np.linalg.norm(g, axis=1), 1.0)


@pytest.mark.parametrize("tag", ["top", "shipped", "shipped_n100"])
def test_pca_dictionary_index_matches_reference(golden, tag):
    d = golden("pca_di")
    mode = "top" if tag == "top" else "reference"
    oq, ov, oi = O.pca_dictionary_index(d["master_pattern"], d["patterns"], (16, 16), (0.5, 0.5, 0.6),
                                        d["learn_dictionary"].astype(np.float64),
                                        d["dictionary"].astype(np.float64), int(d[f"ncomp_{tag}"][0]), mode, 2)
    top1 = np.abs(oq[:, 0] - d[f"quats_{tag}"][:, 0]).max(-1) < 1e-5
    assert top1.mean() == 1.0
    ref = d[f"metrics_{tag}"]
    assert np.abs(ov - ref).max() <= 1e-4 * np.abs(ref).max()


def test_rot6d_conversions_match_reference(golden):
    g = golden("rot6d")
    assert np.abs(O.zh2om(g["zh"]) - g["om"]).max() < 1e-12
    assert _sign_invariant_maxdiff(O.zh2qu(g["zh"]), g["qu"]) < 1e-12
    assert np.abs(O.qu2zh(g["qu_in"]) - g["zh_out"]).max() < 1e-12
    assert np.abs(O.qu2om(g["qu_in"]) - g["om_out"]).max() < 1e-12
    assert _sign_invariant_maxdiff(O.om2qu(O.qu2om(g["qu_in"])), g["qu_back"]) < 1e-12


def test_rot6d_sym_loss_gradient_finite_difference():
    rng = np.random.default_rng(3)
    zh = rng.standard_normal((40, 6))
    q = rng.standard_normal((40, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    loss, grad = O.rot6d_sym_loss(zh, q, 11)
    eps = 1e-6
    for j in range(6):
        dz = np.zeros_like(zh)
        dz[:, j] = eps
        lp, _ = O.rot6d_sym_loss(zh + dz, q, 11)
        lm, _ = O.rot6d_sym_loss(zh - dz, q, 11)
        assert np.allclose((lp - lm) / (2 * eps), grad[:, j], atol=1e-5, rtol=1e-4)
    # the loss vanishes at any symmetry-equivalent target g q
    g = O.laue_elements(11)
    qt = O._qmul(np.broadcast_to(g[5], q.shape), q)
    l0, g0 = O.rot6d_sym_loss(O.qu2zh(qt), q, 11)
    assert np.abs(l0).max() < 1e-20 and np.abs(g0).max() < 1e-9


def test_cnn_oracle_gradient_finite_difference():
    """The FP64 CNN oracle (checker of the GPU CNN kernels) is itself exact."""
    rng = np.random.default_rng(0)
    ch = (1, 4, 6)
    params = {}
    for i, (a, b) in enumerate(zip(ch[:-1], ch[1:])):
        params[f"conv{i}.w"] = rng.standard_normal((b, 9 * a)) * np.sqrt(2 / (9 * a))
        params[f"conv{i}.b"] = rng.standard_normal(b) * 0.1
    params["fc1.w"] = rng.standard_normal((5, 24)) * 0.3
    params["fc1.b"] = rng.standard_normal(5) * 0.1
    params["fc2.w"] = rng.standard_normal((6, 5)) * 0.3
    params["fc2.b"] = rng.standard_normal(6) * 0.1
    x = rng.standard_normal((3, 8, 8))
    q = rng.standard_normal((3, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    _, _, g = O.cnn_forward_backward(params, x, q, 11)
    eps = 1e-6
    for k, v in params.items():
        for _ in range(3):
            idx = tuple(rng.integers(0, s) for s in v.shape)
            p2 = {kk: vv.copy() for kk, vv in params.items()}
            p3 = {kk: vv.copy() for kk, vv in params.items()}
            p2[k][idx] += eps
            p3[k][idx] -= eps
            num = (O.cnn_forward_backward(p2, x, q, 11)[1] - O.cnn_forward_backward(p3, x, q, 11)[1]) / (2 * eps)
            assert abs(num - g[k][idx]) <= 1e-6 * max(1.0, abs(num))


def test_symmetry_acts_on_the_left():
    """pattern(g q) == pattern(q) for crystal symmetry g with the projector's
    q v q* ray rotation; the learned-path loss and local search rely on it."""
    from ebsdtorch_b200.synthetic import synthetic_master_pattern

    mp = synthetic_master_pattern(129, seed=1, noise=0.0).numpy().astype(np.float64)
    rays = O.unit_rays(O.detector_coords_sample_frame((24, 24), (0.5, 0.5, 0.6), (0, 70, 0)))
    q = np.array([0.7, 0.1, -0.5, 0.2])
    q /= np.linalg.norm(q)
    base = O.project_patterns(mp, rays, q[None])[0]
    g = O.laue_elements(11)[1]  # 180 deg about z: maps lattice points onto lattice points exactly
    assert np.abs(O.project_patterns(mp, rays, O._qmul(g, q)[None])[0] - base).max() < 1e-3
    assert np.abs(O.project_patterns(mp, rays, O._qmul(q, g)[None])[0] - base).max() > 0.1


# ------------------------------------------------- orientation grid refinement


def test_local_orientation_grid_matches_reference(golden):
    g = golden("refine")
    for i in range(4):
        e, r, a = g[f"grid{i}_args"]
        mine = O.local_orientation_grid(float(e), int(r), int(a))
        assert mine.shape == g[f"grid{i}"].shape
        assert np.abs(mine - g[f"grid{i}"]).max() < 1e-7


def _refine_case(g, ci):
    det0, det1, b, edge, radius, axial, n_iter, shrink, avg = g[f"case{ci}_meta"]
    det, b = (int(det0), int(det1)), int(b)
    mp = O.avg_pool(g[f"case{ci}_master_pattern"].astype(np.float64), b)
    coords = O.detector_coords_sample_frame(det, (0.5, 0.5, 0.6), (0.0, 70.0, 0.0), binning=(b, b))
    rows = O.prep_patterns(g[f"case{ci}_patterns"].astype(np.float64), b)
    off = None if avg else g[f"case{ci}_spatial"].astype(np.float64)
    if avg:
        coords = O.unit_rays(coords)
    return O.orientation_grid_refinement(mp, coords, rows, g[f"case{ci}_start"].astype(np.float64), 11, float(edge),
                                         int(n_iter), int(axial), int(radius), float(shrink), offsets=off)


@pytest.mark.parametrize("ci", [0, 1, 2])
def test_refinement_oracle_matches_reference(golden, ci):
    """The FP64 restatement of orientation_grid_refinement reproduces the
    reference's refined orientations and per-iteration best dot products
    (radius 1 and 2, full / biaxial / uniaxial grids, binning 2, per-pattern
    source points; float32 reference)."""
    g = golden("refine")
    q, dots = _refine_case(g, ci)
    ref = g[f"case{ci}_refined"].astype(np.float64)
    err = np.minimum(np.abs(q - ref).max(1), np.abs(q + ref).max(1))
    assert err.max() < 5e-5
    ref_d = g[f"case{ci}_dots"]
    assert np.abs(dots - ref_d).max() <= 2e-4 * np.abs(ref_d).max()


def test_left_fz_reduction_keeps_the_pattern():
    """The left reduction g q moves a rotation into the FZ without changing
    its simulated pattern (up to interpolation on the Lambert grid); the
    reference's right product q g changes it."""
    from ebsdtorch_b200 import synthetic

    rng = np.random.default_rng(3)
    rays = O.unit_rays(O.detector_coords_sample_frame((12, 12), (0.5, 0.5, 0.6), (0.0, 70.0, 0.0)))
    q = rng.standard_normal((40, 4))
    q = O.qu_std(q / np.linalg.norm(q, axis=1, keepdims=True))
    # noise-free cubic bands: exactly m-3m symmetric
    mp = synthetic.synthetic_master_pattern(257, seed=2, noise=0.0).numpy().astype(np.float64)
    left = O.ori_to_fz_laue_left(q, 11)
    right = O.ori_to_fz_laue_right(q, 11)
    assert np.all(O.ori_in_fz_laue(left, 11))
    p0 = O.project_patterns(mp, rays, q)
    assert np.abs(O.project_patterns(mp, rays, left) - p0).max() < 0.05
    assert np.abs(O.project_patterns(mp, rays, right) - p0).max() > 0.3


# ---- experimental-pattern preprocessing -----------------------------------


def _rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


def test_background_and_normalisation_oracle_match_reference(golden):
    """subtract_overall_background and the three normalize_per_pattern modes
    (experiment_pats.py:223-285) on 11 patterns of 40 x 36."""
    g = golden("preprocess")
    pats = g["pats"].astype(np.float64)
    assert _rel(O.subtract_overall_background(pats), g["background"]) < 1e-5
    for mode, tol in (("minmax", 1e-6), ("zeromean", 1e-5), ("standard", 1e-5)):
        assert _rel(O.normalize_per_pattern(pats, mode), g[f"norm_{mode}"]) < tol, mode


@pytest.mark.parametrize("name", ["clahe_a", "clahe_b", "clahe_c"])
def test_clahe_oracle_matches_reference(golden, name):
    """clahe_grayscale (clahe.py:17-130): clip 40 / 64 bins / 4 x 4 grid
    (reflect padding on both axes), clip 2 / 32 bins / 3 x 5 grid, and no
    clipping / 16 bins / 2 x 2 grid."""
    g = golden("preprocess")
    clip, bins, gh, gw = g[name + "_args"]
    out = O.clahe(g["unit"].astype(np.float64), float(clip), int(bins), (int(gh), int(gw)))
    assert np.abs(out - g[name]).max() < 1e-5


def test_standard_clean_oracle_matches_reference(golden):
    g = golden("preprocess")
    assert np.abs(O.standard_clean(g["pats"].astype(np.float64)) - g["standard_clean"]).max() < 1e-5


@pytest.mark.parametrize("name", ["nlpar_a", "nlpar_b"])
def test_nlpar_oracle_matches_reference(golden, name):
    """nlpar (nlpar.py:19-192) on a 7 x 9 scan of 16 x 12 patterns with
    k_rad 1 / coeff 0.375 and k_rad 3 / coeff 0.5."""
    g = golden("preprocess")
    k, c = g[name + "_args"]
    out = O.nlpar(g["nlpar_in"].astype(np.float64), int(k), float(c))
    assert _rel(out, g[name]) < 1e-6


def test_nlpar_offsets_order():
    """Offsets sorted by L1 norm: 0 is the point itself, 1..4 its axial
    neighbours, 5..8 four of the L1-norm-2 offsets (diagonals or axial at
    distance 2, as torch.argsort breaks the ties), which feed the noise
    estimate and the coefficient fit."""
    for k in (1, 3, 5, 7):
        off = O.nlpar_offsets(k)
        l1 = np.abs(off).sum(1)
        assert off.shape == ((2 * k + 1) ** 2, 2)
        assert l1[0] == 0 and (l1[1:5] == 1).all() and (l1[5:9] == 2).all()
        assert (l1[:-1] <= l1[1:]).all()
        assert len({tuple(o) for o in off}) == off.shape[0]


# ---- pattern-centre fitting ---------------------------------------------------


def _pcfit_args(g, ci):
    H, W, b, x0, x1, y0, y1, z0, z1, zs, tilt, sec, res, bs, seed = g[f"case{ci}_meta"]
    return dict(pc_x_min=x0, pc_x_max=x1, pc_y_min=y0, pc_y_max=y1, pc_z_min=z0, pc_z_max=z1, pc_z_steps=int(zs),
                primary_tilt_deg=tilt, secondary_tilt_deg=sec, virtual_binning=int(b)), int(bs), int(seed)


@pytest.mark.parametrize("ci", [0, 1, 2])
def test_pc_fit_oracle_matches_reference(golden, ci):
    """spatial_fft_pc_fitter (fitting.py:359-540): the enlarged pixel grid,
    the simulated dictionary on it, and the fitted pattern centre and
    orientations (binning 1 / 2, one and two dictionary batches, secondary
    tilt, an odd enlarged height)."""
    g = golden("pcfit")
    kw, bs, _ = _pcfit_args(g, ci)
    H, W = (int(v) for v in g[f"case{ci}_meta"][:2])
    pix, pad, shape = O.pixel_coords_with_periphery((H, W), kw["pc_x_min"], kw["pc_x_max"], kw["pc_y_min"],
                                                    kw["pc_y_max"], kw["virtual_binning"])
    assert np.array_equal(pix, g[f"case{ci}_pixel_coords"].astype(np.float64))
    assert (*pad, *shape) == tuple(g[f"case{ci}_padding"])
    rot, t = O.bruker_se3((0.5, 0.5, float(np.float32(kw["pc_z_min"]))), -kw["primary_tilt_deg"],
                          kw["secondary_tilt_deg"], (H, W))
    mp = O.avg_pool(g[f"case{ci}_master_pattern"].astype(np.float64), kw["virtual_binning"])
    sims = O.project_patterns(mp, O.unit_rays(pix @ rot.T + t), g[f"case{ci}_dictionary"][:4].astype(np.float64))
    assert np.abs(sims.reshape(g[f"case{ci}_sims"].shape) - g[f"case{ci}_sims"]).max() < 2e-4
    pc, idx, _ = O.spatial_fft_pc_fit(g[f"case{ci}_master_pattern"], g[f"case{ci}_patterns"],
                                      g[f"case{ci}_dictionary"], batch_size=bs, batch_local_index=True, **kw)
    assert np.abs(pc - g[f"case{ci}_best_pc"]).max() < 1e-6
    assert np.array_equal(g[f"case{ci}_dictionary"][idx], g[f"case{ci}_best_quats"])


def test_bruker_se3_round_trip():
    import torch

    from ebsdtorch_b200.ebsd import fitting as F

    pcs = torch.tensor([[0.45, 0.55, 0.6], [0.5, 0.4, 0.7]], dtype=torch.float64)
    r, t = F.bruker_geometries_to_SE3(pcs, torch.tensor(70.0), torch.tensor(10.0), (60, 80))
    back, tilt, sec = F.bruker_geometry_from_SE3(r, t, (60, 80))
    assert torch.allclose(back, pcs, atol=1e-12)
    assert torch.allclose(tilt, torch.full((2,), 70.0, dtype=torch.float64))
    assert torch.allclose(sec, torch.full((2,), 10.0, dtype=torch.float64))


# ---- EMsoft master-pattern reader -------------------------------------------

_EMSOFT_KEYS = ("EMData/MCOpenCL/accum_e", "EMData/EBSDmaster/mLPNH", "EMData/EBSDmaster/mLPSH",
                "CrystalData/SpaceGroupNumber")


def _emsoft_case(g, ci):
    return {k: g[f"case{ci}/{k}"] for k in _EMSOFT_KEYS}


@pytest.mark.parametrize("ci", [0, 1, 2])
def test_emsoft_reader_oracle_and_port_match_reference(golden, ci):
    """read_master_pattern (io/read_master_pattern.py:7-53), run by the
    reference on the same arrays: 5 / 1 / 7 energy bins, space groups 225 /
    194 / 62. The FP64 oracle and the reader agree with it."""
    from ebsdtorch_b200.io import master_pattern_from_emsoft

    g = golden("emsoft_reader")
    d = _emsoft_case(g, ci)
    ref = g[f"case{ci}_master_pattern"]
    ora = O.emsoft_master_pattern(d[_EMSOFT_KEYS[0]], d[_EMSOFT_KEYS[1]], d[_EMSOFT_KEYS[2]])
    assert np.abs(ora - ref).max() <= 1e-6 * np.abs(ref).max()
    mp = master_pattern_from_emsoft(d[_EMSOFT_KEYS[0]], d[_EMSOFT_KEYS[1]], d[_EMSOFT_KEYS[2]],
                                    int(d[_EMSOFT_KEYS[3]][0]))
    assert str(mp.master_pattern.dtype) == "torch.float32" and tuple(mp.master_pattern.shape) == ref.shape
    assert np.abs(mp.master_pattern.numpy() - ref).max() <= 1e-6 * np.abs(ref).max()
    assert mp.laue_group == int(g[f"case{ci}_laue_group"][0])


def test_read_master_pattern_through_the_file_api(golden):
    """The reader opens the file with h5py's File API: an in-memory stand-in
    of that API gives the reference's result; without h5py it raises."""
    import types

    from ebsdtorch_b200.io import read_master_pattern

    g = golden("emsoft_reader")
    d = _emsoft_case(g, 0)

    class _File:
        def __init__(self, path, mode):
            assert path == "scan.h5" and mode == "r"

        def __enter__(self):
            return d

        def __exit__(self, *a):
            return False

    fake = types.SimpleNamespace(File=_File)
    mp = read_master_pattern("scan.h5", h5py_module=fake)
    ref = g["case0_master_pattern"]
    assert np.abs(mp.master_pattern.numpy() - ref).max() <= 1e-6 * np.abs(ref).max()
    try:
        import h5py  # noqa: F401
    except ImportError:
        with pytest.raises(ImportError, match="h5py"):
            read_master_pattern("scan.h5")


def test_config0_inputs_reproduce_the_golden_checksums(golden):
    """The config-0 inputs (tests/golden/config0_inputs.py) rebuild bit-exactly."""
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import config0_inputs as C

    d = golden("config0")
    inp = C.make_inputs(C.CASE)
    assert inp["sha256_master_pattern"] == str(d["sha256_master_pattern"])
    assert inp["sha256_counts"] == str(d["sha256_counts"])
    # the oracle's float32 DI of the first 48 patterns agrees with the
    # reference's top-4 over the whole 36,829-row dictionary
    c = C.CASE
    import torch

    base = O.sample_ori_fz_laue_angle(11, c["res"])
    assert base.shape[0] == int(d["n_dictionary"][0])
    torch.manual_seed(c["perm_seed"])  # the reference's randperm convention
    dictionary = base[torch.randperm(base.shape[0]).numpy()]
    rays = O.unit_rays(O.detector_coords_sample_frame(c["det"], c["pc"], c["tilts"]))
    rows = O.dictionary_rows(inp["master_pattern"], rays, dictionary, dtype=np.float32, chunk=1024)
    q = O.prep_patterns(inp["counts"][:48].astype(np.float32), dtype=np.float32)
    idx, val = O.topk_dot(q, rows, c["k"])
    ref_i, ref_m = d["indices"][:48], d["metrics"][:48]
    assert (idx[:, 0] == ref_i[:, 0]).all()
    same = idx == ref_i
    assert same.mean() >= 0.99
    assert (np.abs(val - ref_m)[same] / np.abs(ref_m[:, :1]).repeat(4, 1)[same]).max() < 1e-4


@pytest.mark.parametrize("case", [0, 1, 2, 3])
def test_distance_metric_dictionary_index_matches_reference(golden, case):
    """distance_metric="euclidean" (knn.py:85-91, squared distances) and
    "manhattan" (:92-93, L1 distances) of the zero-mean rows, smallest first."""
    d = golden("di_euclid")
    m = d[f"case{case}_meta"]
    det, res, k, b = (int(m[0]), int(m[1])), m[2], int(m[4]), int(m[5])
    mask = d[f"case{case}_mask"] if d[f"case{case}_mask"].size else None
    oq, ov, _, _ = O.dictionary_index(d[f"case{case}_master_pattern"], 11, d[f"case{case}_patterns"], det,
                                      (0.5, 0.5, 0.6), (0, 70, 0), res, top_k=k, mask=mask, binning=b,
                                      dictionary=d[f"case{case}_dictionary"].astype(np.float64),
                                      distance_metric=str(d[f"case{case}_metric"]))
    assert np.abs(oq - d[f"case{case}_quats"]).max() < 1e-6
    assert np.abs(ov - d[f"case{case}_dists"]).max() <= 1e-4 * np.abs(d[f"case{case}_dists"]).max()
    assert (np.diff(ov, axis=1) >= 0).all()
