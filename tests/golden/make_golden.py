"""Generate golden vectors by running the reference ebsdtorch itself (CPU torch).

Run in a container that holds the reference source tree:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py [--<case>-only] [REFERENCE_ROOT]

REFERENCE_ROOT is the directory holding the reference's ``ebsdtorch/``; without
it, $EBSD_REFERENCE_ROOT, then the copy staged by ``oracle/stage_ref.py`` in
``oracle/_ref`` are used (``oracle/ref_loader.py``). The reference's
``ebsdtorch/ebsd/indexing.py`` ends in a module-level demo script that imports
``kikuchipy`` (absent), so the two DI functions are loaded by executing only
the file's lines 1-477 into a fresh module; nothing in the reference tree is
modified. The PCA variant is also loaded with line 355's component slice
``[:, -n : -n + 300]`` replaced by ``[:, -n:]`` (the "top" slice).

Outputs ``tests/golden/*.npz``; each file holds the inputs and the reference
outputs of one case (``--refinement-only`` / ``--preprocessing-only`` /
``--pcfit-only`` / ``--reader-only`` write just refine.npz / preprocess.npz /
pcfit.npz / emsoft_reader.npz; ``--config0-only`` writes config0.npz, the
reference's own plain DI at the small configuration on inputs rebuilt by
``config0_inputs.py``; ``--euclidean-only`` writes di_euclid.npz, plain DI with
the euclidean distance; ``--pca-config0-only`` writes pca_config0.npz, the
reference's own PCA DI on the config-0 inputs). The files are small (< 1 MB
each) and committed.
"""

from __future__ import annotations

import contextlib
import io
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import ref_loader  # noqa: E402


def load_reference(root=None):
    """(indexing module as shipped, indexing module with the "top" PCA slice)."""
    return ref_loader.load_indexing(root), ref_loader.load_indexing(root, top_slice=True)


def smooth_master_pattern(seed: int, n: int) -> torch.Tensor:
    """Seeded smooth random (n, 2n) side-by-side master pattern."""
    g = torch.Generator().manual_seed(seed)
    base = torch.rand((1, 1, 2 * n // 4 + 2, 2 * (2 * n // 4) + 2), generator=g)
    mp = torch.nn.functional.interpolate(base, size=(n, 2 * n), mode="bicubic", align_corners=True)[0, 0]
    return mp.contiguous().float()


def refinement_goldens(root=None):
    """Orientation grid refinement (ebsd/refining.py): local grids and three
    refinement cases (kernel radius, axial grid, binning, shrink factor,
    pattern-centre mode), float32 matching."""
    ref_loader.import_reference(root)
    from ebsdtorch.ebsd.refining import get_local_orientation_grid, orientation_grid_refinement
    from ebsdtorch.s2_and_so3.sampling import so3_uniform_quat
    from ebsdtorch.s2_and_so3.quaternions import qu_prod
    from ebsdtorch.s2_and_so3.orientations import ax2qu
    from ebsdtorch.ebsd.geometry import EBSDGeometry
    from ebsdtorch.ebsd.master_pattern import MasterPattern
    from ebsdtorch.ebsd.experiment_pats import ExperimentPatterns
    from ebsdtorch.s2_and_so3.quaternions import qu_apply

    out = {}
    for i, (e, r, a) in enumerate(((2.0, 1, 3), (1.0, 2, 2), (1.5, 2, 1), (3.0, 3, 3))):
        out[f"grid{i}"] = get_local_orientation_grid(e, r, a).numpy()
        out[f"grid{i}_args"] = np.array([e, r, a], dtype=np.float64)
    cases = [
        dict(det=(20, 20), seed=31, n=14, b=1, edge=2.0, radius=1, axial=3, n_iter=3, shrink=0.5, avg=True),
        dict(det=(24, 20), seed=32, n=9, b=2, edge=1.5, radius=2, axial=2, n_iter=4, shrink=0.6, avg=True),
        dict(det=(16, 16), seed=33, n=7, b=1, edge=2.5, radius=1, axial=1, n_iter=3, shrink=0.5, avg=False),
    ]
    for ci, c in enumerate(cases):
        torch.manual_seed(c["seed"])
        mp_t = smooth_master_pattern(c["seed"], 41)
        mp = MasterPattern(mp_t.clone(), laue_group=11)
        geom = EBSDGeometry(c["det"], tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
        truth = so3_uniform_quat(c["n"], torch.device("cpu"))
        dc = geom.get_coords_sample_frame(binning=(1, 1))
        dc = dc / dc.norm(dim=-1, keepdim=True)
        with torch.no_grad():
            pats = mp.interpolate(qu_apply(truth[:, None, :], dc[None]), normalize_coords=False).reshape(
                c["n"], *c["det"])
            pats = pats + 0.01 * torch.randn_like(pats)
        # starting orientations: the truth rotated by 1-2.5 degrees about random axes
        ax = torch.randn((c["n"], 3))
        ax = ax / ax.norm(dim=1, keepdim=True)
        ang = torch.deg2rad(1.0 + 1.5 * torch.rand(c["n"]))
        start = qu_prod(ax2qu(torch.cat((ax, ang[:, None]), dim=1)), truth)
        exp = ExperimentPatterns(pats.clone())
        exp.set_orientations(start.clone())
        exp.phases = torch.zeros(c["n"], dtype=torch.int64)
        spatial = None
        if not c["avg"]:
            spatial = 3.0 * torch.randn((c["n"], 2))
            exp.set_spatial_coords(spatial.clone())
        with contextlib.redirect_stdout(io.StringIO()):
            dots = orientation_grid_refinement(
                mp, geom, exp, grid_semi_edge_in_degrees=c["edge"], batch_size=5, virtual_binning=c["b"],
                n_iter=c["n_iter"], axial_grid_dimension=c["axial"], kernel_radius_in_steps=c["radius"],
                shrink_factor=c["shrink"], average_pattern_center=c["avg"], match_dtype=torch.float32)
        out[f"case{ci}_master_pattern"] = mp_t.numpy()
        out[f"case{ci}_patterns"] = pats.numpy()
        out[f"case{ci}_truth"] = truth.numpy()
        out[f"case{ci}_start"] = start.numpy()
        out[f"case{ci}_spatial"] = spatial.numpy() if spatial is not None else np.zeros((0, 2), np.float32)
        out[f"case{ci}_refined"] = exp.orientations.numpy()
        out[f"case{ci}_dots"] = dots[0].numpy()
        out[f"case{ci}_meta"] = np.array([*c["det"], c["b"], c["edge"], c["radius"], c["axial"], c["n_iter"],
                                          c["shrink"], float(c["avg"])], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "refine.npz"), **out)


def preprocessing_goldens(root=None):
    """Pattern preprocessing (experiment_pats.py:223-316, preprocessing/
    clahe.py, nlpar.py): overall background, per-pattern normalisation,
    CLAHE (divisible and reflect-padded sizes), standard_clean, NLPAR."""
    ref_loader.import_reference(root)
    from ebsdtorch.ebsd.experiment_pats import ExperimentPatterns
    from ebsdtorch.preprocessing.clahe import clahe_grayscale
    from ebsdtorch.preprocessing.nlpar import nlpar

    out = {}
    g = torch.Generator().manual_seed(71)
    base = torch.rand((1, 1, 12, 12), generator=g)
    img = torch.nn.functional.interpolate(base, size=(40, 36), mode="bicubic", align_corners=True)[0, 0]
    pats = (img[None] * 200 + 40 * torch.rand((11, 40, 36), generator=g)).float()
    out["pats"] = pats.numpy()
    e = ExperimentPatterns(pats.clone())
    e.subtract_overall_background()
    out["background"] = e.patterns.numpy()
    for mode in ("minmax", "zeromean", "standard"):
        e = ExperimentPatterns(pats.clone())
        e.normalize_per_pattern(norm_type=mode)
        out[f"norm_{mode}"] = e.patterns.numpy()
    unit = pats - pats.amin(dim=(1, 2), keepdim=True)
    unit = unit / unit.amax(dim=(1, 2), keepdim=True)
    out["unit"] = unit.numpy()
    for name, (clip, bins, grid) in {"clahe_a": (40.0, 64, (4, 4)), "clahe_b": (2.0, 32, (3, 5)),
                                     "clahe_c": (0.0, 16, (2, 2))}.items():
        out[name] = clahe_grayscale(unit[:, None].clone(), clip_limit=clip, n_bins=bins, grid_shape=grid)[:, 0].numpy()
        out[name + "_args"] = np.array([clip, bins, *grid], dtype=np.float64)
    e = ExperimentPatterns(pats.clone())
    e.standard_clean()
    out["standard_clean"] = e.patterns.numpy()
    # NLPAR on a 7 x 9 scan of 16 x 12 patterns: smooth grains plus noise
    scan = torch.zeros((7, 9, 16, 12))
    for k, (a, b) in enumerate(((0, 4), (4, 9))):
        bp = torch.nn.functional.interpolate(torch.rand((1, 1, 5, 5), generator=g), size=(16, 12), mode="bicubic",
                                             align_corners=True)[0, 0]
        scan[:, a:b] = bp * 100
    scan[3:, 2:6] += 30
    scan = scan + 8 * torch.randn(scan.shape, generator=g)
    out["nlpar_in"] = scan.numpy()
    for name, (k, c) in {"nlpar_a": (1, 0.375), "nlpar_b": (3, 0.5)}.items():
        out[name] = nlpar(scan.clone(), k_rad=k, coeff=c).numpy()
        out[name + "_args"] = np.array([k, c], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "preprocess.npz"), **out)


def pcfit_goldens(root=None):
    """Pattern-centre fitting (ebsd/fitting.py:359-540, spatial FFT fitter):
    three cases (binning 1 / 2, one or several dictionary batches, tilts),
    the enlarged pixel grid and the first simulated dictionary patterns.
    fitting.py imports matplotlib (for a plotting helper that is commented
    out) and, through io/read_master_pattern.py, h5py; neither is used by the
    fitter, so empty stand-in modules are registered when they are absent."""
    ref_loader.import_reference(root)
    for name in ("matplotlib", "matplotlib.pyplot", "h5py"):
        try:
            __import__(name)
        except ImportError:
            sys.modules[name] = types.ModuleType(name)
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    from ebsdtorch.ebsd import fitting as F
    from ebsdtorch.ebsd.master_pattern import MasterPattern
    from ebsdtorch.s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle

    out = {}
    cases = [
        dict(det=(16, 16), b=1, seed=41, pc=(0.5625, 0.4375, 0.5), x=(0.4, 0.6), y=(0.4, 0.6), z=(0.4, 0.6, 5),
             tilt=70.0, sec=0.0, res=10.0, bs=1024, n=3),
        dict(det=(24, 20), b=2, seed=42, pc=(0.4, 0.5833333, 0.55), x=(0.3, 0.75), y=(0.35, 0.65),
             z=(0.45, 0.75, 4), tilt=70.0, sec=0.0, res=12.0, bs=16, n=2),
        dict(det=(20, 20), b=1, seed=43, pc=(0.55, 0.5, 0.62), x=(0.4, 0.6), y=(0.45, 0.65), z=(0.5, 0.7, 3),
             tilt=65.0, sec=5.0, res=12.0, bs=1024, n=2),
    ]
    for ci, c in enumerate(cases):
        mp_t = smooth_master_pattern(c["seed"], 41)
        mp = MasterPattern(mp_t.clone(), laue_group=11)
        H, W = c["det"]
        # patterns simulated with the fitter's own helpers at the true PC
        torch.manual_seed(c["seed"])
        dict_q = sample_ori_fz_laue_angle(laue_id=11, angular_resolution_deg=c["res"], device=torch.device("cpu"))
        truth_idx = torch.randint(0, dict_q.shape[0], (c["n"],))
        rot, tr = F.bruker_geometries_to_SE3(torch.tensor([list(c["pc"])]), torch.tensor(-c["tilt"]),
                                             torch.tensor(c["sec"]), (H, W))
        pix = F.get_3D_pixel_coords((H, W), torch.device("cpu"))
        with torch.no_grad():
            coords = F.generate_dictionary_coords(pix, dict_q[truth_idx], rot, tr)
            pats = mp.interpolate(coords, normalize_coords=False).view(c["n"], 1, H, W)
            pats = pats + 0.02 * torch.randn(pats.shape, generator=torch.Generator().manual_seed(c["seed"]))
        kw = dict(pc_x_min=c["x"][0], pc_x_max=c["x"][1], pc_y_min=c["y"][0], pc_y_max=c["y"][1],
                  pc_z_min=c["z"][0], pc_z_max=c["z"][1], pc_z_steps=c["z"][2], primary_tilt_deg=c["tilt"],
                  secondary_tilt_deg=c["sec"], dictionary_resolution_deg=c["res"],
                  dictionary_indexing_batch_size=c["bs"], virtual_binning=c["b"], metric="dot")
        torch.manual_seed(1000 + ci)  # fixes the dictionary permutation inside the fitter
        with contextlib.redirect_stdout(io.StringIO()), contextlib.redirect_stderr(io.StringIO()):
            best_pc, best_q = F.spatial_fft_pc_fitter(MasterPattern(mp_t.clone(), laue_group=11), pats.clone(), **kw)
        torch.manual_seed(1000 + ci)
        fit_dict = sample_ori_fz_laue_angle(laue_id=11, angular_resolution_deg=c["res"], device=torch.device("cpu"))
        pp, padding, shape = F.get_3D_pixel_coords_with_periphery(
            (H, W), torch.device("cpu"), c["x"][0], c["x"][1], c["y"][0], c["y"][1], c["b"])
        r0, t0 = F.bruker_geometries_to_SE3(torch.tensor([[0.5, 0.5, c["z"][0]]]), torch.tensor(-c["tilt"]),
                                            torch.tensor(c["sec"]), (H, W))
        with torch.no_grad():
            mpb = MasterPattern(mp_t.clone(), laue_group=11)
            sims = mpb.interpolate(F.generate_dictionary_coords(pp, fit_dict[:4], r0, t0), mode="bilinear",
                                   align_corners=False, normalize_coords=False, virtual_binning=c["b"])
        out[f"case{ci}_master_pattern"] = mp_t.numpy()
        out[f"case{ci}_patterns"] = pats.numpy()
        out[f"case{ci}_dictionary"] = fit_dict.numpy()
        out[f"case{ci}_best_pc"] = best_pc.numpy()
        out[f"case{ci}_best_quats"] = best_q.numpy()
        out[f"case{ci}_pixel_coords"] = pp.numpy()
        out[f"case{ci}_padding"] = np.array([*padding, *shape], dtype=np.int64)
        out[f"case{ci}_sims"] = sims.reshape(4, *shape).numpy()
        out[f"case{ci}_meta"] = np.array([H, W, c["b"], *c["x"], *c["y"], c["z"][0], c["z"][1], c["z"][2],
                                          c["tilt"], c["sec"], c["res"], c["bs"], 1000 + ci], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "pcfit.npz"), **out)


def emsoft_reader_goldens(root=None):
    """EMsoft master-pattern reader (io/read_master_pattern.py:7-53). h5py is
    absent, so the reference's read_master_pattern runs on an in-memory
    stand-in of h5py.File serving seeded arrays with EMsoft's dataset names
    and layouts: accum_e (H, W, n_energies), mLPNH / mLPSH (1, n_energies, H,
    W), SpaceGroupNumber (1,). Cases: 5 energies / m-3m (225), 1 energy
    (the squeeze edge) / 6/mmm (194), 7 energies / mmm (62)."""
    ref_loader.import_reference(root)
    files = {}

    class _File:
        def __init__(self, path, mode="r"):
            self.data = files[path]

        def __enter__(self):
            return self.data

        def __exit__(self, *a):
            return False

    fake = types.ModuleType("h5py")
    fake.File = _File
    sys.modules["h5py"] = fake
    from ebsdtorch.io.read_master_pattern import read_master_pattern

    out = {}
    for ci, (n_e, h, sg) in enumerate(((5, 33, 225), (1, 17, 194), (7, 25, 62))):
        g = torch.Generator().manual_seed(300 + ci)
        arrays = {
            "EMData/MCOpenCL/accum_e": (torch.rand((h + 8, h + 8, n_e), generator=g) * 1000).round().numpy()
                                       .astype(np.int32),
            "EMData/EBSDmaster/mLPNH": torch.rand((1, n_e, h, h), generator=g).numpy().astype(np.float32),
            "EMData/EBSDmaster/mLPSH": torch.rand((1, n_e, h, h), generator=g).numpy().astype(np.float32),
            "CrystalData/SpaceGroupNumber": np.array([sg], dtype=np.int32),
        }
        files[f"case{ci}.h5"] = arrays
        mp = read_master_pattern(f"case{ci}.h5")
        for k, v in arrays.items():
            out[f"case{ci}/{k}"] = v
        out[f"case{ci}_master_pattern"] = mp.master_pattern.numpy()
        out[f"case{ci}_laue_group"] = np.array([mp.laue_group], dtype=np.int64)
    del sys.modules["h5py"]
    np.savez_compressed(os.path.join(HERE, "emsoft_reader.npz"), **out)


def config0_goldens(root=None):
    """The reference's own plain DI at the small configuration (60 x 60 px,
    m-3m 1.0 deg dictionary of 36,829 rows, 4,096 patterns, top-4, float32
    matching, chunked over both axes) on the inputs of config0_inputs.py.
    Commits the seeds, the inputs' checksums and the results: per pattern the
    top-4 dictionary indices (into the permuted dictionary) and metrics."""
    import config0_inputs as C

    ref_idx, _ = load_reference(root)
    from ebsdtorch.ebsd.experiment_pats import ExperimentPatterns
    from ebsdtorch.ebsd.geometry import EBSDGeometry
    from ebsdtorch.ebsd.master_pattern import MasterPattern
    from ebsdtorch.s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle

    c = C.CASE
    inp = C.make_inputs(c)
    mp = MasterPattern(torch.from_numpy(inp["master_pattern"]).clone(), laue_group=11)
    geom = EBSDGeometry(c["det"], tilts_degrees=c["tilts"], proj_center=c["pc"])
    exp = ExperimentPatterns(torch.from_numpy(inp["counts"].astype(np.float32)))
    torch.manual_seed(c["perm_seed"])
    with ref_loader.quiet_stdout():
        ref_idx.dictionary_index_orientations(
            mp, geom, exp, dictionary_resolution_degrees=c["res"], top_k_matches=c["k"],
            dictionary_chunk_size=c["dictionary_chunk_size"], experiment_chunk_size=c["experiment_chunk_size"],
            match_dtype=torch.float32, quantized_if_x86=False)
    quats_k, metrics_k = exp.raw_indexing_results[0]
    torch.manual_seed(c["perm_seed"])
    dictionary = sample_ori_fz_laue_angle(11, c["res"], torch.device("cpu"), permute=True).numpy()
    lookup = {row.tobytes(): i for i, row in enumerate(dictionary)}
    q = quats_k.numpy()
    idx = np.array([[lookup[q[i, j].tobytes()] for j in range(q.shape[1])] for i in range(q.shape[0])],
                   dtype=np.int32)
    np.savez_compressed(
        os.path.join(HERE, "config0.npz"),
        indices=idx, metrics=metrics_k.numpy().astype(np.float32),
        n_dictionary=np.array([dictionary.shape[0]]),
        sha256_master_pattern=np.array(inp["sha256_master_pattern"]),
        sha256_counts=np.array(inp["sha256_counts"]),
        case=np.array(repr(sorted(c.items()))))


PCA_CONFIG0 = dict(n_components=256, learn_res=2.0)


def pca_config0_goldens(root=None):
    """The reference's own PCA DI at the small configuration: the inputs of
    config0_inputs.py, the 256 leading components (indexing.py:355 with the
    "top" slice) learned on the m-3m 2.0 deg dictionary (4,344 rows),
    indexing the 1.0 deg dictionary (36,829 rows), top-4, FP32 matching.
    Commits the per-pattern top-4 indices (into the permuted index
    dictionary) and metrics."""
    import config0_inputs as C

    _, ref_top = load_reference(root)
    from ebsdtorch.ebsd.experiment_pats import ExperimentPatterns
    from ebsdtorch.ebsd.geometry import EBSDGeometry
    from ebsdtorch.ebsd.master_pattern import MasterPattern
    from ebsdtorch.s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle

    c, pc = C.CASE, PCA_CONFIG0
    inp = C.make_inputs(c)
    mp = MasterPattern(torch.from_numpy(inp["master_pattern"]).clone(), laue_group=11)
    geom = EBSDGeometry(c["det"], tilts_degrees=c["tilts"], proj_center=c["pc"])
    exp = ExperimentPatterns(torch.from_numpy(inp["counts"].astype(np.float32)))
    torch.manual_seed(c["perm_seed"])
    with ref_loader.quiet_stdout():
        ref_top.pca_dictionary_index_orientations(
            mp, geom, exp, n_pca_components=pc["n_components"], dictionary_resolution_learn_deg=pc["learn_res"],
            dictionary_resolution_index_deg=c["res"], top_k_matches=c["k"],
            dictionary_chunk_size=c["dictionary_chunk_size"], experiment_chunk_size=c["experiment_chunk_size"],
            match_dtype=torch.float32, quantized_via_ao=False)
    quats_k, metrics_k = exp.raw_indexing_results[0]
    # the same draws: the learning dictionary's permutation, then the index dictionary's
    torch.manual_seed(c["perm_seed"])
    sample_ori_fz_laue_angle(11, pc["learn_res"], torch.device("cpu"), permute=True)
    dictionary = sample_ori_fz_laue_angle(11, c["res"], torch.device("cpu"), permute=True).numpy()
    lookup = {row.tobytes(): i for i, row in enumerate(dictionary)}
    q = quats_k.numpy()
    idx = np.array([[lookup[q[i, j].tobytes()] for j in range(q.shape[1])] for i in range(q.shape[0])],
                   dtype=np.int32)
    np.savez_compressed(
        os.path.join(HERE, "pca_config0.npz"),
        indices=idx, metrics=metrics_k.numpy().astype(np.float32),
        n_dictionary=np.array([dictionary.shape[0]]), n_components=np.array([pc["n_components"]]),
        learn_res=np.array([pc["learn_res"]]),
        sha256_master_pattern=np.array(inp["sha256_master_pattern"]),
        sha256_counts=np.array(inp["sha256_counts"]),
        case=np.array(repr(sorted(c.items()))))


def euclidean_goldens(root=None):
    """The reference's plain DI with distance_metric="euclidean" (knn.py:85-91,
    squared distance of the zero-mean rows) and "manhattan" (:92-93, L1
    distance), smallest first, float32 matching: per metric one case on its
    chunked query path (top-3) and one with a signal mask and binning 2 on
    the all-at-once path (top-2)."""
    ref_idx, _ = load_reference(root)
    from ebsdtorch.ebsd.experiment_pats import ExperimentPatterns
    from ebsdtorch.ebsd.geometry import EBSDGeometry
    from ebsdtorch.ebsd.master_pattern import MasterPattern
    from ebsdtorch.preprocessing.radial_mask import get_radial_mask
    from ebsdtorch.s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle
    from ebsdtorch.s2_and_so3.quaternions import qu_apply
    from ebsdtorch.s2_and_so3.sampling import so3_uniform_quat

    out = {}
    for ci, c in enumerate((dict(det=(20, 20), res=8.0, Q=31, k=3, b=1, mask=False, ec=8, dcs=50, seed=91,
                                 metric="euclidean"),
                            dict(det=(24, 24), res=9.0, Q=19, k=2, b=2, mask=True, ec=4096, dcs=4096, seed=92,
                                 metric="euclidean"),
                            dict(det=(20, 20), res=8.0, Q=23, k=3, b=1, mask=False, ec=8, dcs=50, seed=93,
                                 metric="manhattan"),
                            dict(det=(24, 24), res=9.0, Q=17, k=2, b=2, mask=True, ec=4096, dcs=4096, seed=94,
                                 metric="manhattan"))):
        torch.manual_seed(c["seed"])
        mp_t = smooth_master_pattern(c["seed"], 41)
        mp = MasterPattern(mp_t.clone(), laue_group=11)
        geom = EBSDGeometry(c["det"], tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
        qq = so3_uniform_quat(c["Q"], torch.device("cpu"))
        with torch.no_grad():
            dc = geom.get_coords_sample_frame(binning=(1, 1))
            dc = dc / dc.norm(dim=-1, keepdim=True)
            pats = mp.interpolate(qu_apply(qq[:, None, :], dc[None]), normalize_coords=False).reshape(
                c["Q"], *c["det"])
            pats = 50.0 * (pats + 0.05 * torch.randn_like(pats))
        exp = ExperimentPatterns(pats.clone())
        bdet = (c["det"][0] // c["b"], c["det"][1] // c["b"])
        mask = get_radial_mask(bdet) if c["mask"] else None
        torch.manual_seed(c["seed"] + 1000)
        with ref_loader.quiet_stdout():
            ref_idx.dictionary_index_orientations(
                mp, geom, exp, signal_mask=mask, experiment_chunk_size=c["ec"],
                dictionary_resolution_degrees=c["res"], dictionary_chunk_size=c["dcs"], virtual_binning=c["b"],
                top_k_matches=c["k"], distance_metric=c["metric"], match_dtype=torch.float32,
                quantized_if_x86=False)
        torch.manual_seed(c["seed"] + 1000)
        dictionary = sample_ori_fz_laue_angle(11, c["res"], torch.device("cpu"), permute=True).numpy()
        out[f"case{ci}_master_pattern"] = mp_t.numpy()
        out[f"case{ci}_patterns"] = pats.numpy()
        out[f"case{ci}_mask"] = mask.numpy() if mask is not None else np.zeros(0, bool)
        out[f"case{ci}_meta"] = np.array([*c["det"], c["res"], c["Q"], c["k"], c["b"], c["ec"], c["dcs"],
                                          c["seed"] + 1000], dtype=np.float64)
        out[f"case{ci}_metric"] = np.array(c["metric"])
        out[f"case{ci}_quats"] = exp.raw_indexing_results[0][0].numpy()
        out[f"case{ci}_dists"] = exp.raw_indexing_results[0][1].numpy()
        out[f"case{ci}_best"] = exp.best_metrics.numpy()
        out[f"case{ci}_dictionary"] = dictionary
    np.savez_compressed(os.path.join(HERE, "di_euclid.npz"), **out)


def main(root=None):
    ref_idx, ref_idx_top = load_reference(root)
    from ebsdtorch.s2_and_so3.laue_fz_ori import sample_ori_fz_laue_angle
    from ebsdtorch.s2_and_so3.orientations import cu2qu, qu2cu
    from ebsdtorch.s2_and_so3.sphere import rosca_lambert_side_by_side
    from ebsdtorch.s2_and_so3.sampling import so3_uniform_quat
    from ebsdtorch.s2_and_so3.laue_fz_misori import disori_angle_laue
    from ebsdtorch.ebsd.geometry import EBSDGeometry
    from ebsdtorch.ebsd.master_pattern import MasterPattern
    from ebsdtorch.ebsd.experiment_pats import ExperimentPatterns
    from ebsdtorch.utils.pca_covmat import OnlineCovMatrix
    from ebsdtorch.preprocessing.radial_mask import get_radial_mask

    cpu = torch.device("cpu")
    out = {}

    # ---- A1/A2: FZ grids for all 11 Laue groups (unpermuted) ----
    grids = {}
    for laue in range(1, 12):
        for res in (15.0, 7.5):
            q = sample_ori_fz_laue_angle(laue, res, cpu, permute=False)
            grids[f"q_{laue}_{res}"] = q.numpy()
    # counts of the config-sized dictionaries
    counts = []
    for laue, res in ((11, 1.0), (11, 0.9), (11, 0.5), (9, 0.6), (5, 0.9), (10, 2.0), (7, 2.0), (3, 3.0)):
        q = sample_ori_fz_laue_angle(laue, res, cpu, permute=False)
        counts.append((laue, res, q.shape[0]))
        if (laue, res) == (11, 1.0):
            grids["q_11_1.0"] = q.numpy()
    grids["counts"] = np.array(counts, dtype=np.float64)
    # permutation convention: one randperm(n) on the global CPU generator
    torch.manual_seed(1234)
    q_perm = sample_ori_fz_laue_angle(11, 7.5, cpu, permute=True)
    grids["q_11_7.5_perm_seed1234"] = q_perm.numpy()
    np.savez_compressed(os.path.join(HERE, "grid.npz"), **grids)

    # ---- cu2qu / qu2cu ----
    g = torch.Generator().manual_seed(7)
    a = 0.5 * np.pi ** (2 / 3)
    cu = (torch.rand((4000, 3), generator=g) * 2 - 1) * a
    np.savez_compressed(os.path.join(HERE, "cu2qu.npz"), cu=cu.numpy(), qu=cu2qu(cu).numpy(),
                        cu64=cu.double().numpy(), qu64=cu2qu(cu.double()).numpy())

    # ---- A3: detector rays ----
    rays = {}
    for name, shape, pc, tilts, b in (
        ("d60", (60, 60), (0.5, 0.5, 0.6), (0.0, 70.0, 0.0), 1),
        ("d60b2", (60, 60), (0.5, 0.5, 0.6), (0.0, 70.0, 0.0), 2),
        ("d5", (5, 5), (0.4221, 0.2179, 0.4954), (0.0, 70.0, 0.0), 1),
        ("d40x32", (40, 32), (0.45, 0.55, 0.7), (3.0, 68.0, 5.0), 1),
        ("d128", (128, 128), (0.5, 0.5, 0.6), (0.0, 70.0, 0.0), 1),
    ):
        geom = EBSDGeometry(shape, tilts_degrees=tilts, proj_center=pc)
        with torch.no_grad():
            r = geom.get_coords_sample_frame(binning=(b, b))
        rays[name] = r.numpy()
        rays[name + "_meta"] = np.array([shape[0], shape[1], *pc, *tilts, b], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "rays.npz"), **rays)

    # ---- A5: Lambert side-by-side ----
    g = torch.Generator().manual_seed(11)
    v = torch.randn((5000, 3), generator=g)
    v = v / v.norm(dim=-1, keepdim=True)
    special = torch.tensor([[0, 0, 1.0], [0, 0, -1.0], [1.0, 0, 0], [0, 1.0, 0], [-1.0, 0, 0], [0, -1.0, 0],
                            [0.6, 0.8, 0.0], [0.6, -0.8, 0.0], [-0.7071, 0.7071, 0.0]])
    v = torch.cat((v, special))
    np.savez_compressed(os.path.join(HERE, "lambert.npz"), xyz=v.numpy(), uv=rosca_lambert_side_by_side(v).numpy())

    # ---- A4-A7: projector ----
    proj = {}
    torch.manual_seed(3)
    mp_t = smooth_master_pattern(5, 33)
    mp = MasterPattern(mp_t, laue_group=11)
    quats = so3_uniform_quat(64, cpu)
    quats = torch.where(quats[:, :1] >= 0, quats, -quats)
    for b in (1, 2):
        geom = EBSDGeometry((16, 16), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.45, 0.6))
        with torch.no_grad():
            dc = geom.get_coords_sample_frame(binning=(b, b))
            dc = dc / dc.norm(dim=-1, keepdim=True)
            rot = __import__("ebsdtorch.s2_and_so3.quaternions", fromlist=["qu_apply"]).qu_apply(
                quats[:, None, :], dc[None])
            sims = mp.interpolate(rot, mode="bilinear", align_corners=False, normalize_coords=False,
                                  virtual_binning=b).squeeze()
        mp.master_pattern_binned = None
        proj[f"sims_b{b}"] = sims.reshape(64, -1).numpy()
        proj[f"rays_b{b}"] = dc.numpy()
    proj["master_pattern"] = mp_t.numpy()
    proj["quats"] = quats.numpy()
    np.savez_compressed(os.path.join(HERE, "projector.npz"), **proj)

    # ---- A1-A13: end-to-end plain DI ----
    def make_queries(mp_obj, geom, n, seed, b=1):
        torch.manual_seed(seed)
        qq = so3_uniform_quat(n, cpu)
        with torch.no_grad():
            dc = geom.get_coords_sample_frame(binning=(1, 1))
            dc = dc / dc.norm(dim=-1, keepdim=True)
            from ebsdtorch.s2_and_so3.quaternions import qu_apply
            pats = mp_obj.interpolate(qu_apply(qq[:, None, :], dc[None]), normalize_coords=False).reshape(
                n, *geom.detector_shape)
            pats = pats + 0.02 * torch.randn_like(pats)
        return qq, pats

    cases = [
        dict(name="di_a", det=(16, 16), pc=(0.5, 0.5, 0.6), res=10.0, Q=24, k=3, mask=False, b=1,
             ec=4096, dcs=4096, seed=21),
        dict(name="di_b", det=(20, 20), pc=(0.45, 0.55, 0.62), res=12.0, Q=17, k=4, mask=True, b=2,
             ec=5, dcs=7, seed=22),
        dict(name="di_c", det=(12, 16), pc=(0.5, 0.5, 0.55), res=15.0, Q=9, k=1, mask=False, b=1,
             ec=4, dcs=16, seed=23),
    ]
    for c in cases:
        torch.manual_seed(c["seed"])
        mp_t = smooth_master_pattern(c["seed"], 41)
        mp = MasterPattern(mp_t.clone(), laue_group=11)
        geom = EBSDGeometry(c["det"], tilts_degrees=(0.0, 70.0, 0.0), proj_center=c["pc"])
        qq, pats = make_queries(mp, geom, c["Q"], c["seed"] + 100)
        exp = ExperimentPatterns(pats.clone())
        mask = get_radial_mask(tuple(c["det"] if c["b"] == 1 else (c["det"][0] // c["b"], c["det"][1] // c["b"])))\
            if c["mask"] else None
        torch.manual_seed(c["seed"] + 1000)
        with contextlib.redirect_stdout(io.StringIO()):
            ref_idx.dictionary_index_orientations(
                mp, geom, exp, signal_mask=mask, experiment_chunk_size=c["ec"],
                dictionary_resolution_degrees=c["res"], dictionary_chunk_size=c["dcs"], virtual_binning=c["b"],
                top_k_matches=c["k"], match_dtype=torch.float32, quantized_if_x86=False)
        quats_k, metrics_k = exp.raw_indexing_results[0]
        torch.manual_seed(c["seed"] + 1000)
        dict_q = sample_ori_fz_laue_angle(11, c["res"], cpu, permute=True)
        np.savez_compressed(
            os.path.join(HERE, f"{c['name']}.npz"),
            master_pattern=mp_t.numpy(), patterns=pats.numpy(), true_quats=qq.numpy(),
            mask=(mask.numpy() if mask is not None else np.zeros(0, bool)),
            meta=np.array([*c["det"], *c["pc"], c["res"], c["Q"], c["k"], c["b"], c["ec"], c["dcs"],
                           c["seed"] + 1000], dtype=np.float64),
            quats=quats_k.numpy(), metrics=metrics_k.numpy(), orientations=exp.orientations.numpy(),
            best_metrics=exp.best_metrics.numpy(), dictionary=dict_q.numpy(),
        )

    # the reference's own DI test case (tests/test_di.py:9-48), fp32 matching
    torch.manual_seed(0)
    geom = EBSDGeometry(detector_shape=(5, 5), proj_center=(0.4221, 0.2179, 0.4954))
    mp_t = torch.randn((10, 10), dtype=torch.float32)
    pats = torch.randn((2, 5, 5), dtype=torch.float32)
    mp = MasterPattern(mp_t.clone(), laue_group=11)
    exp = ExperimentPatterns(pats.clone())
    torch.manual_seed(99)
    with contextlib.redirect_stdout(io.StringIO()):
        ref_idx.dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=10.0,
                                              dictionary_chunk_size=4096, experiment_chunk_size=4096,
                                              match_dtype=torch.float32, quantized_if_x86=False)
    np.savez_compressed(os.path.join(HERE, "di_reftest.npz"), master_pattern=mp_t.numpy(), patterns=pats.numpy(),
                        quats=exp.raw_indexing_results[0][0].numpy(),
                        metrics=exp.raw_indexing_results[0][1].numpy(), seed=np.array([99]))

    # ---- A11/A12: PCA DI (shipped slice and top slice) ----
    # learn on 5 deg (296 orientations > 256 pixels, full-rank covariance),
    # index on 8 deg; n = 24 (both slices give the top 24 for P < 300) and
    # n = 100 with the shipped slice (components 57-100).
    torch.manual_seed(31)
    mp_t = smooth_master_pattern(31, 41)
    geom = EBSDGeometry((16, 16), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
    mp = MasterPattern(mp_t.clone(), laue_group=11)
    qq, pats = make_queries(mp, geom, 20, 131)
    pca = dict(master_pattern=mp_t.numpy(), patterns=pats.numpy(), true_quats=qq.numpy(),
               meta=np.array([5.0, 8.0, 777], dtype=np.float64))
    for tag, mod, ncomp in (("top", ref_idx_top, 24), ("shipped", ref_idx, 24), ("shipped_n100", ref_idx, 100)):
        exp = ExperimentPatterns(pats.clone())
        torch.manual_seed(777)
        with contextlib.redirect_stdout(io.StringIO()):
            mod.pca_dictionary_index_orientations(
                MasterPattern(mp_t.clone(), laue_group=11), geom, exp, n_pca_components=ncomp,
                dictionary_resolution_learn_deg=5.0, dictionary_resolution_index_deg=8.0,
                dictionary_chunk_size=4096, experiment_chunk_size=4096, top_k_matches=2,
                match_dtype=torch.float32, quantized_via_ao=False)
        pca[f"quats_{tag}"] = exp.raw_indexing_results[0][0].numpy()
        pca[f"metrics_{tag}"] = exp.raw_indexing_results[0][1].numpy()
        pca[f"ncomp_{tag}"] = np.array([ncomp])
    torch.manual_seed(777)
    pca["learn_dictionary"] = sample_ori_fz_laue_angle(11, 5.0, cpu, permute=True).numpy()
    pca["dictionary"] = sample_ori_fz_laue_angle(11, 8.0, cpu, permute=True).numpy()
    np.savez_compressed(os.path.join(HERE, "pca_di.npz"), **pca)

    # ---- A11: covariance ----
    g = torch.Generator().manual_seed(41)
    x = torch.randn((300, 24), generator=g) @ torch.randn((24, 24), generator=g) + 3.0
    cov = OnlineCovMatrix(24)
    for chunk in torch.split(x, 64):
        cov(chunk)
    np.savez_compressed(os.path.join(HERE, "covariance.npz"), x=x.numpy(), cov=cov.get_covmat().numpy())

    # ---- A15: 6-D (Zhou) rotation representation ----
    from ebsdtorch.s2_and_so3.orientations import zh2om, zh2qu, qu2zh, om2qu, qu2om
    g = torch.Generator().manual_seed(61)
    zh = torch.randn((3000, 6), generator=g, dtype=torch.float64)
    qr = so3_uniform_quat(3000, cpu, dtype=torch.float64)
    qr = torch.where(qr[:, :1] >= 0, qr, -qr)
    np.savez_compressed(os.path.join(HERE, "rot6d.npz"), zh=zh.numpy(), om=zh2om(zh).numpy(), qu=zh2qu(zh).numpy(),
                        qu_in=qr.numpy(), zh_out=qu2zh(qr).numpy(), om_out=qu2om(qr).numpy(),
                        qu_back=om2qu(qu2om(qr)).numpy())

    # ---- A14: disorientation ----
    dis = {}
    torch.manual_seed(51)
    for laue in (11, 9, 5, 3, 1):
        q1 = so3_uniform_quat(500, cpu, dtype=torch.float64)
        q2 = so3_uniform_quat(500, cpu, dtype=torch.float64)
        dis[f"q1_{laue}"] = q1.numpy()
        dis[f"q2_{laue}"] = q2.numpy()
        dis[f"ang_{laue}"] = disori_angle_laue(q1, q2, laue, laue).numpy()
    np.savez_compressed(os.path.join(HERE, "disori.npz"), **dis)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    args = sys.argv[1:]
    if args and args[0] == "--refinement-only":
        refinement_goldens(*args[1:])
    elif args and args[0] == "--preprocessing-only":
        preprocessing_goldens(*args[1:])
    elif args and args[0] == "--pcfit-only":
        pcfit_goldens(*args[1:])
    elif args and args[0] == "--reader-only":
        emsoft_reader_goldens(*args[1:])
    elif args and args[0] == "--config0-only":
        config0_goldens(*args[1:])
    elif args and args[0] == "--euclidean-only":
        euclidean_goldens(*args[1:])
    elif args and args[0] == "--pca-config0-only":
        pca_config0_goldens(*args[1:])
    else:
        main(*args)
        refinement_goldens(*args)
        preprocessing_goldens(*args)
        pcfit_goldens(*args)
        emsoft_reader_goldens(*args)
        config0_goldens(*args)
        euclidean_goldens(*args)
