"""The checking build (-DEBSD_CHECK, `python -m ebsdtorch_b200.build
--check`): the same workloads run through it record no failed device
check. Runs in a child process that loads libebsd_b200_check.so
(EBSD_CHECK_BUILD=1)."""

import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK_LIB = os.path.join(ROOT, "ebsdtorch_b200", "_lib", "libebsd_b200_check.so")

CHILD = r"""
import sys, torch
sys.path.insert(0, sys.argv[1])
from ebsdtorch_b200 import _capi, synthetic
from ebsdtorch_b200.ebsd import EBSDGeometry, ExperimentPatterns, MasterPattern, dictionary_index_orientations
from ebsdtorch_b200.ebsd import spatial_fft_pc_fitter
assert _capi.LIB_PATH.endswith("libebsd_b200_check.so")
assert _capi.debug_check() == (0, "")
mp_t = synthetic.synthetic_master_pattern(129, seed=1, device="cuda")
mp = MasterPattern(mp_t, laue_group=11)
geom = EBSDGeometry((32, 32), tilts_degrees=(0.0, 70.0, 0.0), proj_center=(0.5, 0.5, 0.6))
q = synthetic.random_quaternions(300, 2).to("cuda")
pats = synthetic.synthetic_patterns(mp_t, geom, q, mean_counts=200.0, seed=3)
exp = ExperimentPatterns(pats)
dictionary_index_orientations(mp, geom, exp, dictionary_resolution_degrees=4.0, top_k_matches=4)
# e4m3 rows, two 128-row query tiles: the two-query-tile match kernel
exp8 = ExperimentPatterns(pats[:256].clone())
dictionary_index_orientations(mp, geom, exp8, dictionary_resolution_degrees=4.0, top_k_matches=4, precision="fp8")
spatial_fft_pc_fitter(mp, pats[:4].reshape(4, 1, 32, 32).clone(), pc_x_min=0.4, pc_x_max=0.6, pc_y_min=0.4,
                      pc_y_max=0.6, pc_z_min=0.55, pc_z_max=0.65, pc_z_steps=2, dictionary_resolution_deg=8.0)
torch.cuda.synchronize()
line, file = _capi.debug_check()
print("check", line, file)
assert line == 0, (line, file)
"""


@pytest.mark.skipif(not os.path.exists(CHECK_LIB), reason="checking build not built (python -m ebsdtorch_b200.build --check)")
def test_workloads_pass_the_device_checks():
    env = dict(os.environ, EBSD_CHECK_BUILD="1")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "check 0" in r.stdout
