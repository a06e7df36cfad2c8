"""Parity on the 512x512x320 workload (shrink 2: a 256x256x160 fitting grid,
10.5 M fitting voxels, final lattice 11x11x11), which runs on the whole-GPU
path.  Every control point of the last level sums over about 5e5 fitting
voxels (N4.py:229-237), the longest FP32 sums of any workload here, so this
is where accumulated round-off would show first.

Tolerance: 1e-4 relative (max|gpu - ref| / max|ref|) for the lattice, the
full-resolution log bias field and the corrected volume, against the FP64
oracle at a fixed iteration count.
"""
import numpy as np
import pytest

import n4_oracle as O
from n4b200.phantom import make_phantom

pytestmark = pytest.mark.gpu
TOL = 1e-4


def nrel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return float(np.abs(a.astype(np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.fixture(scope="module")
def c3_phantom():
    return make_phantom((512, 512, 320), seed=3, sigma=0.02, grid=8, coeff_std=0.25)


def test_c3_whole_gpu_path_fixed_iterations(cuda, c3_phantom):
    import n4b200
    ph = c3_phantom
    its = [3, 3, 3, 3]
    p = n4b200.N4Param(NumberOfFittingLevels=4, MaximumNumberOfIterations=its, ConvergenceThreshold=0.0,
                       low_value=0.0, ShrinkFactor=2)
    im, mk = cuda.tensor(ph.im, device="cuda"), cuda.tensor(ph.mask, device="cuda")
    res = n4b200.N4(im, mk, p, return_bias=True)
    assert res.report["status"] == "N4_OK"
    assert res.report["path"] == "grid"
    assert res.report["iterations"][:4] == its
    out, lat, lb = O.N4Shrink(ph.im, ph.mask, 2, low_value=0, maximumNumberOfLevels=4,
                              maximumNumberOfIterations=its, ConvergenceThreshold=0.0, return_log_bias=True)
    e_lat = nrel(res.lattice, lat)
    e_lb = nrel(np.log(res.bias_field.cpu().numpy()), lb)
    e_out = nrel(res.im_normalized, out)
    print(f"c3 fixed {its}: lattice {e_lat:.3e} log-bias {e_lb:.3e} corrected {e_out:.3e}")
    assert e_lat < TOL and e_lb < TOL and e_out < TOL
