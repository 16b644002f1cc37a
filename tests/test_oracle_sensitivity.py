"""The reference's own results depend on float rounding where the
Gauss-Newton tolerance is below the float spacing of the mapped pixel
coordinates.

Coordinates are floats, so for x in [1024, 2048) they move in steps of
1.2e-4 px, twelve times the 1e-5 tolerance of the 2048^2 sequence workload.
There the last updates of a solve oscillate at that step, and whether a solve
meets the tolerance within its 25 iterations (or falls back to the simplex)
depends on rounding.  The oracle built with one legitimate rounding change,
the mean of the deformed intensities summed in double
(libdiceoracle_meanfp64.so), changes the iteration count of ~2 % of such
subsets and the optimiser path of some; solves that converge in both agree
to far inside 1e-4 px.  GPU-vs-oracle parity is assessed the same way.
"""
import numpy as np

from dice_b200 import abi
from dice_b200 import synthetic as syn
from oracle import oracle as O


def test_reference_rounding_decides_noise_floor_solves():
    w, h = 2048, 128
    ref = syn.speckle_image(w, h, seed=2, r_min=3, r_max=5, grey_lo=1000.0, grey_hi=64000.0, blur_sigma=0.8)
    deff = syn.warp_image(ref, syn.config2_field(5), noise_sigma=50.0, seed=205, clip=(0.0, 65535.0)).numpy()
    ref = ref.numpy()
    cx, cy = syn.grid_points(w, h, 31, 5)
    keep = cx >= 1024
    cx, cy = cx[keep], cy[keep]
    p = abi.default_params(subset_size=31, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1,
                           fast_solver_tolerance=1e-5)
    a = syn.init_fields(cx, cy)
    O.execute_frame(p, ref, deff, a, nthreads=8)
    with O.use_library("libdiceoracle_meanfp64.so"):
        b = syn.init_fields(cx, cy)
        O.execute_frame(p, ref, deff, b, nthreads=8)
    assert np.array_equal(a[:, abi.F_STATUS], b[:, abi.F_STATUS])
    changed = a[:, abi.F_ITERATIONS] != b[:, abi.F_ITERATIONS]
    assert 0.005 < changed.mean() < 0.1
    sa, sb = a[:, abi.F_ITERATIONS] > p.max_solver_iterations_fast, b[:, abi.F_ITERATIONS] > p.max_solver_iterations_fast
    assert (sa != sb).sum() >= 1            # some solves switch to the simplex
    gn = ~sa & ~sb
    assert np.max(np.abs(a[gn, abi.F_DISP_X] - b[gn, abi.F_DISP_X])) < 1e-4
    assert np.max(np.abs(a[gn, abi.F_DISP_Y] - b[gn, abi.F_DISP_Y])) < 1e-4
