"""Pins the CPU oracle to the reference's own regression gold.

Gold files (paths inside the DICe project), converted by
tests/golden/make_fixtures.py:
  tests/regression/parallel_subsets/gold/DICe_solution_0.txt  (49 subsets)
  tests/regression/single_speckled_shift/gold/*.txt            (7 subsets)
Both were produced from 8-bit TIFFs read from files, i.e. reference-gradient
mode (compute_def_gradients = false, DICe_Schema.cpp:185), subset 27,
translation only, KEYS_FOURTH, GRADIENT_BASED_THEN_SIMPLEX, tolerance 1e-4.
The gold prints 5 significant digits; the oracle must reproduce every
iteration count and status flag exactly and u, v, gamma, sigma to the
printed precision plus a small allowance for the reference build's
LAPACK / libm rounding (5e-5 px, 5e-5 relative).
"""
import numpy as np

from dice_b200 import abi
from oracle import oracle as O


def _params():
    return abi.default_params(subset_size=27, use_def_gradients=0)


def test_parallel_subsets_gold(gold):
    ref = gold["ref_speckled"].astype(np.float32)
    de = gold["def_speckled"].astype(np.float32)
    g = gold["parallel_subsets_gold"]
    f = np.zeros((g.shape[0], abi.FIELD_STRIDE))
    f[:, abi.F_COORD_X] = g[:, 1]
    f[:, abi.F_COORD_Y] = g[:, 2]
    O.execute_frame(_params(), ref, de, f, first_frame=True)
    assert np.all(f[:, abi.F_ITERATIONS] == g[:, 9])
    assert np.all(f[:, abi.F_STATUS] == g[:, 10])
    assert np.max(np.abs(f[:, abi.F_DISP_X] - g[:, 3])) < 5e-5
    assert np.max(np.abs(f[:, abi.F_DISP_Y] - g[:, 4])) < 5e-5
    assert np.max(np.abs(f[:, abi.F_GAMMA] - g[:, 8]) / g[:, 8]) < 5e-5


def test_single_speckled_shift_gold(gold):
    ref = gold["ref_speckled"].astype(np.float32)
    de = gold["def_speckled"].astype(np.float32)
    s = gold["single_speckled_shift_gold"]
    f = np.zeros((s.shape[0], abi.FIELD_STRIDE))
    f[:, abi.F_COORD_X] = s[:, 1]
    f[:, abi.F_COORD_Y] = s[:, 2]
    O.execute_frame(_params(), ref, de, f, first_frame=True)
    assert np.all(f[:, abi.F_STATUS] == s[:, 10])
    assert np.max(np.abs(f[:, abi.F_DISP_X] - s[:, 3])) < 5e-5
    assert np.max(np.abs(f[:, abi.F_DISP_Y] - s[:, 4])) < 5e-5
    assert np.max(np.abs(f[:, abi.F_SIGMA] - s[:, 9]) / s[:, 9]) < 5e-5


def test_oracle_threads_match_serial(gold):
    """Splitting subsets over workers (the MPI-split analogue) changes nothing."""
    ref = gold["ref_speckled"].astype(np.float32)
    de = gold["def_speckled"].astype(np.float32)
    g = gold["parallel_subsets_gold"]
    f1 = np.zeros((g.shape[0], abi.FIELD_STRIDE))
    f1[:, 0] = g[:, 1]
    f1[:, 1] = g[:, 2]
    f2 = f1.copy()
    O.execute_frame(_params(), ref, de, f1, nthreads=1)
    O.execute_frame(_params(), ref, de, f2, nthreads=4)
    assert np.array_equal(f1, f2)
