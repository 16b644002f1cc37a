"""Shared bar of the GPU-vs-oracle tests: equality of result columns.

The library computes the reference's float operations in the reference's
order, so every column a correlation writes equals the oracle's bit for bit.
"""
import numpy as np

from dice_b200 import abi

# every column a correlation writes
RESULT_COLS = [abi.F_DISP_X, abi.F_DISP_Y, abi.F_ROT_Z, abi.F_STRETCH_XX, abi.F_STRETCH_YY, abi.F_SHEAR_XY] + \
              [abi.F_QUAD_A + i for i in range(12)] + \
              [abi.F_SIGMA, abi.F_GAMMA, abi.F_BETA, abi.F_NOISE, abi.F_CONTRAST, abi.F_ACTIVE_PIXELS,
               abi.F_STATUS, abi.F_ITERATIONS, abi.F_MATCH, abi.F_CONDITION]


def assert_rows_equal(g, o, rows=None, cols=RESULT_COLS):
    """Every listed column equal, bit for bit (NaN equal to NaN)."""
    g = np.asarray(g)
    o = np.asarray(o)
    if rows is not None:
        g, o = g[rows], o[rows]
    for col in cols:
        a, b = g[:, col], o[:, col]
        same = (a == b) | (np.isnan(a) & np.isnan(b))
        assert same.all(), "column %d differs at rows %s: %s vs %s" % (
            col, np.where(~same)[0][:8], a[~same][:4], b[~same][:4])
