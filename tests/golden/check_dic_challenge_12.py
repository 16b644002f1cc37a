"""End-to-end check of the dic_challenge_12 regression on the oracle.

Run in a container that has the DICe reference checked out:

    python tests/golden/check_dic_challenge_12.py /path/to/dice

It runs the regression's own inputs (tests/regression/dic_challenge_12:
subset_file.dat region of interest, step 35, subset 27, Keys-4,
USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY, GRADIENT_BASED_THEN_SIMPLEX, translation
and normal strain, VSG strain over a 360 px window, reference oht_cfrp_00,
frames 01..11) through the oracle, writes the result files with the
library's writer (unsorted, and sorted as dic_challenge_12_sorted asks) and
compares every gold file with DICe_Diff's rule (-t 0.05 -f 5.0E-5).  The
images belong to the DIC Challenge and are read in place, never copied;
nothing here is a fixture.  Prints the failed-line count per gold file and
exits non-zero if any file fails.
"""
import os
import sys
import tempfile

import numpy as np
from PIL import Image

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from dice_b200 import abi, synthetic as syn  # noqa: E402
from dice_b200.results import Output, diff_text  # noqa: E402
from dice_b200.subset_file import SubsetFile, regular_grid  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main(root):
    reg = os.path.join(root, "tests", "regression")
    src = os.path.join(reg, "dic_challenge_12")

    def img(k):
        return np.asarray(Image.open(os.path.join(src, "images", "oht_cfrp_%02d.tiff" % k)).convert("L"), np.float32)

    ref = img(0)
    h, w = ref.shape
    with open(os.path.join(src, "subset_file.dat")) as fh:
        sf = SubsetFile(text=fh.read())
    xy, neigh, _ = regular_grid(sf, w, h, 35, 27)
    p = abi.default_params(subset_size=27, interpolation=abi.KEYS_FOURTH,
                           initialization_method=abi.USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY,
                           optimization=abi.GRADIENT_BASED_THEN_SIMPLEX, enable_rotation=0, enable_normal_strain=1,
                           enable_shear_strain=0)
    cols = ["COORDINATE_X", "COORDINATE_Y", "DISPLACEMENT_X", "DISPLACEMENT_Y", "VSG_STRAIN_XX", "VSG_STRAIN_YY",
            "GAMMA", "MATCH"]
    variants = {"dic_challenge_12": False, "dic_challenge_12_sorted": True}
    out = {v: Output(p, fields=cols, delimiter=",", omit_row_id=True, ref_image="./images/oht_cfrp_00.tiff",
                     step_size=(35, 35), strain_window=360, sort_rows=s,
                     initialization_method="USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY") for v, s in variants.items()}
    tmp = tempfile.mkdtemp()
    f = syn.init_fields(xy[:, 0], xy[:, 1])
    for k in range(1, 12):
        O.execute_frame(p, ref, img(k), f, first_frame=(k == 1), neighbors=neigh)
        vsg = np.zeros((len(f), abi.VSG_STRIDE))
        vsg[:, :7], failed = O.vsg_strain(f, 360)
        g = f.copy()
        g[failed == 1, abi.F_MATCH] = -1.0
        for v, o in out.items():
            o.set_images(def_image="./images/oht_cfrp_%02d.tiff" % k)
            d = os.path.join(tmp, v)
            os.makedirs(d, exist_ok=True)
            o.write_frame(d + "/", "DICe_solution", k, g, vsg=vsg, first_frame=0, num_frames=11,
                          separate_files=False)
    bad = 0
    for v in variants:
        for k in (1, 6, 11):
            with open(os.path.join(reg, v, "gold", "DICe_solution_%02d.txt" % k)) as fh:
                gold = fh.read()
            with open(os.path.join(tmp, v, "DICe_solution_%02d.txt" % k)) as fh:
                got = fh.read()
            n, _ = diff_text(gold, got, tol=0.05, floor=5.0e-5)
            print("%s frame %02d: %d failed lines" % (v, k, n))
            bad += n
    return 1 if bad else 0


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/check_dic_challenge_12.py <path to the DICe source tree>")
    sys.exit(main(sys.argv[1]))
