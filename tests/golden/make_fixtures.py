"""Generates the committed golden fixtures from the DICe reference tree.

Run in a container that has the reference checked out (read-only is fine):

    python tests/golden/make_fixtures.py /path/to/dice

It converts the 8-bit test images the reference's regression and component
tests use (OpenCV IMREAD_GRAYSCALE reads them as 8-bit grey, DICe_ImageIO.cpp:454;
Pillow's "L" mode gives the same values) and parses the reference's gold
output files into `reference_gold.npz`.  Nothing at test time reads the
reference tree; the tests only read the .npz written here.

Sources (paths inside the DICe project):
  tests/component/images/refSpeckled.tif, defSpeckled.tif          (512 x 512)
  tests/component/images/refSyntheticSpeckled.tif,
      defSyntheticSpeckled0..5.tif                                (100 x 100)
  tests/regression/parallel_subsets/{input,params}.xml + gold/DICe_solution_0.txt
  tests/regression/single_speckled_shift/{input,params}.xml, subsets.dat,
      gold/single_speckled_shift_{0..6}.txt
  tests/component/images/ImageB.tif, outFilter{5,7,9,11,13}.rawi  (240 x 161)
  tests/component/images/conformal.rawi                            (60 x 56)
  tests/regression/conformal_subset_def/{subset_defs.txt, gold/DICe_solution_{0..4}.txt}
  tests/regression/simple_obstruction/{subsets.txt, images/Img_{00..36}.tif,
      gold/DICe_solution_0.txt}
  tests/regression/dic_challenge_12{,_sorted}/{subset_file.dat, gold/DICe_solution_{01,06,11}.txt}
  tests/examples/{mechanism, obstruction}/subsets.txt,
      tests/regression/mechanism_{skip_solves, optical_flow}/subsets.txt
  tests/examples/obstruction/{images/obstruction_{01..12}.tif,
      gold/DICe_solution_{0,1}.txt}                                (200 x 200)
  tests/regression/{parallel_seed_first_step_only, parallel_subsets_seed}/
      {subset_file.dat, gold/DICe_solution_*.txt}
  tests/regression/incremental/gold/DICe_solution_{0..5}.txt
  tests/regression/bitmap_star/{images/DIC_Challenge_Wave_*_Noisy.bmp,
      gold/DICe_solution_0.txt}                                   (2000 x 501)
"""
import os
import sys

import numpy as np


def _img(root, name):
    from PIL import Image
    im = Image.open(os.path.join(root, "tests", "component", "images", name))
    if im.mode != "L":
        im = im.convert("L")
    return np.asarray(im, dtype=np.uint8)


def _rows(path):
    rows = []
    with open(path) as fh:
        for line in fh:
            line = line.strip()
            if not line or line.startswith("***") or line[0].isalpha():
                continue
            rows.append([float(t) for t in line.split()])
    return np.asarray(rows, dtype=np.float64)


def main(root):
    out = {}
    out["ref_speckled"] = _img(root, "refSpeckled.tif")
    out["def_speckled"] = _img(root, "defSpeckled.tif")
    out["ref_synthetic"] = _img(root, "refSyntheticSpeckled.tif")
    for k in range(6):
        out["def_synthetic_%d" % k] = _img(root, "defSyntheticSpeckled%d.tif" % k)
    # parallel_subsets: subset 27, step 75, translation only, KEYS_FOURTH,
    # GRADIENT_BASED_THEN_SIMPLEX, images read from files (reference-gradient mode).
    # columns: id x y u v exx eyy gxy gamma iterations status
    out["parallel_subsets_gold"] = _rows(os.path.join(
        root, "tests", "regression", "parallel_subsets", "gold", "DICe_solution_0.txt"))
    # single_speckled_shift: 7 hand-placed subsets of size 27, frame 0 rows.
    # columns: frame x y u v theta exx eyy gxy sigma status
    rows = []
    for k in range(7):
        r = _rows(os.path.join(root, "tests", "regression", "single_speckled_shift", "gold",
                               "single_speckled_shift_%d.txt" % k))
        rows.append(r[0])
    out["single_speckled_shift_gold"] = np.asarray(rows)
    # DICe_TestImage: ImageB.tif Gauss-filtered with mask 5..13 against the
    # float-build outputs images/outFilter<M>.rawi (header: uint32 width,
    # height, bytes per value; then row-major values).  A 64 x 64 window
    # whose corner is stored beside the crops keeps the fixture small.
    out["image_b"] = _img(root, "ImageB.tif")
    y0, x0 = 40, 60
    out["gauss_gold_origin"] = np.array([y0, x0], np.int32)
    for m in (5, 7, 9, 11, 13):
        with open(os.path.join(root, "tests", "component", "images", "outFilter%d.rawi" % m), "rb") as fh:
            raw = fh.read()
        w, h, nb = np.frombuffer(raw[:12], np.uint32)
        assert nb == 4
        gold = np.frombuffer(raw[12:], np.float32).reshape(h, w)
        out["gauss_gold_%d" % m] = gold[y0:y0 + 64, x0:x0 + 64].copy()
    # DICe_TestSubset: the image of a conformal subset (two polygons minus
    # a rectangle) that Subset::write_image writes over its bounding box,
    # re-read with spread/floored intensities: 0 outside the subset, the
    # excluded pixels at one common grey, owned pixels above it.
    with open(os.path.join(root, "tests", "component", "images", "conformal.rawi"), "rb") as fh:
        raw = fh.read()
    w, h, nb = np.frombuffer(raw[:12], np.uint32)
    assert nb == 4
    out["conformal_subset_image"] = np.frombuffer(raw[12:], np.float32).reshape(h, w).copy()
    # Subset files (read as text by the parser tests) and the regression
    # runs that use them: conformal_subset_def (five subsets on the speckled
    # pair, two conformal, one with excluded / obstructed shapes and blocking
    # subsets; TRACKING_ROUTINE) and simple_obstruction (a rectangle subset
    # moving 2 px per frame under a static obstruction, 37 frames of 200 x 200).
    for name, rel in (("conformal_subset_def", "regression/conformal_subset_def/subset_defs.txt"),
                      ("simple_obstruction", "regression/simple_obstruction/subsets.txt"),
                      ("mechanism", "examples/mechanism/subsets.txt"),
                      ("obstruction_example", "examples/obstruction/subsets.txt"),
                      ("mechanism_skip_solves", "regression/mechanism_skip_solves/subsets.txt"),
                      ("mechanism_optical_flow", "regression/mechanism_optical_flow/subsets.txt")):
        with open(os.path.join(root, "tests", rel)) as fh:
            out["subset_file_" + name] = np.array(fh.read())
    # columns: frame x y u v theta exx eyy gxy sigma status, one row per subset
    out["conformal_subset_def_gold"] = np.concatenate([
        _rows(os.path.join(root, "tests", "regression", "conformal_subset_def", "gold",
                           "DICe_solution_%d.txt" % k)) for k in range(5)])
    # the gold files as text, for comparisons the way the reference's
    # regression harness makes them (DICe_Diff -t 0.05 -f 5.0E-5)
    for k in range(5):
        with open(os.path.join(root, "tests", "regression", "conformal_subset_def", "gold",
                               "DICe_solution_%d.txt" % k)) as fh:
            out["conformal_subset_def_gold_text_%d" % k] = np.array(fh.read())
    with open(os.path.join(root, "tests", "regression", "simple_obstruction", "gold", "DICe_solution_0.txt")) as fh:
        out["simple_obstruction_gold_text"] = np.array(fh.read())
    # dic_challenge_12 (region-of-interest grid, step 35, subset 27; VSG strain
    # over a 360 px window): frames 1, 6 and 11 of the unsorted and the
    # sorted output, and the region-of-interest subset file
    for variant in ("dic_challenge_12", "dic_challenge_12_sorted"):
        for k in (1, 6, 11):
            with open(os.path.join(root, "tests", "regression", variant, "gold", "DICe_solution_%02d.txt" % k)) as fh:
                out["%s_gold_text_%02d" % (variant, k)] = np.array(fh.read())
    with open(os.path.join(root, "tests", "regression", "dic_challenge_12", "subset_file.dat")) as fh:
        out["subset_file_dic_challenge_12"] = np.array(fh.read())
    from PIL import Image
    out["simple_obstruction_frames"] = np.stack([
        np.array(Image.open(os.path.join(root, "tests", "regression", "simple_obstruction", "images",
                                         "Img_%02d.tif" % k)).convert("L")) for k in range(37)])
    # columns: frame x y u
    out["simple_obstruction_gold"] = _rows(os.path.join(root, "tests", "regression", "simple_obstruction",
                                                        "gold", "DICe_solution_0.txt"))
    # examples/obstruction: a conformal subset with an excluded and an
    # obstructed region rotating 2 degrees per frame behind a static bar,
    # blocked by a second subset (tracking defaults, subset evolution)
    ex = os.path.join(root, "tests", "examples", "obstruction")
    out["obstruction_example_frames"] = np.stack([
        np.array(Image.open(os.path.join(ex, "images", "obstruction_%02d.tif" % k)).convert("L"))
        for k in range(1, 13)])
    for i in range(2):
        with open(os.path.join(ex, "gold", "DICe_solution_%d.txt" % i)) as fh:
            out["obstruction_example_gold_text_%d" % i] = np.array(fh.read())
    # seeded region-of-interest grids with neighbour initialization on the
    # speckled pair (first step only: two frames; every step: one) and the
    # incremental formulation on the synthetic speckle sequence
    for name, frames in (("parallel_seed_first_step_only", 2), ("parallel_subsets_seed", 1)):
        reg = os.path.join(root, "tests", "regression", name)
        with open(os.path.join(reg, "subset_file.dat")) as fh:
            out["subset_file_" + name] = np.array(fh.read())
        for k in range(frames):
            with open(os.path.join(reg, "gold", "DICe_solution_%d.txt" % k)) as fh:
                out["%s_gold_text_%d" % (name, k)] = np.array(fh.read())
    for k in range(6):
        with open(os.path.join(root, "tests", "regression", "incremental", "gold", "DICe_solution_%d.txt" % k)) as fh:
            out["incremental_gold_text_%d" % k] = np.array(fh.read())
    # bitmap_star: the DIC challenge wave pair (8-bit BMP, 2000 x 501; the
    # reference image is the "Deformed" file, as its input.xml names them),
    # subset 31 at step 25, KEYS_FOURTH, GRADIENT_BASED, translation only.
    # Its gold prints UNCERTAINTY = SIGMA / FIELD_1 (Uncertainty_Post_Processor,
    # DICe_PostProcessor.cpp:1507-1537).  Kept: every 20th gold row and a
    # 45 x 45 patch of each image centred on those subsets (the subset's
    # pixels, the interpolation taps, the gradient stencil and the noise box
    # all fit), cut from the images padded by 22 zero pixels.
    bs = os.path.join(root, "tests", "regression", "bitmap_star")
    from PIL import Image
    pair = [np.asarray(Image.open(os.path.join(bs, "images", nm)).convert("L"), dtype=np.uint8)
            for nm in ("DIC_Challenge_Wave_Deformed_Noisy.bmp", "DIC_Challenge_Wave_Reference_Noisy.bmp")]
    with open(os.path.join(bs, "gold", "DICe_solution_0.txt")) as fh:
        lines = fh.read().strip().splitlines()
    gold = np.array([[float(t) for t in ln.split(",")] for ln in lines[1:]])[::20]
    out["bitmap_star_columns"] = np.array(lines[0])
    out["bitmap_star_gold"] = gold
    out["bitmap_star_shape"] = np.array(pair[0].shape, np.int32)
    for key, img in zip(("ref", "def"), pair):
        padded = np.pad(img, 22)
        out["bitmap_star_%s_patches" % key] = np.stack([
            padded[int(y):int(y) + 45, int(x):int(x) + 45] for x, y in gold[:, 1:3]])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_gold.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <path to the DICe source tree>")
    main(sys.argv[1])
