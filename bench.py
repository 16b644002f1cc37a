"""Benchmark: subset solves per second of the local DIC hot path on B200.

Workload (one "step" = one frame of the sequence): a 2048 x 2048 speckle image
in 16-bit range (speckle radius 3-5 px), imposed field
u = 0.5 sin(2 pi x/128), v = 0.3 cos(2 pi y/96) plus 0.2 % uniform strain,
scaled by k/10 for frame k of a 10-frame sequence; 31 x 31 subsets at step 5
(398^2 = 158,404 subsets); affine shape function (6 parameters), ZNSSD
Gauss-Newton with Keys-4, tolerance 1e-5, 25 iterations, simplex fallback;
each frame initialised from the previous frame's solution.  The sequence
restarts from zero motion after frame 10 (a device-to-device field reset
that is part of the step).  Seeded synthetic images (no dataset).

Arms
  default            libdicegpu.so persistent batched launch (value), the same
                     through the C ABI with host buffers (e2e), and the plain
                     one-launch-per-subset path on a sample for comparison.
  --impl reference   the reference algorithm's CPU restatement (the reference
                     itself does not build here: Trilinos / OpenCV / LAPACK are
                     absent) on all host cores, a bounded sample per step.

Multi-GPU (torchrun): every rank correlates its own copy of the sequence
(subsets are independent, no collective on the data path); value is the
aggregate over ranks, time is the max over ranks (weak scaling).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

W = H = 2048
SUBSET = 31
STEP = 5
NFRAMES = 10
METRIC = "subset solves/sec at <=1e-4 px vs reference; batched vs plain on one B200"
UNIT = "subsets/s"
# algorithmic work per pixel-iteration of affine Gauss-Newton (Keys-4,
# deformed-image gradients): 390 FP32 flop + 27 FP64 flop
FP32_FLOP_PER_PIXEL_ITER = 390.0
FP64_FLOP_PER_PIXEL_ITER = 27.0
# bytes of the three interpolated planes + reference value per pixel-iteration
# if every tap came from DRAM once per subset (compulsory traffic per frame
# is the images: 6 planes of W*H floats)


def params():
    from dice_b200 import abi
    return abi.default_params(subset_size=SUBSET, enable_rotation=1, enable_normal_strain=1,
                              enable_shear_strain=1, fast_solver_tolerance=1e-5,
                              max_solver_iterations_fast=25)


def workload_config(n_subsets, n_gpus, sharded=False):
    return {"workload": "2048x2048 16-bit speckle sequence, 10 frames, 31x31 affine subsets at step 5",
            "image": [W, H], "subset_size": SUBSET, "step": STEP, "subsets_per_frame": n_subsets,
            "frames": NFRAMES, "shape_function": "affine (6 params)", "interpolation": "keys_fourth",
            "optimization": "gradient_based_then_simplex", "tolerance": 1e-5, "max_iterations": 25,
            "parallelism": ("dp%d: balanced contiguous subset ranges, NCCL all-gather of the field rows "
                            "at frame end" % n_gpus) if sharded else
                           "replicas x%d (independent subsets, no collective)" % n_gpus,
            "l2": "flushed between timed steps (256 MiB write)",
            "uncertainty_fields": "off (the reference computes them on every converged solve; the "
                                  "CPU baseline is reported with them off and on, the GPU value "
                                  "with them on beside the headline)"}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._proc = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self._proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def stop(self):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = []
        for k, nm in enumerate(names):
            if any(s[3 + k].lower().startswith("active") for s in self.samples):
                reasons.append(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_setup(n_gpus):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch
        import torch.distributed as dist
        dist.barrier(device_ids=[torch.cuda.current_device()])


def max_over_ranks(x, world):
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_sample(p, ref, frames, n_sample, nthreads, timed_frames=1, uncertainty=False):
    """The oracle on a bounded sample: the first `n_sample` subsets of the
    grid (contiguous rows), run through `timed_frames` frames from zero motion,
    with the uncertainty fields off (the GPU headline's work) or on (as the
    reference always computes them, Objective::computeUncertaintyFields on
    every converged solve)."""
    from dice_b200 import abi
    from dice_b200 import synthetic as syn
    from oracle import oracle as O
    cx, cy = syn.grid_points(W, H, SUBSET, STEP)
    f = syn.init_fields(cx[:n_sample], cy[:n_sample])
    unc = np.zeros((n_sample, abi.UNCERTAINTY_STRIDE)) if uncertainty else None
    t0 = time.perf_counter()
    for k in range(timed_frames):
        O.execute_frame(p, ref, frames[k], f, first_frame=(k == 0), nthreads=nthreads, uncertainty=unc)
    dt = time.perf_counter() - t0
    return n_sample * timed_frames / dt, dt, f


SIMPLEX_FLOP_PER_PIXEL_EVAL = 200.0
# DRAM bytes (read + write) of one frame_kernel launch of the full frame
# (158,404 subsets, a frame of the sequence), from an ncu capture of that
# launch: dram__bytes_read.sum 157.6 MB + dram__bytes_write.sum 38.2 MB
FRAME_KERNEL_DRAM_BYTES = 157.641e6 + 38.175e6


def oracle_sequence_sample(p, ref_h, frames_h, stride, nthreads, uncertainty=False, library=None):
    """The oracle over the whole frame sequence on every `stride`-th subset
    (subsets are independent under USE_FIELD_VALUES), with the uncertainty
    fields on (as the reference computes them) or off (the GPU headline's
    work), optionally through another build of the oracle.  Returns the
    sampled ids, the oracle's fields, Gauss-Newton passes and simplex
    evaluations per subset after each frame, and the wall time."""
    from dice_b200 import abi
    from dice_b200 import synthetic as syn
    from oracle import oracle as O
    cx, cy = syn.grid_points(W, H, SUBSET, STEP)
    ids = np.arange(0, len(cx), stride)
    f = syn.init_fields(cx[ids], cy[ids])
    unc = np.zeros((len(ids), abi.UNCERTAINTY_STRIDE)) if uncertainty else None
    out = []

    def run():
        t0 = time.perf_counter()
        for k, fr in enumerate(frames_h):
            gn, sx = O.execute_frame(p, ref_h, fr, f, first_frame=(k == 0), nthreads=nthreads, counters=True,
                                     uncertainty=unc)
            out.append((f.copy(), gn.copy(), sx.copy()))
        return time.perf_counter() - t0

    if library:
        with O.use_library(library):
            dt = run()
    else:
        dt = run()
    return ids, out, dt


RESULT_COLUMNS_TEXT = ("u, v, theta, strains, sigma, gamma, noise, contrast, active pixels, status, iterations, "
                       "condition number")


COLUMN_NAMES = {}


def _column_names():
    from dice_b200 import abi
    if not COLUMN_NAMES:
        for name in ("DISP_X", "DISP_Y", "ROT_Z", "STRETCH_XX", "STRETCH_YY", "SHEAR_XY", "SIGMA", "GAMMA", "NOISE",
                     "CONTRAST", "ACTIVE_PIXELS", "STATUS", "ITERATIONS", "CONDITION"):
            COLUMN_NAMES[getattr(abi, "F_" + name)] = name.lower()
    return COLUMN_NAMES


class RowComparison:
    """Rows of one run against the oracle's, frame by frame (n x stride
    each): the fractions of subset-frames with equal status, equal
    iterations and every result column equal, and the subset-frames grouped
    by optimiser path (Gauss-Newton converged on both sides, the simplex
    fallback on both, or on one side only) with the largest |du|, |dv| in
    each group."""

    def __init__(self, max_fast_iterations):
        _column_names()
        self.mx = max_fast_iterations
        self.eq_status = self.eq_iters = self.eq_all = self.tot = 0
        self.col_bad = {}
        self.groups = {"gn_both": [0, 0.0, 0.0], "simplex_both": [0, 0.0, 0.0], "path_differs": [0, 0.0, 0.0]}

    def add(self, g, o):
        from dice_b200 import abi
        cols = [abi.F_DISP_X, abi.F_DISP_Y, abi.F_ROT_Z, abi.F_STRETCH_XX, abi.F_STRETCH_YY, abi.F_SHEAR_XY,
                abi.F_SIGMA, abi.F_GAMMA, abi.F_NOISE, abi.F_CONTRAST, abi.F_ACTIVE_PIXELS, abi.F_STATUS,
                abi.F_ITERATIONS, abi.F_CONDITION]
        both = (g[:, abi.F_STATUS] < 2) & (o[:, abi.F_STATUS] < 2)
        self.eq_status += int(np.sum(g[:, abi.F_STATUS] == o[:, abi.F_STATUS]))
        self.eq_iters += int(np.sum(g[:, abi.F_ITERATIONS] == o[:, abi.F_ITERATIONS]))
        same = (g[:, cols] == o[:, cols]) | (np.isnan(g[:, cols]) & np.isnan(o[:, cols]))
        self.eq_all += int(np.sum(np.all(same, axis=1)))
        for ci, c in enumerate(cols):
            bad = ~same[:, ci]
            if bad.any():
                name = COLUMN_NAMES.get(c, str(c))
                cnt, mag = self.col_bad.get(name, (0, 0.0))
                diff = np.abs(g[bad, c] - o[bad, c])
                self.col_bad[name] = (cnt + int(bad.sum()), max(mag, float(np.nanmax(diff, initial=0.0))))
        self.tot += len(g)
        gs, os_ = g[:, abi.F_ITERATIONS] > self.mx, o[:, abi.F_ITERATIONS] > self.mx
        for name, m in (("gn_both", both & ~gs & ~os_), ("simplex_both", both & gs & os_),
                        ("path_differs", both & (gs != os_))):
            grp = self.groups[name]
            grp[0] += int(m.sum())
            grp[1] = max(grp[1], float(np.max(np.abs(g[m, abi.F_DISP_X] - o[m, abi.F_DISP_X]), initial=0.0)))
            grp[2] = max(grp[2], float(np.max(np.abs(g[m, abi.F_DISP_Y] - o[m, abi.F_DISP_Y]), initial=0.0)))
        return self

    def result(self):
        t = max(self.tot, 1)
        return {"status_equal_frac": self.eq_status / t, "iterations_equal_frac": self.eq_iters / t,
                "all_columns_equal_frac": self.eq_all / t, "status_mismatches": self.tot - self.eq_status,
                "differing_by_column": {k: {"subset_frames": v[0], "max_abs_diff": v[1]}
                                        for k, v in self.col_bad.items()},
                "by_path": {k: {"subset_frames": v[0], "max_abs_du_px": v[1], "max_abs_dv_px": v[2]}
                            for k, v in self.groups.items()}}


def compare_rows(a_rows, o_rows, max_fast_iterations):
    c = RowComparison(max_fast_iterations)
    for g, o in zip(a_rows, o_rows):
        c.add(g, o)
    return c.result()


def run_reference(args):
    """--impl reference: the reference algorithm's CPU restatement (the
    reference itself does not build here) on all host cores.  Step k is
    frame k mod 10 of the sequence on every `oracle-stride`-th subset (each
    frame from the previous frame's solution, the sequence restarting at
    frame 0), so ten steps cover the repo arm's CPU sample once; each step's
    wall time is measured, and the uncertainty fields are off as in the GPU
    headline."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from dice_b200 import abi
    from dice_b200 import synthetic as syn
    from oracle import oracle as O
    ref, frames = syn.config2(device="cpu", nframes=NFRAMES)
    ref = ref.numpy()
    frames = [fr.numpy() for fr in frames]
    p = params()
    cores = os.cpu_count() or 1
    stride = max(1, args.oracle_stride)
    cx, cy = syn.grid_points(W, H, SUBSET, STEP)
    ids = np.arange(0, len(cx), stride)
    f0 = syn.init_fields(cx[ids], cy[ids])
    state = {"k": 0, "f": f0.copy()}

    def step():
        k = state["k"] % NFRAMES
        if k == 0:
            state["f"] = f0.copy()
        t0 = time.perf_counter()
        O.execute_frame(p, ref, frames[k], state["f"], first_frame=(k == 0), nthreads=cores)
        state["k"] += 1
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        step()
    dts = [step() for _ in range(args.steps)]
    total = sum(dts)
    value = len(ids) * args.steps / total
    sample = ("every %dth subset (%d of %d), one frame of the 10-frame sequence per step in order, "
              "%d threads, uncertainty fields off" % (stride, len(ids), len(cx), cores))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded speckle sequence)", "impl": "reference",
            "config": dict(workload_config(len(cx), 1), sample=sample),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _line(metric, value, unit, world, args, ms_per_step, config, **extra):
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded speckle images)",
            "config": config}
    line.update(extra)
    return line


def _timed(fn, steps, warmup, stream, flush=None):
    """Runs fn() warmup + steps times; CUDA-event milliseconds of the timed runs."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        if flush is not None:
            flush_l2(flush)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        ms.append((a, b))
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ms]


def run_crack(args):
    """8192^2 mode-I crack sequence (8 frames, 21x21 affine subsets at step 4,
    ~4.15M subsets): the frame loop as one CUDA graph of persistent
    work-stealing launches; every result column compared with the oracle on
    every subset of a band of rows across the full width around the crack,
    every frame, beside an oracle build variant on the same subsets."""
    import torch
    from dice_b200 import abi, synthetic as syn
    from dice_b200.schema import Schema
    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    size, nf, ss, step = args.crack_size, 8, 21, 4
    ref, frames = syn.config5(device=dev, w=size, h=size, nframes=nf)
    torch.cuda.synchronize()
    cx, cy = syn.grid_points(size, size, ss, step)
    n = len(cx)
    p = abi.default_params(subset_size=ss, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1,
                           final_gamma_threshold=0.02)
    f0 = syn.init_fields(cx, cy)
    f0_dev = torch.from_numpy(f0).to(dev)
    stream = torch.cuda.current_stream()
    s = Schema(p, stream=stream)
    s.set_ref_image(ref)
    s.set_fields(f0)
    s.capture_sequence(frames, reset_fields=f0_dev)
    launches0 = s.launch_count()
    clocks = ClockSampler(torch.cuda.current_device())
    barrier(world)
    clocks.start()
    ms = _timed(s.launch_sequence, args.steps, args.warmup, stream)
    barrier(world)
    clocks.stop()
    per_launch = (s.launch_count() - launches0) / max(1, args.steps + args.warmup)
    total_ms = max_over_ranks(sum(ms), world)
    value = n * nf * args.steps * world / (total_ms / 1000.0)
    final = s.fields()
    st_final = final[:, abi.F_STATUS]
    cpu = flags = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # every subset whose centre lies in a band of rows across the whole
        # width, centred on the crack line, through all frames
        from oracle import oracle as O
        half = args.flags_band / 2.0
        ids = np.nonzero(np.abs(cy - size / 2.0) < half)[0]
        ref_h = ref.cpu().numpy()
        fdev = torch.empty((n, abi.FIELD_STRIDE), dtype=torch.float64, device=dev)
        cores = os.cpu_count() or 1
        mx = p.max_solver_iterations_fast
        gpu_vs, var_vs = RowComparison(mx), RowComparison(mx)
        failed = [0] * nf
        dt = 0.0
        # the band in chunks of subsets (bounded host memory), each chunk
        # through the whole sequence on the GPU, the oracle and the variant
        for c0 in range(0, len(ids), args.flags_chunk):
            cid = ids[c0:c0 + args.flags_chunk]
            idt = torch.from_numpy(cid).to(dev)
            s.load_fields(f0_dev)
            fo = syn.init_fields(cx[cid], cy[cid])
            fv = fo.copy()
            for k in range(nf):
                s.set_def_image(frames[k])
                s.execute_correlation()
                s.store_fields(fdev)
                g = fdev.index_select(0, idt).cpu().numpy()
                fr_h = frames[k].cpu().numpy()
                t0 = time.perf_counter()
                O.execute_frame(p, ref_h, fr_h, fo, first_frame=(k == 0), nthreads=cores)
                dt += time.perf_counter() - t0
                with O.use_library("libdiceoracle_meanfp64.so"):
                    O.execute_frame(p, ref_h, fr_h, fv, first_frame=(k == 0), nthreads=cores)
                del fr_h
                gpu_vs.add(g, fo)
                var_vs.add(fv, fo)
                failed[k] += int(np.sum(fo[:, abi.F_STATUS] >= 2))
            del g, fo, fv
        flags = dict(gpu_vs.result(), subsets=int(len(ids)), frames=nf,
                     columns=RESULT_COLUMNS_TEXT, bar="every column equal to the oracle's, bit for bit",
                     oracle_failed_per_frame=failed,
                     sample="every subset with |y - %d| < %g px (a %d-px band of rows across the full width, "
                            "centred on the crack)" % (size // 2, half, args.flags_band),
                     oracle_build_variant=dict(var_vs.result(),
                                               build="the oracle with the deformed mean summed in double"))
        cpu = {"value": len(ids) * nf / dt, "unit": "subsets/s", "cores": cores, "kind": "port",
               "sample": "the %d band subsets through %d frames, %.1f s, uncertainty fields off"
                         % (len(ids), nf, dt)}
    if rank == 0:
        cfg = {"workload": "%dx%d crack sequence, %d frames, 21x21 affine subsets at step 4" % (size, size, nf),
               "subsets_per_frame": n, "frames": nf, "tolerance": p.fast_solver_tolerance,
               "final_gamma_threshold": 0.02, "frame_loop": "one CUDA graph per sequence",
               "l2": "inputs larger than L2 (8 frames x %d MB)" % (size * size * 4 >> 20),
               "parallelism": "replicas x%d" % world}
        print(json.dumps(_line("subset solves/sec, crack sequence", value, "subsets/s", world, args,
                               total_ms / args.steps, cfg, cpu_baseline=cpu, flags_vs_oracle=flags,
                               gpu_launches=int(per_launch * args.steps), clocks=clocks.summary(),
                               accuracy={"status_counts_last_frame": {str(int(a)): int(b) for a, b in
                                                                      zip(*np.unique(st_final, return_counts=True))}})),
              flush=True)
    s.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_mixed(args):
    """4096x3000 arbitrary-shape batching: 50k seeded circles, thin ellipses
    and convex polygons under rotation plus shear.  Subsets with a minor
    extent of 10 px or more run quadratic Gauss-Newton over their pixel
    lists; thinner ones run the simplex (FORCE_SIMPLEX) in an affine
    context.  The launch shape (subsets in flight per CTA, CTAs per SM) is
    swept for each context and the fastest is used."""
    import torch
    from dice_b200 import abi, synthetic as syn
    from dice_b200.schema import Schema
    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    w, h, nsub = 4096, 3000, 50000
    ref, deff, field, sub = syn.config3(device=dev, w=w, h=h, n=nsub)
    cx, cy, offs, px, py, kind, minor = sub
    u0, v0 = field(torch.from_numpy(cx.astype(np.float64)).to(dev), torch.from_numpy(cy.astype(np.float64)).to(dev))
    u0, v0 = np.round(u0.cpu().numpy()), np.round(v0.cpu().numpy())

    def select(idx):
        no, lx, ly = [0], [], []
        for i in idx:
            lx.append(px[offs[i]:offs[i + 1]])
            ly.append(py[offs[i]:offs[i + 1]])
            no.append(no[-1] + offs[i + 1] - offs[i])
        return np.asarray(no, np.int32), np.concatenate(lx), np.concatenate(ly)

    thin = minor < 10.0
    groups = []
    stream = torch.cuda.current_stream()
    iq = np.nonzero(~thin)[0]
    pq = abi.default_params(shape_function=abi.QUADRATIC_SF, subset_size=0, fast_solver_tolerance=1e-3)
    fq = syn.init_fields(cx[iq], cy[iq], quadratic=True)
    fq[:, abi.F_QUAD_A + 5] = u0[iq]
    fq[:, abi.F_QUAD_A + 11] = v0[iq]
    groups.append(("quadratic_gauss_newton", iq, pq, fq, None))
    it = np.nonzero(thin)[0]
    ps = abi.default_params(subset_size=0, enable_rotation=1)
    fs = syn.init_fields(cx[it], cy[it])
    fs[:, abi.F_DISP_X] = u0[it]
    fs[:, abi.F_DISP_Y] = v0[it]
    groups.append(("forced_simplex", it, ps, fs, np.ones(len(it), np.uint8)))
    ctxs = []
    sweep = {}
    for name, idx, pp, ff, force in groups:
        sc = Schema(pp, stream=stream)
        sc.set_ref_image(ref)
        sc.set_fields(ff)
        sc.set_subset_pixels(*select(idx))
        if force is not None:
            sc.set_force_simplex(force)
        sc.set_def_image(deff)
        fdev = torch.from_numpy(ff).to(dev)
        times = {}
        for shape in ((8, 0), (4, 0), (2, 0), (8, 1), (4, 2), (4, 3)):
            sc.set_launch_shape(*shape)

            def once(sc=sc, fdev=fdev):
                sc.load_fields(fdev)
                sc.execute_correlation()
            times["%dx%d" % shape] = statistics.median(_timed(once, 2, 1, stream))
        best = min(times, key=times.get)
        sc.set_launch_shape(*[int(t) for t in best.split("x")])
        sweep[name] = {"ms_by_warps_x_ctas_per_sm": times, "chosen": best,
                       "library_autotune": list(sc.autotune())}
        ctxs.append((name, idx, pp, ff, force, sc, fdev))

    def step():
        for name, idx, pp, ff, force, sc, fdev in ctxs:
            sc.load_fields(fdev)
            sc.execute_correlation()

    launches0 = sum(c[5].launch_count() for c in ctxs)
    clocks = ClockSampler(torch.cuda.current_device())
    l2 = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    barrier(world)
    clocks.start()
    ms = _timed(step, args.steps, args.warmup, stream, flush=l2)
    barrier(world)
    clocks.stop()
    launches = sum(c[5].launch_count() for c in ctxs) - launches0
    total_ms = max_over_ranks(sum(ms), world)
    value = nsub * args.steps * world / (total_ms / 1000.0)
    acc, par = {}, {}
    cpu = None
    dt_cpu, n_cpu = 0.0, 0
    for name, idx, pp, ff, force, sc, fdev in ctxs:
        g = sc.fields()
        st = g[:, abi.F_STATUS]
        acc[name] = {"subsets": int(len(idx)), "converged_frac": float(np.mean(st < 2)),
                     "simplex_fallback_frac": float(np.mean((st < 2) & (g[:, abi.F_ITERATIONS] >
                                                                        pp.max_solver_iterations_fast)))
                     if force is None else None}
        if rank == 0 and world == 1 and not args.no_cpu:
            from oracle import oracle as O
            sel = np.arange(0, len(idx), 25)
            no, lx, ly = select(idx[sel])
            fo = ff[sel].copy()
            t0 = time.perf_counter()
            O.execute_frame(pp, ref.cpu().numpy(), deff.cpu().numpy(), fo, first_frame=True,
                            nthreads=os.cpu_count() or 1, offsets=no, px=lx, py=ly,
                            force_simplex=None if force is None else force[sel],
                            uncertainty=np.zeros((len(sel), abi.UNCERTAINTY_STRIDE)))
            dt_cpu += time.perf_counter() - t0
            n_cpu += len(sel)
            gs = g[sel]
            both = (gs[:, abi.F_STATUS] < 2) & (fo[:, abi.F_STATUS] < 2)
            if force is None:
                both &= (gs[:, abi.F_ITERATIONS] <= pp.max_solver_iterations_fast) & \
                        (fo[:, abi.F_ITERATIONS] <= pp.max_solver_iterations_fast)
            par[name] = {"subsets": int(len(sel)),
                         "status_equal_frac": float(np.mean(gs[:, abi.F_STATUS] == fo[:, abi.F_STATUS])),
                         "compared": int(both.sum()),
                         "max_abs_du_px": float(np.max(np.abs(gs[both, abi.F_DISP_X] - fo[both, abi.F_DISP_X]),
                                                       initial=0.0)),
                         "max_abs_dv_px": float(np.max(np.abs(gs[both, abi.F_DISP_Y] - fo[both, abi.F_DISP_Y]),
                                                       initial=0.0))}
    if n_cpu:
        cpu = {"value": n_cpu / dt_cpu, "unit": "subsets/s", "cores": os.cpu_count() or 1, "kind": "port",
               "sample": "every 25th subset of each group (%d), %.1f s, uncertainty fields on" % (n_cpu, dt_cpu)}
    if rank == 0:
        cfg = {"workload": "4096x3000 mixed conformal subsets (circles r 7-25, 60x8 ellipses, convex polygons)",
               "subsets": nsub, "groups": {k: v["subsets"] for k, v in acc.items()},
               "quadratic_tolerance": 1e-3,
               "tolerance_note": "1e-3: mapped coordinates up to 4096 px are spaced 4.9e-4 px in float",
               "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas x%d" % world}
        print(json.dumps(_line("subset solves/sec, mixed arbitrary-shape subsets", value, "subsets/s", world,
                               args, total_ms / args.steps, cfg, cpu_baseline=cpu, launch_shape_sweep=sweep,
                               parity_vs_oracle=par, accuracy=acc, gpu_launches=int(launches),
                               clocks=clocks.summary())), flush=True)
    for c in ctxs:
        c[5].close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


ADJ_FLOP_PER_PIXEL = 560.0


def run_adjoint(args):
    """1024^2 pair with a 16x16 cubic B-spline field: the adjoint of the
    subset objective (gamma, d/dparams, d/d deformed image) for 19,600
    affine 25x25 subsets per step, then the B-spline control grid fitted by
    gradient descent through it and compared with per-subset Gauss-Newton."""
    import torch
    from dice_b200 import abi, bspline, synthetic as syn
    from dice_b200.schema import Schema
    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    size = 1024
    ref, deff, field, ctrl = syn.config4(device=dev, w=size, h=size)
    cx, cy = syn.grid_points(size, size, 25, 7)
    n = len(cx)
    p = abi.default_params(subset_size=25, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1,
                           fast_solver_tolerance=1e-5)
    stream = torch.cuda.current_stream()
    s = Schema(p, stream=stream)
    s.set_ref_image(ref)
    s.set_subsets(cx, cy)
    s.set_def_image(deff)
    tcx, tcy = torch.from_numpy(cx).to(dev), torch.from_numpy(cy).to(dev)
    rows = torch.from_numpy(syn.init_fields(cx, cy)).to(dev)
    rows[:, abi.F_DISP_X:abi.F_DISP_X + 6] = field.subset_params(ctrl, tcx, tcy)
    rows = rows.contiguous()
    seed = torch.ones(n, dtype=torch.float64, device=dev)
    ddef = torch.zeros((size, size), dtype=torch.float32, device=dev)
    l2 = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        ddef.zero_()
        s.adjoint(rows, seed=seed, ddef=ddef)

    launches0 = s.launch_count()
    clocks = ClockSampler(torch.cuda.current_device())
    barrier(world)
    clocks.start()
    ms = _timed(step, args.steps, args.warmup, stream, flush=l2)
    barrier(world)
    clocks.stop()
    launches = s.launch_count() - launches0
    total_ms = max_over_ranks(sum(ms), world)
    value = n * args.steps * world / (total_ms / 1000.0)
    val, _ = s.adjoint(rows)
    torch.cuda.synchronize()
    active = float(n * 625)
    achieved = active * ADJ_FLOP_PER_PIXEL / (statistics.median(ms) / 1000.0) / 1e12
    peak = fp32_peak_tflops(dev)
    # per-subset Gauss-Newton, then the B-spline fit through the adjoint
    s.execute_correlation()
    gn = s.fields()
    t0 = time.perf_counter()
    fit = bspline.fit(s, deff, field, tcx, tcy, iters=args.fit_iters, lr=0.05)
    torch.cuda.synchronize()
    fit_s = time.perf_counter() - t0
    ut, vt = field.eval(ctrl, tcx, tcy)
    uf, vf = field.eval(fit, tcx, tcy)
    ok = torch.from_numpy(gn[:, abi.F_STATUS] < 2).to(dev)
    ug = torch.from_numpy(gn[:, abi.F_DISP_X]).to(dev)
    vg = torch.from_numpy(gn[:, abi.F_DISP_Y]).to(dev)
    fit_res = {"iterations": args.fit_iters, "seconds": fit_s, "control_grid": [2, 16, 16],
               "rms_error_fit_px": bspline.rms(torch.cat([(uf - ut)[ok], (vf - vt)[ok]])),
               "rms_error_gauss_newton_px": bspline.rms(torch.cat([(ug - ut)[ok], (vg - vt)[ok]])),
               "rms_fit_minus_gauss_newton_px": bspline.rms(torch.cat([(uf - ug)[ok], (vf - vg)[ok]])),
               "gauss_newton_converged_frac": float(ok.float().mean())}
    if rank == 0:
        cfg = {"workload": "1024x1024 B-spline field pair, 19,600 affine 25x25 subsets at step 7",
               "subsets": n, "outputs": "gamma, d/dparams (6), d/d deformed image (atomic scatter)",
               "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas x%d" % world}
        roof = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if peak else None, "traffic": None,
                "per_unit": "%d FP32 flop per subset pixel (both passes) plus 36 atomic adds" % ADJ_FLOP_PER_PIXEL,
                "kernel": "adjoint_kernel (median step incl. clearing the image derivative)"}
        print(json.dumps(_line("subset objective adjoints/sec (value, d/dparams, d/dimage)", value, "subsets/s",
                               world, args, total_ms / args.steps, cfg, roofline=roof,
                               cpu_baseline={"value": None, "note": "the reference has no derivative code"},
                               bspline_fit=fit_res, mean_gamma=float(val.mean()),
                               gpu_launches=int(launches), clocks=clocks.summary())), flush=True)
    s.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def conformal_case(nside=50, step=40, seed=9, rmin=14, rmax=20):
    """nside x nside conformal subsets (convex polygons or rectangles,
    radius rmin-rmax px) on a step-px grid of the 2048^2 sequence's first
    frame pair, 30 % with an obstructed rectangle near the centre, each
    blocked by its right neighbour and every tenth also by its left."""
    from dice_b200 import abi
    rng = np.random.default_rng(seed)
    shapes, vx, vy, cx, cy, blockers = [], [], [], [], [], []
    x0 = (W - (nside - 1) * step) // 2
    y0 = (H - (nside - 1) * step) // 2
    for j in range(nside):
        for i in range(nside):
            k = len(cx)
            x, y = x0 + i * step, y0 + j * step
            cx.append(float(x))
            cy.append(float(y))
            if rng.random() < 0.5:
                shapes.append(abi.rectangle(k, x, y, int(rng.integers(2 * rmin + 1, 2 * rmax + 1)),
                                            int(rng.integers(2 * rmin + 1, 2 * rmax + 1))))
            else:
                m = int(rng.integers(5, 8))
                ang = np.sort(rng.uniform(0, 2 * np.pi, m))
                rad = rng.uniform(rmin, rmax, m)
                shapes.append(abi.polygon(k, len(vx), m))
                vx += list(np.round(x + rad * np.cos(ang)).astype(int))
                vy += list(np.round(y + rad * np.sin(ang)).astype(int))
            if rng.random() < 0.3:
                shapes.append(abi.rectangle(k, x + int(rng.integers(-6, 7)), y + int(rng.integers(-6, 7)),
                                            int(rng.integers(5, 10)), int(rng.integers(5, 10)),
                                            role=abi.ROLE_OBSTRUCTED))
            b = [k + 1] if i + 1 < nside else []
            if i > 0 and k % 10 == 0:
                b.append(k - 1)
            blockers.append(b)
    return (np.asarray(cx), np.asarray(cy), shapes, np.asarray(vx, np.int32), np.asarray(vy, np.int32), blockers)


def run_conformal(args):
    """Conformal subsets built on the device from shapes, with obstructed
    regions and blocking subsets, under the tracking routine (ordered waves,
    blocked bitmaps rebuilt per wave): one step is one frame over all
    subsets.  Also times the rasterization and the same subsets without
    obstructions or blocking."""
    import torch
    from dice_b200 import abi, synthetic as syn
    from dice_b200.schema import Schema
    from oracle import oracle as O
    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    ref, frames = syn.config2(device=dev, count=1)
    cx, cy, shapes, vx, vy, blockers = conformal_case()
    n = len(cx)
    # the tracking defaults' degrees of freedom (translation, rotation); Gauss-Newton kept for every subset
    p = abi.default_params(subset_size=0, enable_rotation=1, correlation_routine=abi.TRACKING_ROUTINE,
                           override_force_simplex=1, fast_solver_tolerance=1e-3)
    f0 = syn.init_fields(cx, cy)
    stream = torch.cuda.current_stream()
    s = Schema(p, stream=stream)
    s.set_ref_image(ref)
    s.set_fields(f0)
    s.set_def_image(frames[0])
    # rasterization: every subset's pixel list from its shapes
    raster_ms = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.set_subset_shapes(shapes, vx, vy)
        torch.cuda.synchronize()
        raster_ms.append((time.perf_counter() - t0) * 1000.0)
    offs_l, px_l, py_l = s.subset_pixels()
    s.set_blocking(blockers)
    f0_dev = torch.from_numpy(f0).to(dev)

    def step():
        s.load_fields(f0_dev)
        s.execute_correlation()

    l2 = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    launches0 = s.launch_count()
    clocks = ClockSampler(torch.cuda.current_device())
    barrier(world)
    clocks.start()
    ms = _timed(step, args.steps, args.warmup, stream, flush=l2)
    barrier(world)
    clocks.stop()
    launches = s.launch_count() - launches0
    total_ms = max_over_ranks(sum(ms), world)
    value = n * args.steps * world / (total_ms / 1000.0)
    g = s.fields()
    # the same pixel lists without obstruction or blocking (generic, unmasked kernel)
    p_plain = p.copy()
    p_plain.correlation_routine = abi.GENERIC_ROUTINE
    s2 = Schema(p_plain, stream=stream)
    s2.set_ref_image(ref)
    s2.set_fields(f0)
    s2.set_subset_pixels(offs_l, px_l, py_l)
    s2.set_def_image(frames[0])

    def step_plain():
        s2.load_fields(f0_dev)
        s2.execute_correlation()
    plain_ms = statistics.median(_timed(step_plain, args.steps, args.warmup, stream, flush=l2))
    par, cpu = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        fo = f0.copy()
        offs = np.zeros(n + 1, np.int32)
        ids = []
        for i, b in enumerate(blockers):
            ids += b
            offs[i + 1] = offs[i] + len(b)
        t0 = time.perf_counter()
        O.execute_frame_shapes(p, ref.cpu().numpy(), frames[0].cpu().numpy(), fo, shapes, vx, vy, offs,
                               np.asarray(ids, np.int32), first_frame=True)
        dt = time.perf_counter() - t0
        cpu = {"value": n / dt, "unit": "subsets/s", "cores": 1, "kind": "port",
               "sample": "the whole frame (%d subsets; tracking order is sequential), %.1f s" % (n, dt)}
        # where both sides take the Gauss-Newton path (the simplex stops on flat valleys by rounding)
        both = (g[:, abi.F_STATUS] < 2) & (fo[:, abi.F_STATUS] < 2) & \
               (g[:, abi.F_ITERATIONS] <= p.max_solver_iterations_fast) & \
               (fo[:, abi.F_ITERATIONS] <= p.max_solver_iterations_fast)
        par = {"status_equal_frac": float(np.mean(g[:, abi.F_STATUS] == fo[:, abi.F_STATUS])),
               "active_pixels_equal_frac": float(np.mean(g[:, abi.F_ACTIVE_PIXELS] == fo[:, abi.F_ACTIVE_PIXELS])),
               "active_pixels_equal_frac_gauss_newton": float(np.mean(g[both, abi.F_ACTIVE_PIXELS] ==
                                                                      fo[both, abi.F_ACTIVE_PIXELS])),
               "compared": int(both.sum()),
               "max_abs_du_px": float(np.max(np.abs(g[both, abi.F_DISP_X] - fo[both, abi.F_DISP_X]), initial=0.0)),
               "max_abs_dv_px": float(np.max(np.abs(g[both, abi.F_DISP_Y] - fo[both, abi.F_DISP_Y]), initial=0.0))}
        # at tolerance 1e-3 a solve stopping one iteration apart differs by up to the tolerance
        same = both & (g[:, abi.F_ITERATIONS] == fo[:, abi.F_ITERATIONS])
        par["iterations_equal_frac"] = float(np.mean(same[both]))
        par["max_abs_du_px_same_iterations"] = float(np.max(np.abs(g[same, abi.F_DISP_X] - fo[same, abi.F_DISP_X]),
                                                            initial=0.0))
    if rank == 0:
        npix = np.diff(offs_l)
        cfg = {"workload": "%d conformal subsets (polygons / rectangles, r 14-20 px, step 40) on the 2048x2048 "
                           "sequence's first pair, 30 %% obstructed, blocked by right neighbours (every 10th also "
                           "left), tracking routine, translation + rotation" % n,
               "subsets": n, "mean_pixels": float(npix.mean()),
               "masked_subsets": int(sum(1 for sh in shapes if sh.role == abi.ROLE_OBSTRUCTED)),
               "blocking_lists": int(sum(1 for b in blockers if b)),
               "tolerance": 1e-3, "l2": "flushed between timed steps (256 MiB write)",
               "parallelism": "replicas x%d" % world}
        print(json.dumps(_line("conformal subset solves/sec (device rasterized, obstructions, blocking, tracking)",
                               value, "subsets/s", world, args, total_ms / args.steps, cfg,
                               rasterize_ms={"median": statistics.median(raster_ms), "note": "set_subset_shapes: "
                                             "host validation, count kernel, offsets, fill kernel, obstruction "
                                             "bitmaps"},
                               same_lists_without_masks_ms=plain_ms,
                               active_pixels_frac=float(np.sum(g[:, abi.F_ACTIVE_PIXELS].clip(0)) / npix.sum()),
                               cpu_baseline=cpu, parity_vs_oracle=par, gpu_launches=int(launches),
                               clocks=clocks.summary())), flush=True)
    s.close()
    s2.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_vsg(args):
    """VSG strain of the 2048^2 sequence's subset field (158,404 subsets at
    step 5 after correlating frame 1; strain window 41 px): one step is one
    VSG_Strain_Post_Processor pass over every subset (uniform-grid
    neighbourhoods, per-subset plane fits).  e2e: the field rows uploaded from
    host memory, the pass, and the VSG rows read back through the C ABI."""
    import ctypes
    import torch
    from dice_b200 import abi, synthetic as syn
    from dice_b200.schema import Schema
    from oracle import oracle as O
    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    window = args.vsg_window
    p = params()
    ref, frames = syn.config2(device=dev, nframes=2)
    cx, cy = syn.grid_points(W, H, SUBSET, STEP)
    n = len(cx)
    stream = torch.cuda.current_stream()
    s = Schema(p, stream=stream)
    s.set_ref_image(ref)
    s.set_fields(syn.init_fields(cx, cy))
    s.set_def_image(frames[1])
    s.execute_correlation()
    fields = s.fields()
    fields_pinned = torch.from_numpy(fields).pin_memory()
    out_pinned = torch.empty((n, abi.VSG_STRIDE), dtype=torch.float64).pin_memory()
    lib = s.lib
    l2 = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        abi.check(lib.dicegpu_vsg_strain(s.ctx, window, None, 1), "vsg_strain")

    def step_e2e():
        abi.check(lib.dicegpu_load_fields(s.ctx, ctypes.c_void_p(fields_pinned.data_ptr()), 0), "load_fields")
        abi.check(lib.dicegpu_vsg_strain(s.ctx, window, ctypes.c_void_p(out_pinned.data_ptr()), 0), "vsg")

    step()   # builds the neighbour grid
    torch.cuda.synchronize()
    launches0 = s.launch_count()
    clocks = ClockSampler(torch.cuda.current_device())
    barrier(world)
    clocks.start()
    ms = _timed(step, args.steps, args.warmup, stream, flush=l2)
    barrier(world)
    clocks.stop()
    launches = s.launch_count() - launches0
    total_ms = max_over_ranks(sum(ms), world)
    value = n * args.steps * world / (total_ms / 1000.0)
    # end to end through the C ABI (the grid is rebuilt after load_fields)
    step_e2e()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_steps = max(3, args.steps // 2)
    for _ in range(e2e_steps):
        step_e2e()
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    got = s.vsg_strain(window)
    # parity against the oracle on the whole field, and the CPU baseline
    t0 = time.perf_counter()
    want, failed = O.vsg_strain(fields, window)
    cpu_s = time.perf_counter() - t0
    ok = failed == 0
    rel = float(np.max(np.abs(got[ok, :7] - want[ok]) / np.maximum(np.abs(want[ok]), 1e-9)))
    flags_equal = bool(np.array_equal(got[:, :7][~ok], np.zeros_like(want[~ok])) and
                       np.array_equal(s.fields()[:, abi.F_MATCH] == -1.0, (failed == 1) | (fields[:, abi.F_MATCH] == -1.0)))
    neighbours = float(np.mean(got[:, abi.VSG_NEIGHBORS]))
    med = statistics.median(ms)
    # algorithmic bytes: each subset's coordinates, u, v and sigma read once
    # (5 doubles) and its 8 VSG values written
    alg_bytes = n * (5 + 8) * 8.0
    peak = measured_peaks().get("hbm_gbs") or 6650.0
    achieved = alg_bytes / (med / 1000.0) / 1e9
    if rank == 0:
        cfg = {"workload": "VSG strain of 158,404 subsets (2048x2048 sequence, frame 1, step 5), window %d px"
                           % window, "subsets": n, "window": window, "mean_valid_neighbours": neighbours,
               "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas x%d" % world}
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "kernel": "vsg_kernel",
                "per_unit": "104 B per subset (5 doubles read, 8 written); the %.0f neighbour gathers per subset "
                            "come from L2" % neighbours}
        print(json.dumps(_line("VSG strain subsets/sec", value, "subsets/s", world, args, total_ms / args.steps,
                               cfg, roofline=roof,
                               e2e={"value": n / e2e_s, "unit": "subsets/s", "h2d_bytes_per_step": fields.nbytes,
                                    "d2h_bytes_per_step": n * abi.VSG_STRIDE * 8},
                               cpu_baseline={"value": n / cpu_s, "unit": "subsets/s", "cores": 1, "kind": "port",
                                             "sample": "all subsets, one core (grid neighbour search)"},
                               parity_vs_oracle={"max_rel_diff": rel, "failed_and_match_equal": flags_equal,
                                                 "failed": int(failed.sum())},
                               gpu_launches=int(launches), clocks=clocks.summary())), flush=True)
    s.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def flush_l2(buf):
    buf.zero_()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dicegpu", choices=["dicegpu", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="subsets in the CPU sample (0: sized for ~15 s of CPU work)")
    ap.add_argument("--plain-sample", type=int, default=4000)
    ap.add_argument("--oracle-stride", type=int, default=10,
                    help="the oracle runs every n-th subset through the sequence")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--uncertainty-steps", type=int, default=5,
                    help="timed frames of the GPU with the uncertainty fields on (0: skip)")
    ap.add_argument("--warps", type=int, default=0)
    ap.add_argument("--ctas", type=int, default=0)
    ap.add_argument("--workload", default="sequence",
                    choices=["sequence", "crack", "mixed", "adjoint", "vsg", "conformal"],
                    help="sequence: the 2048^2 ten-frame sequence (default, the headline); crack: the "
                         "8192^2 crack sequence; mixed: arbitrary-shape subsets; adjoint: objective "
                         "derivatives and the B-spline fit; vsg: VSG strain of the sequence's field; "
                         "conformal: device-rasterized subsets with obstructions and blocking")
    ap.add_argument("--vsg-window", type=int, default=41)
    ap.add_argument("--crack-size", type=int, default=8192)
    ap.add_argument("--flags-band", type=int, default=4096,
                    help="crack workload: height in px of the band of rows checked against the oracle")
    ap.add_argument("--flags-chunk", type=int, default=400000,
                    help="crack workload: subsets of the band per pass through the sequence")
    ap.add_argument("--fit-iters", type=int, default=2000)
    ap.add_argument("--profile-timed", action="store_true",
                    help="sequence workload: bracket the timed steps with cudaProfilerStart/Stop "
                         "(for ncu --profile-from-start off)")
    ap.add_argument("--section-timers", action="store_true",
                    help="sequence workload, with a library built with -DDG_PROFILE: add the frame "
                         "kernel's section timers over the timed steps (cycles per subset) to the line")
    ap.add_argument("--shard", action="store_true",
                    help="sequence workload: split the subsets over the ranks (strong scaling) "
                         "instead of running replicas")
    args = ap.parse_args()
    # one process per GPU: started as one process with --gpus N > 1, re-run as
    # N ranks under torch.distributed.run (fails if the ranks come out != N)
    from dice_b200 import launch
    launch.ensure_ranks(args.gpus, script=os.path.abspath(__file__))
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload != "sequence":
        {"crack": run_crack, "mixed": run_mixed, "adjoint": run_adjoint, "vsg": run_vsg,
         "conformal": run_conformal}[args.workload](args)
        return
    import torch
    from dice_b200 import abi, synthetic as syn
    from dice_b200.schema import Schema

    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    p = params()
    ref, frames = syn.config2(device=dev, nframes=NFRAMES)
    torch.cuda.synchronize()
    cx, cy = syn.grid_points(W, H, SUBSET, STEP)
    n_total = len(cx)
    # --shard: this rank's balanced contiguous range of the subsets, and an
    # all-gather of the field rows at the end of every frame (strong
    # scaling); otherwise every rank runs the whole frame (replicas)
    sharded = args.shard and world > 1
    if sharded:
        from dice_b200 import shard
        starts = shard.partition(np.full(n_total, float(SUBSET * SUBSET)), world)
        cx, cy = cx[starts[rank]:starts[rank + 1]], cy[starts[rank]:starts[rank + 1]]
    n = len(cx)
    f0 = syn.init_fields(cx, cy)
    stream = torch.cuda.current_stream()

    s = Schema(p, stream=stream)
    if args.warps or args.ctas:
        s.set_launch_shape(args.warps, args.ctas)
    s.set_ref_image(ref)
    s.set_fields(f0)
    f0_dev = torch.from_numpy(f0).to(dev)
    nbytes_fields = f0.nbytes
    l2_buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    lib = s.lib

    state = {"frame": 0}
    local_rows = torch.empty((n, abi.FIELD_STRIDE), dtype=torch.float64, device=dev) if sharded else None

    def step_device():
        k = state["frame"]
        if k == 0:
            s.load_fields(f0_dev)   # sequence restart: zero motion, frame 0
        s.set_def_image(frames[k])
        s.execute_correlation()
        if sharded:
            s.store_fields(local_rows)
            state["gathered"] = shard.gather_rows(local_rows, starts)
        state["frame"] = (k + 1) % NFRAMES

    # warm-up (first frame includes the field-of-view test path)
    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()
    launches0 = s.launch_count()

    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    iters_total = 0.0
    npix = SUBSET * SUBSET
    fields_seen = []
    if args.profile_timed:
        torch.cuda.cudart().cudaProfilerStart()
    timers = None
    if args.section_timers:
        import ctypes
        if not hasattr(lib, "dicegpu_prof_read"):
            raise SystemExit("--section-timers needs a library built with -DDG_PROFILE")
        timers = (ctypes.c_ulonglong * 16)()
        torch.cuda.synchronize()
        abi.check(lib.dicegpu_prof_read(timers), "prof_read")   # clears the warm-up's
    for i in range(args.steps):
        flush_l2(l2_buf)
        ev[i][0].record(stream)
        step_device()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    if args.profile_timed:
        torch.cuda.cudart().cudaProfilerStop()
    if timers is not None:
        abi.check(lib.dicegpu_prof_read(timers), "prof_read")
    barrier(world)
    clocks.stop()
    launches = s.launch_count() - launches0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(sum(step_ms), world)
    value = (n_total if sharded else n * world) * args.steps / (total_ms / 1000.0)

    # accuracy of the last timed frame
    fl = s.fields()
    st = fl[:, abi.F_STATUS]
    ok = st < 2
    kernel_ms = statistics.median(step_ms)

    # e2e through the C ABI with host buffers: H2D of the frame, D2H of the fields
    host_frames = [fr.cpu().pin_memory() for fr in frames[:2]]
    host_fields = torch.empty((n, abi.FIELD_STRIDE), dtype=torch.float64).pin_memory()
    import ctypes
    e2e_ev = []
    s.set_fields(f0)
    for i in range(max(3, args.steps // 2) + 2):
        hf = host_frames[i % 2]
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush_l2(l2_buf)
        a.record(stream)
        abi.check(lib.dicegpu_set_def_image(s.ctx, W, H, ctypes.c_void_p(hf.data_ptr()), 0), "set_def_image")
        abi.check(lib.dicegpu_execute_correlation(s.ctx), "execute")
        s.store_fields(host_fields)
        b.record(stream)
        e2e_ev.append((a, b))
    torch.cuda.synchronize()
    e2e_ms = [a.elapsed_time(b) for a, b in e2e_ev[2:]]
    e2e_total = max_over_ranks(sum(e2e_ms), world)
    e2e_value = (n_total if sharded else n * world) * len(e2e_ms) / (e2e_total / 1000.0)

    # plain path (one launch per subset) on a sample of subsets
    plain = None
    if args.plain_sample > 0:
        ns = min(args.plain_sample, n)
        sp = Schema(p, stream=stream)
        sp.set_ref_image(ref)
        sp.set_fields(f0[:ns])
        sp.set_def_image(frames[0])
        sp.execute_correlation_plain()
        torch.cuda.synchronize()
        sp.set_fields(f0[:ns])
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sp.execute_correlation_plain()
        b.record(stream)
        torch.cuda.synchronize()
        plain_ms = a.elapsed_time(b)
        sb = Schema(p, stream=stream)
        sb.set_ref_image(ref)
        sb.set_fields(f0[:ns])
        sb.set_def_image(frames[0])
        sb.execute_correlation()
        torch.cuda.synchronize()
        plain = {"value": ns / (plain_ms / 1000.0), "unit": UNIT, "subsets": ns,
                 "launches": ns, "batched_speedup": value / world / (ns / (plain_ms / 1000.0))}
        sp.close()
        sb.close()

    # The GPU with the uncertainty fields on (Objective::computeUncertaintyFields
    # on every converged solve, as the reference always runs it), a few frames
    unc_value = None
    if args.uncertainty_steps > 0:
        pu = params()
        pu.compute_uncertainty = 1
        su = Schema(pu, stream=stream)
        su.set_ref_image(ref)
        su.set_fields(f0)
        ustate = {"frame": 0}

        def step_unc():
            k = ustate["frame"]
            if k == 0:
                su.load_fields(f0_dev)
            su.set_def_image(frames[k])
            su.execute_correlation()
            ustate["frame"] = (k + 1) % NFRAMES

        ums = _timed(step_unc, args.uncertainty_steps, 1, stream, flush=l2_buf)
        unc_value = n * world * len(ums) / (max_over_ranks(sum(ums), world) / 1000.0)
        su.close()

    # The oracle through the whole sequence on every `stride`-th subset gives
    # the CPU baseline (all host cores; uncertainty fields off as in the GPU
    # headline, and on as the reference always runs them), the algorithmic
    # work of a frame from the oracle's own pass counts (so a change in
    # convergence cannot inflate it), and a full-size parity check of the GPU
    # on the same subsets, beside how far an oracle built with one rounding
    # change (the deformed mean summed in double) moves from the oracle there.
    cpu = None
    work = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        ref_h = ref.cpu().numpy()
        fr_h = [fr.cpu().numpy() for fr in frames]
        cores = os.cpu_count() or 1
        stride = max(1, args.oracle_stride)
        ids, orc, dt = oracle_sequence_sample(p, ref_h, fr_h, stride, cores)
        ns = len(ids)
        v = ns * NFRAMES / dt
        _, _, dt_unc = oracle_sequence_sample(p, ref_h, fr_h, stride, cores, uncertainty=True)
        _, var, _ = oracle_sequence_sample(p, ref_h, fr_h, stride, cores, library="libdiceoracle_meanfp64.so")
        n1 = int(min(ns, max(200, 5.0 * v / cores)))
        v1, dt1, _ = cpu_sample(p, ref_h, fr_h[:1], n1, 1)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "every %dth subset (%d of %d) through all %d frames, %d threads, %.1f s, "
                         "uncertainty fields off (the GPU headline's work)" % (stride, ns, n, NFRAMES, cores, dt),
               "uncertainty_on": {"value": ns * NFRAMES / dt_unc, "unit": UNIT,
                                  "sample": "the same subsets and frames with the uncertainty fields on, "
                                            "%.1f s" % dt_unc},
               "one_core": {"value": v1, "unit": UNIT,
                            "sample": "first %d subsets of frame 1, 1 thread, %.1f s" % (n1, dt1)}}
        gn_flop = sx_flop = 0.0
        for fo, gn, sx in orc:
            act = np.where(fo[:, abi.F_ACTIVE_PIXELS] > 0, fo[:, abi.F_ACTIVE_PIXELS], SUBSET * SUBSET)
            gn_flop += float(np.sum(gn * act)) * FP32_FLOP_PER_PIXEL_ITER
            sx_flop += float(np.sum(sx * act)) * SIMPLEX_FLOP_PER_PIXEL_EVAL
        work = {"flop_per_frame": (gn_flop + sx_flop) * (n / ns) / NFRAMES,
                "gn_pixel_passes_per_frame": gn_flop / FP32_FLOP_PER_PIXEL_ITER * (n / ns) / NFRAMES,
                "sampled_subsets": int(ns)}
        # the GPU through the same sequence from frame 0, compared on the sampled subsets
        s.load_fields(f0_dev)
        fdev = torch.empty((n, abi.FIELD_STRIDE), dtype=torch.float64, device=dev)
        idt = torch.from_numpy(ids).to(dev)
        mx = p.max_solver_iterations_fast
        compare = lambda a_rows, o_rows: compare_rows(a_rows, o_rows, mx)

        gpu_rows = []
        for k in range(NFRAMES):
            s.set_def_image(frames[k])
            s.execute_correlation()
            s.store_fields(fdev)
            gpu_rows.append(fdev.index_select(0, idt).cpu().numpy())
        torch.cuda.synchronize()
        oracle_rows = [o[0] for o in orc]
        parity = dict(compare(gpu_rows, oracle_rows), subsets=int(ns), frames=NFRAMES,
                      columns=RESULT_COLUMNS_TEXT,
                      bar="every column equal to the oracle's, bit for bit",
                      oracle_build_variant=dict(compare([o[0] for o in var], oracle_rows),
                                                build="the oracle with the deformed mean summed in double"))
    fp32_tflops = (work["flop_per_frame"] / (kernel_ms / 1000.0) / 1e12) if work else None

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    fp32_peak = fp32_peak_tflops(dev)
    roof = {"bound": "fp32", "achieved": fp32_tflops, "peak": fp32_peak, "unit": "TFLOP/s",
            "frac": fp32_tflops / fp32_peak if (fp32_peak and fp32_tflops) else None,
            "traffic": FRAME_KERNEL_DRAM_BYTES,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one frame_kernel launch "
                              "on a full frame (reads 157.6 MB, writes 38.2 MB)",
            "issue": {"inst_per_cycle_per_scheduler": 0.43, "warp_instructions_per_frame": 28.9e9,
                      "source": "ncu smsp__issue_active / smsp__inst_executed.sum of the same capture; the "
                                "binding resource is instruction issue, not a math pipe or DRAM"},
            "kernel": "frame_kernel (median step time incl. the gradient and pack kernels)",
            "peak_source": "measured FP32 SGEMM on CUDA cores (TF32 off) in this run",
            "per_unit": "390 FP32 flop per active pixel per Gauss-Newton pass + 200 per simplex evaluation, "
                        "pass counts of the oracle on the sampled subsets scaled to the frame",
            "work": work, "hbm_peak_gbs": peaks.get("hbm_gbs")}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "strong" if sharded else "weak", "vs_baseline": None, "dtype": "f32+f64",
                "data": "synthetic (seeded speckle sequence)",
                "config": workload_config(n_total, world, sharded),
                "roofline": roof, "cpu_baseline": cpu,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": W * H * 4,
                        "d2h_bytes_per_step": nbytes_fields},
                "gpu_launches": int(launches), "clocks": clocks.summary(), "plain": plain,
                "uncertainty_on": ({"value": unc_value, "unit": UNIT, "steps": args.uncertainty_steps,
                                    "note": "the same sequence with the uncertainty fields computed"}
                                   if unc_value else None),
                "parity_vs_oracle": parity,
                "accuracy": {"converged_frac": float(ok.mean()),
                             "status_counts": {str(int(k)): int(v) for k, v in zip(*np.unique(st, return_counts=True))},
                             "mean_iterations": float(np.mean(fl[ok, abi.F_ITERATIONS]))}}
        if timers is not None:
            # cycles of thread 0 of each subset's CTA, per subset of the timed steps
            names = ["subset", "gauss_newton_passes", "first_attempt", "sigma", "final_gamma",
                     "deformed_sum_beside_hessian_sweep", "q_sweep", "solve"]
            per = float(n) * args.steps
            line["section_timers"] = {"unit": "cycles per subset", "subsets": int(per),
                                      **{nm: timers[i] / per for i, nm in enumerate(names)}}
        print(json.dumps(line), flush=True)
    s.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


_FP32_PEAK = None


def fp32_peak_tflops(dev):
    """FP32 CUDA-core throughput measured with cuBLAS SGEMM (TF32 disabled)."""
    global _FP32_PEAK
    if _FP32_PEAK is not None:
        return _FP32_PEAK
    import torch
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 8192
        a = torch.randn(n, n, device=dev)
        b = torch.randn(n, n, device=dev)
        for _ in range(2):
            torch.mm(a, b)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        _FP32_PEAK = 2.0 * n ** 3 / (best / 1000.0) / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old
    return _FP32_PEAK


if __name__ == "__main__":
    main()
