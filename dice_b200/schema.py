"""Python mirror of the reference's Schema boundary over libdicegpu.so.

    schema = Schema(params)                    # DICe::Schema(..., params)
    schema.set_ref_image(ref)                  # Schema::set_ref_image(w, h, array)
    schema.set_subsets(cx, cy)                 # subset centroids (COORDINATES_X/Y fields)
    schema.set_def_image(deformed)             # Schema::set_def_image(w, h, array)
    schema.execute_correlation()               # Schema::execute_correlation()
    u = schema.field(abi.F_DISP_X)             # global_field_value(i, SUBSET_DISPLACEMENT_X_FS)

Every call goes through the C ABI; images may be numpy arrays (host) or
torch CUDA tensors (device pointers, no copy through the host).
"""
import ctypes

import numpy as np

from . import abi


def _as_host_f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _is_cuda_tensor(a):
    try:
        import torch
        return isinstance(a, torch.Tensor) and a.is_cuda
    except Exception:
        return False


class Schema:
    def __init__(self, params=None, stream=None):
        self.lib = abi.load_library()
        self.params = params.copy() if params is not None else abi.default_params()
        self.ctx = ctypes.c_void_p()
        abi.check(self.lib.dicegpu_create(ctypes.byref(self.params), ctypes.byref(self.ctx)),
                  "dicegpu_create")
        self.n = 0
        self.w = self.h = 0
        self._keep = []
        if stream is not None:
            self.set_stream(stream)

    def close(self):
        if self.ctx:
            self.lib.dicegpu_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- configuration ------------------------------------------------------
    def set_params(self, params):
        self.params = params.copy()
        abi.check(self.lib.dicegpu_set_params(self.ctx, ctypes.byref(self.params)), "set_params")

    def set_stream(self, stream):
        """stream: a cudaStream_t handle (int) or a torch.cuda.Stream."""
        h = getattr(stream, "cuda_stream", stream)
        abi.check(self.lib.dicegpu_set_stream(self.ctx, ctypes.c_void_p(int(h))), "set_stream")

    def set_launch_shape(self, warps_per_cta=0, ctas_per_sm=0):
        abi.check(self.lib.dicegpu_set_launch_shape(self.ctx, warps_per_cta, ctas_per_sm),
                  "set_launch_shape")

    def launch_shape(self):
        a, b = ctypes.c_int(), ctypes.c_int()
        abi.check(self.lib.dicegpu_get_launch_shape(self.ctx, ctypes.byref(a), ctypes.byref(b)),
                  "get_launch_shape")
        return a.value, b.value

    # ---- images ---------------------------------------------------------------
    def _image_call(self, fn, img, what):
        # 8- and 16-bit images go through the typed entry points (converted on
        # the device, the raw bytes are what crosses PCIe)
        typed = {"uint8": abi.PIXEL_U8, "uint16": abi.PIXEL_U16}
        dt = str(img.dtype).replace("torch.", "")
        if dt in typed:
            tfn = self.lib.dicegpu_set_ref_image_typed if "ref" in what else self.lib.dicegpu_set_def_image_typed
            if _is_cuda_tensor(img):
                t = img.contiguous()
                self._keep.append(t)
                h, w = t.shape
                rc = tfn(self.ctx, w, h, ctypes.c_void_p(t.data_ptr()), typed[dt], 1)
            else:
                a = np.ascontiguousarray(img)
                self._keep.append(a)
                h, w = a.shape
                rc = tfn(self.ctx, w, h, a.ctypes.data_as(ctypes.c_void_p), typed[dt], 0)
            abi.check(rc, what)
            self.w, self.h = w, h
            return
        if _is_cuda_tensor(img):
            t = img.contiguous().float()
            h, w = t.shape
            self._keep.append(t)
            rc = fn(self.ctx, w, h, ctypes.c_void_p(t.data_ptr()), 1)
        else:
            a = _as_host_f32(img)
            h, w = a.shape
            rc = fn(self.ctx, w, h, a.ctypes.data_as(ctypes.c_void_p), 0)
        abi.check(rc, what)
        self.w, self.h = w, h

    def set_ref_image(self, img):
        self._image_call(self.lib.dicegpu_set_ref_image, img, "set_ref_image")

    def set_def_image(self, img):
        self._image_call(self.lib.dicegpu_set_def_image, img, "set_def_image")
        if len(self._keep) > 4:
            self._keep = self._keep[-4:]

    def set_neighbors(self, neighbor_ids):
        """NEIGHBOR_ID per subset (None clears) for the neighbour initializers."""
        if neighbor_ids is None:
            abi.check(self.lib.dicegpu_set_neighbors(self.ctx, None), "set_neighbors")
            return
        nb = np.ascontiguousarray(neighbor_ids, dtype=np.int32)
        assert nb.shape == (self.n,)
        abi.check(self.lib.dicegpu_set_neighbors(self.ctx, nb.ctypes.data_as(ctypes.c_void_p)), "set_neighbors")

    def set_ref_from_def(self):
        """Incremental sequences: the current deformed image becomes the
        reference (Schema::set_ref_image(prev_img()))."""
        abi.check(self.lib.dicegpu_set_ref_from_def(self.ctx), "set_ref_from_def")

    # ---- subsets ----------------------------------------------------------------
    def set_fields(self, fields):
        f = np.ascontiguousarray(fields, dtype=np.float64)
        assert f.ndim == 2 and f.shape[1] == abi.FIELD_STRIDE
        abi.check(self.lib.dicegpu_set_subsets(self.ctx, f.shape[0], f.ctypes.data_as(ctypes.c_void_p)),
                  "set_subsets")
        self.n = f.shape[0]

    def set_subsets(self, cx, cy, quadratic=None):
        from .synthetic import init_fields
        if quadratic is None:
            quadratic = self.params.shape_function == abi.QUADRATIC_SF
        self.set_fields(init_fields(np.asarray(cx, np.float64), np.asarray(cy, np.float64), quadratic))

    def set_subset_pixels(self, offsets, px, py):
        o = np.ascontiguousarray(offsets, dtype=np.int32)
        x = np.ascontiguousarray(px, dtype=np.int32)
        y = np.ascontiguousarray(py, dtype=np.int32)
        abi.check(self.lib.dicegpu_set_subset_pixels(self.ctx, self.n, o.ctypes.data_as(ctypes.c_void_p),
                                                     x.ctypes.data_as(ctypes.c_void_p),
                                                     y.ctypes.data_as(ctypes.c_void_p)), "set_subset_pixels")

    def set_subset_shapes(self, shapes, vx=None, vy=None):
        """Builds every subset's pixel list on the device from its shapes
        (abi.circle / rectangle / polygon; polygons index vx, vy)."""
        arr = abi.shape_array(list(shapes))
        x = np.ascontiguousarray(vx if vx is not None else [0], dtype=np.int32)
        y = np.ascontiguousarray(vy if vy is not None else [0], dtype=np.int32)
        abi.check(self.lib.dicegpu_set_subset_shapes(self.ctx, len(arr), ctypes.cast(arr, ctypes.c_void_p),
                                                     x.ctypes.data_as(ctypes.c_void_p),
                                                     y.ctypes.data_as(ctypes.c_void_p)), "set_subset_shapes")

    def set_blocking(self, blockers):
        """Blocking subsets: blockers[i] lists the subsets that may block
        subset i (BLOCKING_SUBSETS); None clears them."""
        if blockers is None:
            abi.check(self.lib.dicegpu_set_blocking(self.ctx, None, None), "set_blocking")
            return
        offs = np.zeros(self.n + 1, np.int32)
        ids = []
        for i in range(self.n):
            b = list(blockers[i]) if i < len(blockers) and blockers[i] is not None else []
            ids += b
            offs[i + 1] = offs[i] + len(b)
        ida = np.ascontiguousarray(ids if ids else [0], dtype=np.int32)
        abi.check(self.lib.dicegpu_set_blocking(self.ctx, offs.ctypes.data_as(ctypes.c_void_p),
                                                ida.ctypes.data_as(ctypes.c_void_p)), "set_blocking")

    def vsg_strain(self, window_size):
        """VSG_Strain_Post_Processor on the current field rows: n x VSG_STRIDE
        (strain xx, yy, xy, du/dx, du/dy, dv/dx, dv/dy, valid neighbours);
        sets MATCH = -1 where the fit fails.  A negative window_size takes the
        -window_size nearest subsets as the neighbourhood."""
        out = np.zeros((self.n, abi.VSG_STRIDE), np.float64)
        abi.check(self.lib.dicegpu_vsg_strain(self.ctx, int(window_size), out.ctypes.data_as(ctypes.c_void_p), 0),
                  "vsg_strain")
        return out

    def subset_pixels(self):
        """(offsets, px, py) of the context's subset pixel lists."""
        offs = np.zeros(self.n + 1, np.int32)
        abi.check(self.lib.dicegpu_get_subset_pixels(self.ctx, offs.ctypes.data_as(ctypes.c_void_p), None, None),
                  "get_subset_pixels")
        px = np.zeros(max(int(offs[-1]), 1), np.int32)
        py = np.zeros_like(px)
        abi.check(self.lib.dicegpu_get_subset_pixels(self.ctx, offs.ctypes.data_as(ctypes.c_void_p),
                                                     px.ctypes.data_as(ctypes.c_void_p),
                                                     py.ctypes.data_as(ctypes.c_void_p)), "get_subset_pixels")
        return offs, px[:offs[-1]], py[:offs[-1]]

    def subset_pixel_state(self):
        """(state, ref_values) of the list pixels under subset evolution:
        state 0 inactive, 1 active, 2 turned on with reference intensity
        ref_values (Subset::turn_on_previously_obstructed_pixels)."""
        offs = np.zeros(self.n + 1, np.int32)
        abi.check(self.lib.dicegpu_get_subset_pixels(self.ctx, offs.ctypes.data_as(ctypes.c_void_p), None, None),
                  "get_subset_pixels")
        state = np.zeros(max(int(offs[-1]), 1), np.uint8)
        vals = np.zeros(max(int(offs[-1]), 1), np.float32)
        abi.check(self.lib.dicegpu_get_subset_pixel_state(self.ctx, state.ctypes.data_as(ctypes.c_void_p),
                                                          vals.ctypes.data_as(ctypes.c_void_p)),
                  "get_subset_pixel_state")
        return state[:offs[-1]], vals[:offs[-1]]

    def set_force_simplex(self, flags):
        if flags is None:
            abi.check(self.lib.dicegpu_set_force_simplex(self.ctx, 0, None), "set_force_simplex")
            return
        a = np.ascontiguousarray(flags, dtype=np.uint8)
        abi.check(self.lib.dicegpu_set_force_simplex(self.ctx, a.shape[0], a.ctypes.data_as(ctypes.c_void_p)),
                  "set_force_simplex")

    def set_skip_solve(self, flags):
        """Per-subset flags (non-zero: only evaluate the initial guess and
        record FRAME_SKIPPED) for the following frames; None clears them."""
        if flags is None:
            abi.check(self.lib.dicegpu_set_skip_solve(self.ctx, 0, None), "set_skip_solve")
            return
        a = np.ascontiguousarray(np.asarray(flags) != 0, dtype=np.uint8)
        abi.check(self.lib.dicegpu_set_skip_solve(self.ctx, a.shape[0], a.ctypes.data_as(ctypes.c_void_p)),
                  "set_skip_solve")

    # ---- execution ----------------------------------------------------------------
    def execute_correlation(self):
        abi.check(self.lib.dicegpu_execute_correlation(self.ctx), "execute_correlation")

    def execute_correlation_plain(self):
        abi.check(self.lib.dicegpu_execute_correlation_plain(self.ctx), "execute_correlation_plain")

    def capture_sequence(self, frames, reset_fields=None):
        """Records a frame sequence (list of CUDA tensors) as one CUDA graph."""
        self._seq = [f.contiguous().float() for f in frames]
        ptrs = (ctypes.c_void_p * len(self._seq))(*[f.data_ptr() for f in self._seq])
        self._seq_ptrs = ptrs
        self._seq_reset = reset_fields
        rp = ctypes.c_void_p(reset_fields.data_ptr()) if reset_fields is not None else None
        abi.check(self.lib.dicegpu_capture_sequence(self.ctx, len(self._seq), ptrs, rp), "capture_sequence")

    def launch_sequence(self):
        abi.check(self.lib.dicegpu_launch_sequence(self.ctx), "launch_sequence")

    def autotune(self):
        w, c, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        abi.check(self.lib.dicegpu_autotune(self.ctx, ctypes.byref(w), ctypes.byref(c), ctypes.byref(ms)),
                  "autotune")
        return w.value, c.value, ms.value

    def fields(self):
        out = np.zeros((self.n, abi.FIELD_STRIDE), np.float64)
        abi.check(self.lib.dicegpu_get_fields(self.ctx, out.ctypes.data_as(ctypes.c_void_p)), "get_fields")
        return out

    def field(self, col):
        return self.fields()[:, col]

    def _fit(self, entry, fields):
        f = np.ascontiguousarray(fields, dtype=np.float64).copy()
        assert f.shape == (self.n, abi.FIELD_STRIDE)
        it = np.zeros(self.n, np.int32)
        st = np.zeros(self.n, np.int32)
        vp = ctypes.c_void_p
        abi.check(getattr(self.lib, entry)(self.ctx, f.ctypes.data_as(vp), it.ctypes.data_as(vp),
                                            st.ctypes.data_as(vp)), entry)
        return f, it, st

    def compute_update_fast(self, fields):
        """Objective_ZNSSD::computeUpdateFast per subset from the parameters in
        `fields`: returns (updated fields, iterations, Status_Flag)."""
        return self._fit("dicegpu_compute_update_fast", fields)

    def compute_update_robust(self, fields):
        """Objective::computeUpdateRobust (simplex) per subset: returns
        (updated fields, iterations, Status_Flag)."""
        return self._fit("dicegpu_compute_update_robust", fields)

    def sigma(self, fields):
        """Objective::sigma per subset at the parameters in `fields`:
        returns (sigma, noise_std_dev)."""
        f = np.ascontiguousarray(fields, dtype=np.float64)
        sg = np.zeros(self.n, np.float64)
        no = np.zeros(self.n, np.float64)
        vp = ctypes.c_void_p
        abi.check(self.lib.dicegpu_sigma(self.ctx, f.ctypes.data_as(vp), sg.ctypes.data_as(vp),
                                         no.ctypes.data_as(vp)), "sigma")
        return sg, no

    def adjoint(self, fields, seed=None, objective=0, grad_source=0, ddef=None):
        """dicegpu_adjoint on CUDA tensors: `fields` (n x FIELD_STRIDE float64)
        holds each subset's parameters, `seed` (n float64) weights the
        objectives, `ddef` (H x W float32) receives the derivative with
        respect to the deformed image (added).  Returns (value, dparams):
        n objective values and n x 12 derivatives in parameter-slot order.
        Ordered after the caller's current stream's work."""
        import torch
        assert fields.is_cuda and fields.dtype == torch.float64 and fields.is_contiguous()
        assert fields.shape == (self.n, abi.FIELD_STRIDE)
        value = torch.empty(self.n, dtype=torch.float64, device=fields.device)
        dparams = torch.empty((self.n, 12), dtype=torch.float64, device=fields.device)
        vp = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())  # noqa: E731
        if seed is not None:
            assert seed.is_cuda and seed.dtype == torch.float64 and seed.is_contiguous()
        if ddef is not None:
            assert ddef.is_cuda and ddef.dtype == torch.float32 and ddef.is_contiguous()
        self.set_stream(torch.cuda.current_stream())
        abi.check(self.lib.dicegpu_adjoint(self.ctx, vp(fields), vp(seed), int(objective), int(grad_source),
                                           vp(value), vp(dparams), vp(ddef)), "adjoint")
        return value, dparams

    def uncertainty(self):
        """FIELD_1..FIELD_7 of Objective::computeUncertaintyFields per subset
        (n x UNCERTAINTY_STRIDE); needs params.compute_uncertainty = 1."""
        out = np.zeros((self.n, abi.UNCERTAINTY_STRIDE), np.float64)
        abi.check(self.lib.dicegpu_get_uncertainty(self.ctx, out.ctypes.data_as(ctypes.c_void_p)),
                  "get_uncertainty")
        return out

    def load_fields(self, src):
        """Asynchronous reload of all fields (numpy host array or CUDA tensor); restarts at frame 0."""
        if _is_cuda_tensor(src):
            abi.check(self.lib.dicegpu_load_fields(self.ctx, ctypes.c_void_p(src.data_ptr()), 1), "load_fields")
        else:
            a = np.ascontiguousarray(src, dtype=np.float64)
            self._keep.append(a)
            abi.check(self.lib.dicegpu_load_fields(self.ctx, a.ctypes.data_as(ctypes.c_void_p), 0), "load_fields")

    def store_fields(self, dst):
        """Asynchronous copy of all fields into a CUDA tensor or pinned host tensor (no sync)."""
        on_dev = 1 if _is_cuda_tensor(dst) else 0
        abi.check(self.lib.dicegpu_store_fields(self.ctx, ctypes.c_void_p(dst.data_ptr()), on_dev), "store_fields")

    def fields_device_ptr(self):
        p = ctypes.c_void_p()
        abi.check(self.lib.dicegpu_fields_device_ptr(self.ctx, ctypes.byref(p)), "fields_device_ptr")
        return p.value

    def launch_count(self):
        c = ctypes.c_int64()
        abi.check(self.lib.dicegpu_launch_count(self.ctx, ctypes.byref(c)), "launch_count")
        return c.value

    def device_status(self):
        s = ctypes.c_int32()
        abi.check(self.lib.dicegpu_device_status(self.ctx, ctypes.byref(s)), "device_status")
        return s.value

    def gamma(self, fields):
        f = np.ascontiguousarray(fields, dtype=np.float64)
        out = np.zeros(f.shape[0], np.float64)
        abi.check(self.lib.dicegpu_gamma(self.ctx, f.ctypes.data_as(ctypes.c_void_p),
                                         out.ctypes.data_as(ctypes.c_void_p)), "gamma")
        return out

    def interpolate(self, method, xy, gradients=True):
        xy = np.ascontiguousarray(xy, dtype=np.float32).reshape(-1, 2)
        n = xy.shape[0]
        oi = np.zeros(n, np.float32)
        gx = np.zeros(n, np.float32) if gradients else None
        gy = np.zeros(n, np.float32) if gradients else None
        p = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)
        abi.check(self.lib.dicegpu_interpolate(self.ctx, method, n, p(xy), p(oi), p(gx), p(gy), 0),
                  "interpolate")
        return oi, gx, gy


def correlate(points, subset_size, ref, deff, params=None, update_params=False):
    """dice_correlate mirror: points is an (n, 9) float32 array updated in
    place.  The library keeps one context across calls, as the reference keeps
    a static Schema: the first call fixes the reference image, subset size and
    subsets; later calls correlate `deff` as the next frame and read `params`
    again only with update_params.  correlate_reset() starts over."""
    lib = abi.load_library()
    pts = np.ascontiguousarray(points, dtype=np.float32)
    ref = _as_host_f32(ref)
    deff = _as_host_f32(deff)
    h, w = ref.shape
    dh, dw = deff.shape
    rc = lib.dicegpu_correlate(pts.ctypes.data_as(ctypes.c_void_p), pts.shape[0], subset_size,
                               ref.ctypes.data_as(ctypes.c_void_p), w, h,
                               deff.ctypes.data_as(ctypes.c_void_p), dw, dh,
                               ctypes.byref(params) if params is not None else None, int(bool(update_params)))
    if rc == 0:
        points[...] = pts
    return rc


def correlate_reset():
    """Releases the context `correlate` keeps (dicegpu_correlate_reset)."""
    return abi.load_library().dicegpu_correlate_reset()
