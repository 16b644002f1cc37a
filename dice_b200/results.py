"""DICe text results through the C ABI (include/dicegpu_results.h).

`Output` writes what Schema::write_output / Output_Spec write
(DICe_Schema.cpp:4327-4478, 4673-4943); `diff_text` / `diff_files` compare
result files as DICe_Diff does (tools/DICe_Diff.cpp).
"""
import ctypes

import numpy as np

from . import abi


class OutputInfo(ctypes.Structure):
    _fields_ = [("ref_image", ctypes.c_char_p), ("def_image", ctypes.c_char_p), ("version", ctypes.c_char_p),
                ("subset_size", ctypes.c_int32), ("step_size_x", ctypes.c_int32), ("step_size_y", ctypes.c_int32),
                ("strain_window", ctypes.c_int32), ("incremental", ctypes.c_int32), ("sort_rows", ctypes.c_int32),
                ("initialization_method", ctypes.c_char_p)]


def _text(fn, *args):
    n = ctypes.c_size_t()
    abi.check(fn(*args, None, 0, ctypes.byref(n)), "output text")
    buf = ctypes.create_string_buffer(n.value + 1)
    abi.check(fn(*args, buf, n.value + 1, ctypes.byref(n)), "output text")
    return buf.value.decode()


class Output:
    """An output specification.  fields: column names (list or comma string),
    None for the reference's default columns."""

    def __init__(self, params, fields=None, delimiter=" ", omit_row_id=False, ref_image="", def_image="",
                 subset_size=None, step_size=(-1, -1), strain_window=-1, incremental=False, version=None,
                 sort_rows=False, initialization_method=None):
        self.lib = abi.load_library()
        if isinstance(fields, (list, tuple)):
            fields = ",".join(fields)
        info = OutputInfo(ref_image.encode(), def_image.encode(), version.encode() if version else None,
                          params.subset_size if subset_size is None else subset_size, step_size[0], step_size[1],
                          strain_window, int(incremental), int(sort_rows),
                          initialization_method.encode() if initialization_method else None)
        self._info = info
        h = ctypes.c_void_p()
        abi.check(self.lib.dicegpu_output_create(ctypes.byref(params), fields.encode() if fields else None,
                                                 delimiter.encode(), int(omit_row_id), ctypes.byref(info),
                                                 ctypes.byref(h)), "output_create")
        self.h = h

    def set_images(self, ref_image=None, def_image=None):
        abi.check(self.lib.dicegpu_output_set_images(self.h, ref_image.encode() if ref_image else None,
                                                     def_image.encode() if def_image else None), "set_images")

    def info_text(self):
        return _text(self.lib.dicegpu_output_info_text, self.h)

    def header_text(self, row_id="FRAME"):
        return _text(self.lib.dicegpu_output_header_text, self.h, row_id.encode())

    def row_text(self, row, fields_row, unc_row=None, vsg_row=None):
        f = np.ascontiguousarray(fields_row, np.float64)
        u = None if unc_row is None else np.ascontiguousarray(unc_row, np.float64)
        g = None if vsg_row is None else np.ascontiguousarray(vsg_row, np.float64)
        return _text(self.lib.dicegpu_output_row_text, self.h, int(row), f.ctypes.data_as(ctypes.c_void_p),
                     None if u is None else u.ctypes.data_as(ctypes.c_void_p),
                     None if g is None else g.ctypes.data_as(ctypes.c_void_p))

    def write_frame(self, folder, prefix, frame, fields, unc=None, vsg=None, first_frame=0, num_frames=0,
                    separate_files=True):
        f = np.ascontiguousarray(fields, np.float64)
        u = None if unc is None else np.ascontiguousarray(unc, np.float64)
        g = None if vsg is None else np.ascontiguousarray(vsg, np.float64)
        folder = str(folder)
        if folder and not folder.endswith("/"):
            folder += "/"
        abi.check(self.lib.dicegpu_output_write_frame(self.h, folder.encode(), prefix.encode(), frame, first_frame,
                                                      num_frames, f.shape[0], f.ctypes.data_as(ctypes.c_void_p),
                                                      None if u is None else u.ctypes.data_as(ctypes.c_void_p),
                                                      None if g is None else g.ctypes.data_as(ctypes.c_void_p),
                                                      int(separate_files)), "output_write_frame")

    def close(self):
        if getattr(self, "h", None):
            self.lib.dicegpu_output_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def diff_text(gold, result, tol=1.0e-6, floor=None, numerical_only=False):
    """(lines that differ, report) of DICe_Diff <gold> <result> -t tol [-f floor] [-n]."""
    lib = abi.load_library()
    a, b = gold.encode(), result.encode()
    failed = ctypes.c_int()
    rep = ctypes.create_string_buffer(1 << 16)
    abi.check(lib.dicegpu_diff_text(a, len(a), b, len(b), tol, floor or 0.0, int(floor is not None),
                                    int(numerical_only), ctypes.byref(failed), rep, len(rep)), "diff_text")
    return failed.value, rep.value.decode()


def diff_files(gold, result, tol=1.0e-6, floor=None, numerical_only=False, num_procs=1):
    lib = abi.load_library()
    failed = ctypes.c_int()
    rep = ctypes.create_string_buffer(1 << 16)
    abi.check(lib.dicegpu_diff_files(str(gold).encode(), str(result).encode(), tol, floor or 0.0,
                                     int(floor is not None), int(numerical_only), num_procs, ctypes.byref(failed),
                                     rep, len(rep)), "diff_files")
    return failed.value, rep.value.decode()
