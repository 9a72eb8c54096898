"""ctypes binding of libnufht_b200.so (the C ABI declared in include/nufht_b200.h).

The library is built in-tree by nufht_b200.build.  Importing this module raises if the
library is missing: there is no CPU fallback.
"""
import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnufht_b200.so")

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int_p = ctypes.POINTER(ctypes.c_int)


class NufhtOptions(ctypes.Structure):
    _fields_ = [("tol", ctypes.c_double), ("max_levels", ctypes.c_int), ("min_dim_prod", ctypes.c_int),
                ("z_split", ctypes.c_double), ("K_asy", ctypes.c_int), ("K_loc", ctypes.c_int)]


class Box(ctypes.Structure):
    _fields_ = [("i0", ctypes.c_int), ("i1", ctypes.c_int), ("j0", ctypes.c_int), ("j1", ctypes.c_int)]


class BoxVector(ctypes.Structure):
    _fields_ = [("data", ctypes.POINTER(Box)), ("length", ctypes.c_size_t), ("capacity", ctypes.c_size_t)]


class Boxes(ctypes.Structure):
    _fields_ = [("loc", BoxVector), ("asy", BoxVector), ("dir", BoxVector)]


class NufhtPlan(ctypes.Structure):
    _fields_ = [("nu", ctypes.c_double), ("tol", ctypes.c_double), ("z_split", ctypes.c_double),
                ("K_asy", ctypes.c_int), ("K_loc", ctypes.c_int), ("asy_coef", ctypes.c_double * 64),
                ("m", ctypes.c_int), ("n", ctypes.c_int), ("rs", c_double_p), ("ws", c_double_p),
                ("max_levels", ctypes.c_int), ("min_dim_prod", ctypes.c_int), ("boxes", Boxes),
                ("tables_loaded", ctypes.c_int)]


class NufhtScratch(ctypes.Structure):
    _fields_ = [(f, c_double_p) for f in ("in_buffer", "out_buffer", "real_buffer_1", "real_buffer_2",
                                          "cheb_buffer", "bessel_buffer_1", "bessel_buffer_2")] + \
               [(f, ctypes.c_int) for f in ("m_alloc", "n_alloc", "Kloc_alloc", "extra_alloc")]


class NufhtB200Info(ctypes.Structure):
    _fields_ = [("nu", ctypes.c_double), ("tol", ctypes.c_double), ("z_split", ctypes.c_double),
                ("K_asy", ctypes.c_int), ("K_loc", ctypes.c_int), ("n_loc", ctypes.c_long),
                ("n_asy", ctypes.c_long), ("n_dir", ctypes.c_long), ("fft_points", ctypes.c_long),
                ("spread_width", ctypes.c_int), ("path", ctypes.c_int), ("workspace_bytes", ctypes.c_size_t),
                ("mixed", ctypes.c_int)]


NUFHT_B200_FP64 = 0x0
NUFHT_B200_MIXED = 0x1
NUFHT_B200_MIXED_AVERAGED = 0x2
NUFHT_B200_EXTENDED_TABLES = 0x10
NUFHT_E_UNSORTED_RS = -410
NUFHT_E_UNSORTED_WS = -411
NUFHT_E_CUDA = -420
NUFHT_E_NO_DEVICE = -422
NUFHT_E_TOO_LARGE = -423
NUFHT_E_BAD_FLAGS = -424

class NufhtB200BatchItem(ctypes.Structure):
    _fields_ = [("plan", ctypes.c_void_p), ("cs", ctypes.c_void_p), ("ld_cs", ctypes.c_int),
                ("gs", ctypes.c_void_p), ("ld_gs", ctypes.c_int), ("batch", ctypes.c_int)]


_lib = None


def _declare(lib):
    vp = ctypes.c_void_p
    sig = {
        "nufht_default_options": (NufhtOptions, []),
        "boxes_free": (None, [ctypes.POINTER(Boxes)]),
        "generate_boxes": (Boxes, [c_double_p, ctypes.c_int, c_double_p, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int]),
        "split_box": (None, [c_double_p, ctypes.c_int, c_double_p, ctypes.c_int, ctypes.POINTER(Box),
                             ctypes.c_double, c_int_p, c_int_p]),
        "nufht_plan_init": (ctypes.c_int, [ctypes.POINTER(NufhtPlan), ctypes.c_double, vp, ctypes.c_int, vp,
                                           ctypes.c_int, ctypes.POINTER(NufhtOptions)]),
        "nufht_plan_free": (None, [ctypes.POINTER(NufhtPlan)]),
        "nufht_scratch_init": (ctypes.c_int, [ctypes.POINTER(NufhtScratch), ctypes.POINTER(NufhtPlan)]),
        "nufht_scratch_free": (None, [ctypes.POINTER(NufhtScratch)]),
        "nufht_batch": (ctypes.c_int, [ctypes.POINTER(NufhtPlan), vp, ctypes.c_int, vp, ctypes.c_int,
                                       ctypes.c_int, ctypes.POINTER(NufhtScratch)]),
        "nufht_inplace": (None, [vp, ctypes.c_double, vp, ctypes.c_int, vp, vp, ctypes.c_int,
                                 ctypes.POINTER(NufhtOptions)]),
        "nufht_b200_batch_layout": (ctypes.c_int, [ctypes.POINTER(NufhtPlan), vp, ctypes.c_int, ctypes.c_int, vp,
                                                   ctypes.c_int, ctypes.c_int, ctypes.c_int]),
        "nufht": (vp, [ctypes.c_double, vp, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.POINTER(NufhtOptions)]),
        "generate_tables": (None, []),
        "add_dir": (None, [vp, ctypes.c_double, vp, vp, vp, ctypes.c_int, ctypes.c_int]),
        "add_dir_batch": (None, [vp, ctypes.c_double, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int]),
        "add_asy": (None, [vp, ctypes.c_double, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                           ctypes.c_double, vp, vp, vp, vp, vp]),
        "add_asy_batch": (None, [vp, ctypes.c_double, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_double, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp]),
        "add_loc": (None, [vp, ctypes.c_double, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp]),
        "add_loc_batch": (None, [vp, ctypes.c_double, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp]),
        "nufht_b200_plan_create": (ctypes.c_int, [ctypes.POINTER(vp), ctypes.c_double, vp, ctypes.c_int, vp,
                                                  ctypes.c_int, ctypes.POINTER(NufhtOptions), ctypes.c_int,
                                                  ctypes.c_int]),
        "nufht_b200_execute": (ctypes.c_int, [vp, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp]),
        "nufht_b200_plan_info": (ctypes.c_int, [vp, ctypes.POINTER(NufhtB200Info)]),
        "nufht_b200_plan_destroy": (None, [vp]),
        "nufht_b200_plan_boxes": (ctypes.c_long, [vp, c_int_p, ctypes.c_long]),
        "nufht_b200_strerror": (ctypes.c_char_p, [ctypes.c_int]),
        "nufht_b200_launch_count": (ctypes.c_longlong, []),
        "nufht_b200_besselj": (ctypes.c_int, [ctypes.c_double, vp, vp, ctypes.c_long, vp]),
        "nufht_b200_table_source": (ctypes.c_char_p, []),
        "nufht_b200_write_tables": (ctypes.c_int, [ctypes.c_char_p]),
        "nufht_b200_set_phase_timing": (None, [ctypes.c_int]),
        "nufht_b200_plan_stats": (ctypes.c_int, [vp, c_double_p, ctypes.c_int]),
        "nufht_b200_fp64_peak": (ctypes.c_int, [c_double_p]),
        "nufht_b200_fp32_peak": (ctypes.c_int, [c_double_p]),
        "nufht_b200_add_loc_batch_noalloc": (ctypes.c_int, [vp, ctypes.c_double, vp, vp, vp, ctypes.c_int,
                                                            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                            ctypes.c_int, vp]),
        "nufht_b200_phase_times": (ctypes.c_int, [c_double_p, ctypes.c_int]),
        "nufht_b200_batch_create": (ctypes.c_int, [ctypes.POINTER(vp), ctypes.POINTER(NufhtB200BatchItem),
                                                   ctypes.c_int, ctypes.c_int]),
        "nufht_b200_batch_launch": (ctypes.c_int, [vp, vp]),
        "nufht_b200_batch_info": (ctypes.c_int, [vp, c_int_p, ctypes.POINTER(ctypes.c_float),
                                                 ctypes.POINTER(ctypes.c_long)]),
        "nufht_b200_batch_destroy": (None, [vp]),
        "nufht_b200_plan_buffers": (ctypes.c_int, [vp, ctypes.POINTER(vp), c_int_p, c_int_p]),
        "nufht_b200_generate_boxes_device": (ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_double,
                                                            ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                            ctypes.POINTER(Boxes)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def lib():
    """The loaded product library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libnufht_b200.so is not built; run `python -m nufht_b200.build` "
                               "(there is no CPU fallback)")
        _lib = _declare(ctypes.CDLL(LIB_PATH))
    return _lib


PHASES = ("zero", "loc_proj", "loc_eval", "asy_spread", "asy_fft", "asy_interp", "dir")


def phase_times():
    """Milliseconds per phase accumulated since timing was enabled (then reset)."""
    ms = np.zeros(len(PHASES))
    lib().nufht_b200_phase_times(ms.ctypes.data_as(c_double_p), len(PHASES))
    return dict(zip(PHASES, ms.tolist()))


def strerror(code):
    return lib().nufht_b200_strerror(int(code)).decode()


def options(tol=1e-8, max_levels=0, min_dim_prod=10000, z_split=math.nan, K_asy=0, K_loc=0):
    return NufhtOptions(tol, max_levels, min_dim_prod, z_split, K_asy, K_loc)


def dptr(a):
    """ctypes pointer to a float64 numpy array's data."""
    return a.ctypes.data_as(ctypes.c_void_p)


def as_f64(a, order="C"):
    return np.require(np.asarray(a, dtype=np.float64), dtype=np.float64, requirements=[order, "A"])


def boxes_to_array(boxes):
    """(loc, asy, dir) int arrays of shape (k, 4) from a Boxes struct."""
    out = []
    for v in (boxes.loc, boxes.asy, boxes.dir):
        a = np.zeros((v.length, 4), dtype=np.int64)
        for q in range(v.length):
            b = v.data[q]
            a[q] = (b.i0, b.i1, b.j0, b.j1)
        out.append(a)
    return tuple(out)
