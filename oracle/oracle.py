"""ctypes front end of the CPU oracle.

TEST INFRASTRUCTURE ONLY. Imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker. The shipped library
(openclipp_b200) never imports this module.

Two native libraries sit behind it, both built by oracle/Makefile:
  liborc.so            this repository's C restatement (proximity_oracle.c,
                       integral_oracle.c);
  _ref/libocl_ref.so   the reference's own cl-files/ImageProximity.cl and
                       cl-files/Integral.cl compiled unmodified as host C++
                       through ref_shim.h (built only where the reference
                       sources are present; the built file travels with the
                       repository).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# SImage::EDataType order (reference include/SImage.h:36-46).
TYPES = ["U8", "S8", "U16", "S16", "U32", "S32", "F32", "F64"]
NP_TYPES = [np.uint8, np.int8, np.uint16, np.int16, np.uint32, np.int32,
            np.float32, np.float64]
MEASURES = ["SqrDistance", "SqrDistance_Norm", "AbsDistance", "CrossCorr",
            "CrossCorr_Norm"]

_orc = None
_ref = None


def _lib_orc():
    global _orc
    if _orc is None:
        path = os.path.join(HERE, "liborc.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        _orc = ctypes.CDLL(path)
    return _orc


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libocl_ref.so"))


def _lib_ref():
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libocl_ref.so")
        if not os.path.exists(path):
            raise RuntimeError("reference kernels not built: run `make -C oracle ref`")
        _ref = ctypes.CDLL(path)
    return _ref


def type_index(arr):
    for i, t in enumerate(NP_TYPES):
        if arr.dtype == t:
            return i
    raise TypeError(f"unsupported pixel type {arr.dtype}")


def _img(a):
    """(H, W) or (H, W, C) array -> (ptr, step, W, H, C) in C order."""
    a = np.ascontiguousarray(a)
    if a.ndim == 2:
        h, w = a.shape
        c = 1
    else:
        h, w, c = a.shape
    return a, a.ctypes.data_as(ctypes.c_void_p), a.strides[0], w, h, c


def measure_index(measure):
    return MEASURES.index(measure) if isinstance(measure, str) else int(measure)


def real_dtype(src):
    return np.float64 if src.dtype == np.float64 else np.float32


_ref_fma = None


def _lib_ref_fma():
    global _ref_fma
    if _ref_fma is None:
        path = os.path.join(HERE, "_ref", "libocl_ref_fma.so")
        if not os.path.exists(path):
            raise RuntimeError("reference kernels not built: run `make -C oracle ref`")
        _ref_fma = ctypes.CDLL(path)
    return _ref_fma


def proximity_reference(measure, src, tmpl, mode=0, rows=None, fused=False):
    """Run the reference's own kernel source (through the shim).

    mode 0 = the reference host's choice (_Cached iff template <= 16x16),
    1 = plain kernel, 2 = _Cached kernel. rows = (begin, end) limits the
    computed band (other rows of the result stay 0). fused selects the build
    with FP contraction (every acc += a*b as one fma), as GPU OpenCL
    compilers build the kernels.
    """
    lib = _lib_ref_fma() if fused else _lib_ref()
    src, sp, ss, w, h, c = _img(src)
    tmpl, tp, ts, tw, th, tc = _img(tmpl)
    assert tc == c and tmpl.dtype == src.dtype
    out = np.zeros((h, w, c) if src.ndim == 3 else (h, w), dtype=real_dtype(src))
    fn = getattr(lib, f"ocl_ref_proximity_{TYPES[type_index(src)]}_C{c}")
    r0, r1 = rows if rows else (0, h)
    rc = fn(measure_index(measure), sp, ss, tp, ts,
            out.ctypes.data_as(ctypes.c_void_p), out.strides[0], w, h, tw, th,
            mode, r0, r1)
    if rc:
        raise RuntimeError(f"reference kernel returned {rc}")
    return out


def integral_reference(src, sqr, dst_f64):
    """Run the reference's Integral.cl pipeline (1 channel)."""
    lib = _lib_ref()
    src, sp, ss, w, h, c = _img(src)
    assert c == 1
    out = np.zeros((h, w), dtype=np.float64 if dst_f64 else np.float32)
    fn = getattr(lib, f"ocl_ref_integral_{TYPES[type_index(src)].lower()}")
    rc = fn(int(sqr), sp, ss, out.ctypes.data_as(ctypes.c_void_p),
            out.strides[0], int(dst_f64), w, h)
    if rc:
        raise RuntimeError(f"reference integral returned {rc}")
    return out


def proximity_refexact(measure, src, tmpl, rows=None, fused=False):
    """This repository's restatement of the reference arithmetic (REAL);
    fused=True evaluates each acc += a*b as fma(a, b, acc)."""
    lib = _lib_orc()
    src, sp, ss, w, h, c = _img(src)
    tmpl, tp, ts, tw, th, tc = _img(tmpl)
    assert tc == c and tmpl.dtype == src.dtype
    out = np.zeros((h, w, c) if src.ndim == 3 else (h, w), dtype=real_dtype(src))
    r0, r1 = rows if rows else (0, h)
    rc = lib.orc_proximity_refexact(measure_index(measure), type_index(src), c,
                                    sp, ss, tp, ts,
                                    out.ctypes.data_as(ctypes.c_void_p),
                                    out.strides[0], w, h, tw, th, r0, r1,
                                    int(bool(fused)))
    if rc:
        raise RuntimeError(f"oracle returned {rc}")
    return out


def proximity_exact(measure, src, tmpl):
    """Exact (integer) / long double (float) value, as float64."""
    lib = _lib_orc()
    src, sp, ss, w, h, c = _img(src)
    tmpl, tp, ts, tw, th, tc = _img(tmpl)
    assert tc == c and tmpl.dtype == src.dtype
    out = np.zeros((h, w, c) if src.ndim == 3 else (h, w), dtype=np.float64)
    rc = lib.orc_proximity_exact(measure_index(measure), type_index(src), c,
                                 sp, ss, tp, ts,
                                 out.ctypes.data_as(ctypes.c_void_p), w, h, tw, th)
    if rc:
        raise RuntimeError(f"oracle returned {rc}")
    return out


def proximity_exact_rows(measure, src, tmpl, rows):
    """proximity_exact for the listed output rows only: float64 array of
    shape (len(rows), W[, C]), row i holding output row rows[i]."""
    lib = _lib_orc()
    src, sp, ss, w, h, c = _img(src)
    tmpl, tp, ts, tw, th, tc = _img(tmpl)
    assert tc == c and tmpl.dtype == src.dtype
    r = np.ascontiguousarray(rows, dtype=np.int32)
    out = np.zeros((len(r), w, c) if src.ndim == 3 else (len(r), w), dtype=np.float64)
    rc = lib.orc_proximity_exact_rows(measure_index(measure), type_index(src), c,
                                      sp, ss, tp, ts,
                                      out.ctypes.data_as(ctypes.c_void_p), w, h, tw, th,
                                      r.ctypes.data_as(ctypes.c_void_p), len(r))
    if rc:
        raise RuntimeError(f"oracle returned {rc}")
    return out


def window_terms_exact(src, tmpl):
    """(sum S^2 per window, sum S*T per window, sum T^2 per channel)."""
    lib = _lib_orc()
    src, sp, ss, w, h, c = _img(src)
    tmpl, tp, ts, tw, th, tc = _img(tmpl)
    shape = (h, w, c) if src.ndim == 3 else (h, w)
    e = np.zeros(shape, np.float64)
    x = np.zeros(shape, np.float64)
    t = np.zeros(c, np.float64)
    rc = lib.orc_window_terms_exact(type_index(src), c, sp, ss, tp, ts,
                                    e.ctypes.data_as(ctypes.c_void_p),
                                    x.ctypes.data_as(ctypes.c_void_p),
                                    t.ctypes.data_as(ctypes.c_void_p), w, h, tw, th)
    if rc:
        raise RuntimeError(f"oracle returned {rc}")
    return e, x, t


INDEX_OPS = {"MinIndx": 0, "MaxIndx": 1, "MinAbsIndx": 2, "MaxAbsIndx": 3}


def index_reduce(name, src):
    """(value, x, y) of ocip<name> on a one-channel image, in the
    reference's comparison order."""
    lib = _lib_orc()
    src, sp, ss, w, h, c = _img(src)
    assert c == 1
    v, x, y = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
    rc = lib.orc_index_reduce(INDEX_OPS[name], type_index(src), sp, ss, w, h, ctypes.byref(v),
                              ctypes.byref(x), ctypes.byref(y))
    if rc:
        raise RuntimeError(f"oracle returned {rc}")
    return v.value, x.value, y.value


def integral_exact(src, sqr):
    lib = _lib_orc()
    src, sp, ss, w, h, c = _img(src)
    out = np.zeros((h, w, c) if src.ndim == 3 else (h, w), dtype=np.float64)
    rc = lib.orc_integral_exact(int(sqr), type_index(src), c, sp, ss,
                                out.ctypes.data_as(ctypes.c_void_p), w, h)
    if rc:
        raise RuntimeError(f"oracle returned {rc}")
    return out


def proximity_backward(measure, S, T, g):
    """Long double adjoints (dS, dT) of SqrDistance / CrossCorr_Norm."""
    lib = _lib_orc()
    S = np.ascontiguousarray(S, dtype=np.float64)
    T = np.ascontiguousarray(T, dtype=np.float64)
    g = np.ascontiguousarray(g, dtype=np.float64)
    h, w = S.shape
    th, tw = T.shape
    dS = np.zeros_like(S)
    dT = np.zeros_like(T)
    rc = lib.orc_proximity_backward(measure_index(measure),
                                    S.ctypes.data_as(ctypes.c_void_p),
                                    T.ctypes.data_as(ctypes.c_void_p),
                                    g.ctypes.data_as(ctypes.c_void_p),
                                    dS.ctypes.data_as(ctypes.c_void_p),
                                    dT.ctypes.data_as(ctypes.c_void_p),
                                    w, h, tw, th)
    if rc:
        raise RuntimeError(f"oracle returned {rc}")
    return dS, dT
