"""ctypes mirror of the ocip* C interface (include/OpenCLIPP.h,
include/OpenCLIPP_B200.h).

Every function calls straight into libopenclipp_b200.so; there is no other
implementation behind this module. Importing it fails if the library has not
been built (python -m openclipp_b200.build).

Names follow the C interface: `Context` wraps ocipInitialize/ocipUninitialize,
`Image` wraps ocipCreateImage/ocipSendImage/ocipReadImage/ocipReleaseImage
around a numpy array that stays the host buffer of the image, and the
measure functions (`sqr_distance`, ..., `cross_corr_norm`) call the
identically named ocip* entry points.
"""
import ctypes
import os

import numpy as np

from . import LIBRARY_PATH

# SImage::EDataType (include/SImage.h)
U8, S8, U16, S16, U32, S32, F32, F64 = range(8)
NP_OF_TYPE = {U8: np.uint8, S8: np.int8, U16: np.uint16, S16: np.int16,
              U32: np.uint32, S32: np.int32, F32: np.float32, F64: np.float64}
TYPE_OF_NP = {np.dtype(v): k for k, v in NP_OF_TYPE.items()}

CL_SUCCESS = 0
CL_DEVICE_NOT_FOUND = -1
CL_MEM_OBJECT_ALLOCATION_FAILURE = -4
CL_OUT_OF_RESOURCES = -5
CL_IMAGE_FORMAT_MISMATCH = -9
CL_IMAGE_FORMAT_NOT_SUPPORTED = -10
CL_INVALID_VALUE = -30
CL_INVALID_CONTEXT = -34
CL_INVALID_MEM_OBJECT = -38
CL_INVALID_IMAGE_SIZE = -40
CL_INVALID_PROGRAM = -44
CL_INVALID_OPERATION = -59
CL_INVALID_BUFFER_SIZE = -61
CL_DEVICE_TYPE_GPU = 1 << 2
CL_DEVICE_TYPE_ALL = 0xFFFFFFFF
CL_MEM_READ_WRITE = 1

PATH_AUTO, PATH_PLAIN, PATH_TENSOR = 0, 1, 2

MEASURES = ("SqrDistance", "SqrDistance_Norm", "AbsDistance", "CrossCorr",
            "CrossCorr_Norm")


class SImage(ctypes.Structure):
    _fields_ = [("Width", ctypes.c_uint), ("Height", ctypes.c_uint),
                ("Step", ctypes.c_uint), ("Channels", ctypes.c_uint),
                ("Type", ctypes.c_int)]


def _load():
    if not os.path.exists(LIBRARY_PATH):
        raise ImportError(
            f"{LIBRARY_PATH} is missing: build it with `python -m openclipp_b200.build`")
    lib = ctypes.CDLL(LIBRARY_PATH)
    vp, i32, u32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint
    sig = {
        "ocipInitialize": (i32, [ctypes.POINTER(vp), ctypes.c_char_p, ctypes.c_uint64]),
        "ocipUninitialize": (i32, [vp]),
        "ocipChangeContext": (i32, [vp]),
        "ocipSetCLFilesPath": (None, [ctypes.c_char_p]),
        "ocipGetErrorName": (ctypes.c_char_p, [i32]),
        "ocipGetDeviceName": (i32, [ctypes.c_char_p, u32]),
        "ocipFinish": (i32, []),
        "ocipCreateImage": (i32, [ctypes.POINTER(vp), SImage, vp, ctypes.c_uint64]),
        "ocipSendImage": (i32, [vp]),
        "ocipReadImage": (i32, [vp]),
        "ocipReleaseImage": (i32, [vp]),
        "ocipReleaseProgram": (i32, [vp]),
        "ocipPrepareIntegral": (i32, [ctypes.POINTER(vp), vp]),
        "ocipIntegral": (i32, [vp, vp, vp]),
        "ocipSqrIntegral": (i32, [vp, vp, vp]),
        "ocipPrepareProximity": (i32, [vp]),
        "ocipSqrDistance_Norm": (i32, [vp, vp, vp]),
        "ocipSqrDistance": (i32, [vp, vp, vp]),
        "ocipAbsDistance": (i32, [vp, vp, vp]),
        "ocipCrossCorr": (i32, [vp, vp, vp]),
        "ocipCrossCorr_Norm": (i32, [vp, vp, vp]),
        "ocipIsFFTAvailable": (ctypes.c_char, []),
        "ocipPrepareImageProximityFFT": (i32, [ctypes.POINTER(vp), vp, vp]),
        "ocipSqrDistanceFFT": (i32, [vp, vp, vp, vp]),
        "ocipSqrDistanceFFT_Norm": (i32, [vp, vp, vp, vp]),
        "ocipCrossCorrFFT": (i32, [vp, vp, vp, vp]),
        "ocipCrossCorrFFT_Norm": (i32, [vp, vp, vp, vp]),
        "ocipSetProximityPath": (i32, [ctypes.c_int]),
        "ocipGetProximityPath": (i32, [ctypes.POINTER(ctypes.c_int)]),
        "ocipGetLastProximityPath": (i32, [ctypes.POINTER(ctypes.c_int)]),
        "ocipSetProximityBandHeight": (i32, [ctypes.c_int]),
        "ocipGetLastErrorMessage": (ctypes.c_char_p, []),
        "ocipGetStream": (i32, [ctypes.POINTER(vp)]),
        "ocipGetImageDevicePtr": (i32, [vp, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_size_t)]),
        "ocipGetLaunchCount": (i32, [ctypes.POINTER(ctypes.c_uint64)]),
        "ocipProximityIndx": (i32, [ctypes.c_int, ctypes.c_int, vp, vp, vp,
                                    ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_int)]),
        "ocipIntegralNoAlloc": (i32, [ctypes.c_int, SImage, vp, ctypes.c_size_t, SImage, vp,
                                      ctypes.c_size_t, vp]),
        "ocipPrepareProximityBatch": (i32, [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp),
                                            ctypes.c_int, ctypes.POINTER(vp), ctypes.c_int,
                                            ctypes.POINTER(vp)]),
        "ocipRunProximityBatch": (i32, [vp]),
        "ocipProximityBackward": (i32, [vp, vp, vp, vp, vp, vp, vp]),
        "ocipTestBoundedWait": (i32, [ctypes.c_int]),
        "ocipPrepareStatistics": (i32, [ctypes.POINTER(vp), vp]),
        "ocipMinIndx": (i32, [vp, vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                              ctypes.POINTER(ctypes.c_int)]),
        "ocipMaxIndx": (i32, [vp, vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                              ctypes.POINTER(ctypes.c_int)]),
        "ocipMinAbsIndx": (i32, [vp, vp, ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
        "ocipMaxAbsIndx": (i32, [vp, vp, ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
        "ocipGetProximityBand": (i32, [u32, u32, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(u32)]),
        "ocipGetProximityBatchInfo": (i32, [vp, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class OcipError(RuntimeError):
    def __init__(self, code, where):
        self.code = code
        self.name = lib.ocipGetErrorName(code).decode()
        detail = (lib.ocipGetLastErrorMessage() or b"").decode()
        super().__init__(f"{where}: {self.name} ({code}) {detail}")


def check(code, where=""):
    if code != CL_SUCCESS:
        raise OcipError(code, where)
    return code


def launch_count():
    """Kernels launched by the library so far (ocipGetLaunchCount)."""
    n = ctypes.c_uint64()
    check(lib.ocipGetLaunchCount(ctypes.byref(n)), "ocipGetLaunchCount")
    return n.value


def error_name(code):
    return lib.ocipGetErrorName(code).decode()


class Context:
    """ocipInitialize / ocipUninitialize; current context while open."""

    def __init__(self, device=None, device_type=CL_DEVICE_TYPE_GPU):
        self.handle = ctypes.c_void_p()
        plat = None if device is None else str(device).encode()
        check(lib.ocipInitialize(ctypes.byref(self.handle), plat, device_type),
              "ocipInitialize")

    def make_current(self):
        check(lib.ocipChangeContext(self.handle), "ocipChangeContext")

    def set_path(self, path):
        check(lib.ocipSetProximityPath(path), "ocipSetProximityPath")

    def set_band_height(self, rows):
        check(lib.ocipSetProximityBandHeight(rows), "ocipSetProximityBandHeight")

    def last_path(self):
        v = ctypes.c_int()
        check(lib.ocipGetLastProximityPath(ctypes.byref(v)), "ocipGetLastProximityPath")
        return v.value

    def finish(self):
        check(lib.ocipFinish(), "ocipFinish")

    def stream(self):
        s = ctypes.c_void_p()
        check(lib.ocipGetStream(ctypes.byref(s)), "ocipGetStream")
        return s.value or 0

    def device_name(self):
        buf = ctypes.create_string_buffer(256)
        check(lib.ocipGetDeviceName(buf, 256), "ocipGetDeviceName")
        return buf.value.decode()

    def close(self):
        if self.handle:
            check(lib.ocipUninitialize(self.handle), "ocipUninitialize")
            self.handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def simage_for(shape, dtype, step=None):
    h, w = shape[0], shape[1]
    c = 1 if len(shape) == 2 else shape[2]
    t = TYPE_OF_NP[np.dtype(dtype)]
    if step is None:
        step = w * c * np.dtype(dtype).itemsize
    return SImage(w, h, step, c, t)


class Image:
    """An ocipImage whose host buffer is `array` (kept alive here).

    array=None with shape/dtype gives a device-only image."""

    def __init__(self, array=None, shape=None, dtype=None, step=None):
        if array is not None:
            if not array.flags["C_CONTIGUOUS"] and step is None:
                array = np.ascontiguousarray(array)
            self.array = array
            desc = simage_for(array.shape, array.dtype,
                              step if step is not None else array.strides[0])
            data = array.ctypes.data_as(ctypes.c_void_p)
        else:
            self.array = None
            desc = simage_for(shape, dtype, step)
            data = None
        self.desc = desc
        self.handle = ctypes.c_void_p()
        check(lib.ocipCreateImage(ctypes.byref(self.handle), desc, data, CL_MEM_READ_WRITE),
              "ocipCreateImage")

    def send(self):
        check(lib.ocipSendImage(self.handle), "ocipSendImage")

    def read(self):
        check(lib.ocipReadImage(self.handle), "ocipReadImage")
        return self.array

    def device_ptr(self):
        p = ctypes.c_void_p()
        pitch = ctypes.c_size_t()
        check(lib.ocipGetImageDevicePtr(self.handle, ctypes.byref(p), ctypes.byref(pitch)),
              "ocipGetImageDevicePtr")
        return p.value, pitch.value

    def release(self):
        if self.handle:
            lib.ocipReleaseImage(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def _measure_fn(name):
    return getattr(lib, "ocip" + name)


def sqr_distance(S, T, D):
    return check(lib.ocipSqrDistance(S.handle, T.handle, D.handle), "ocipSqrDistance")


def sqr_distance_norm(S, T, D):
    return check(lib.ocipSqrDistance_Norm(S.handle, T.handle, D.handle), "ocipSqrDistance_Norm")


def abs_distance(S, T, D):
    return check(lib.ocipAbsDistance(S.handle, T.handle, D.handle), "ocipAbsDistance")


def cross_corr(S, T, D):
    return check(lib.ocipCrossCorr(S.handle, T.handle, D.handle), "ocipCrossCorr")


def cross_corr_norm(S, T, D):
    return check(lib.ocipCrossCorr_Norm(S.handle, T.handle, D.handle), "ocipCrossCorr_Norm")


def proximity(measure, S, T, D):
    """Calls ocip<measure>(S, T, D) and returns its error code (no raise)."""
    return _measure_fn(measure)(S.handle, T.handle, D.handle)


def match(measure, src, tmpl, out_dtype=None):
    """Convenience: one measure on host arrays, result as a numpy array.

    Uses the current context and its proximity path."""
    out_dtype = out_dtype or (np.float64 if src.dtype == np.float64 else np.float32)
    out = np.zeros(src.shape, dtype=out_dtype)
    S, T, D = Image(src), Image(tmpl), Image(out)
    try:
        check(proximity(measure, S, T, D), "ocip" + measure)
        D.read()
    finally:
        S.release(); T.release(); D.release()
    return out


class Program:
    def __init__(self, handle):
        self.handle = handle

    def release(self):
        if self.handle:
            lib.ocipReleaseProgram(self.handle)
            self.handle = ctypes.c_void_p()


MEASURE_INDEX = {"SqrDistance": 0, "SqrDistance_Norm": 1, "AbsDistance": 2, "CrossCorr": 3,
                 "CrossCorr_Norm": 4}


class Batch(Program):
    """A prepared batch (ocipPrepareProximityBatch): measure of every
    (image i, template j) pair into dests[i * len(templates) + j]."""

    def __init__(self, measure, images, templates, dests):
        n, m = len(images), len(templates)
        arr = lambda xs: (ctypes.c_void_p * len(xs))(*[x.handle for x in xs])
        self._keep = (arr(images), arr(templates), arr(dests))
        h = ctypes.c_void_p()
        code = measure if isinstance(measure, int) else MEASURE_INDEX[measure]
        rc = lib.ocipPrepareProximityBatch(ctypes.byref(h), code, self._keep[0], n,
                                           self._keep[1], m, self._keep[2])
        super().__init__(h)
        self.rc = rc

    def run(self):
        return lib.ocipRunProximityBatch(self.handle)

    def info(self, tw=0, th=0):
        """(work items, band height used for tw x th templates)."""
        n, bh = ctypes.c_int(), ctypes.c_int()
        check(lib.ocipGetProximityBatchInfo(self.handle, tw, th, ctypes.byref(n), ctypes.byref(bh)),
              "ocipGetProximityBatchInfo")
        return n.value, bh.value


def prepare_batch(measure, images, templates, dests):
    b = Batch(measure, images, templates, dests)
    check(b.rc, "ocipPrepareProximityBatch")
    return b


def proximity_backward(S, T, G1=None, G2=None, N2=None, dS=None, dT=None):
    """ocipProximityBackward on Image handles (None for absent ones); returns
    the error code."""
    h = lambda x: x.handle if x is not None else None
    return lib.ocipProximityBackward(h(S), h(T), h(G1), h(G2), h(N2), h(dS), h(dT))


INDEX_OPS = {"MinIndx": 0, "MaxIndx": 1, "MinAbsIndx": 2, "MaxAbsIndx": 3}


def proximity_index(measure, op, S, T, D=None):
    """ocipProximityIndx: (error code, value, x, y) of the index reduction `op`
    (MinIndx, MaxIndx, MinAbsIndx, MaxAbsIndx) of the measure's map; D, when
    given, receives the map."""
    v, x, y = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
    code = measure if isinstance(measure, int) else MEASURE_INDEX[measure]
    rc = lib.ocipProximityIndx(code, INDEX_OPS[op], S.handle, T.handle,
                               D.handle if D is not None else None, ctypes.byref(v),
                               ctypes.byref(x), ctypes.byref(y))
    return rc, v.value, x.value, y.value


def prepare_statistics(img=None):
    h = ctypes.c_void_p()
    check(lib.ocipPrepareStatistics(ctypes.byref(h), img.handle if img else None),
          "ocipPrepareStatistics")
    return Program(h)


def index_reduce(name, prog, img):
    """ocip<name>(prog, img) for name in MinIndx, MaxIndx, MinAbsIndx, MaxAbsIndx:
    (error code, value, x, y)."""
    v, x, y = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
    rc = getattr(lib, "ocip" + name)(prog.handle, img.handle, ctypes.byref(v), ctypes.byref(x),
                                     ctypes.byref(y))
    return rc, v.value, x.value, y.value


def prepare_integral(img=None):
    h = ctypes.c_void_p()
    check(lib.ocipPrepareIntegral(ctypes.byref(h), img.handle if img else None),
          "ocipPrepareIntegral")
    return Program(h)


def integral(prog, S, D, sqr=False):
    fn = lib.ocipSqrIntegral if sqr else lib.ocipIntegral
    return check(fn(prog.handle, S.handle, D.handle),
                 "ocipSqrIntegral" if sqr else "ocipIntegral")


def prepare_proximity_fft(S=None, T=None):
    h = ctypes.c_void_p()
    check(lib.ocipPrepareImageProximityFFT(ctypes.byref(h), S.handle if S else None,
                                           T.handle if T else None),
          "ocipPrepareImageProximityFFT")
    return Program(h)
