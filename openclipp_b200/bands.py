"""One image split across GPUs in row bands (one process and one context per GPU).

A template-matching map is local: destination row y reads only source rows
y - th/2 .. y - th/2 + th - 1. So an image splits into bands of destination
rows, and each GPU receives only its band's source rows plus a halo of
th - 1 rows (ocipGetProximityBand gives both ranges). The GPUs exchange
nothing while they compute; the only collective is the optional gather of the
bands into one map (NCCL over NVLink for CUDA tensors, gloo for host
tensors). The reference has no counterpart: its contexts never share an
image (OpenCLIPP/OpenCLIPP.cpp:73-75, include/OpenCLIPP.h:107-112).
"""
import ctypes

import numpy as np

from . import ocip


def band(height, tmpl_height, part, parts):
    """(y0, y1, s0, s1): part `part` of `parts` owns destination rows y0..y1
    (exclusive) and needs source rows s0..s1 (ocipGetProximityBand)."""
    rows = (ctypes.c_uint * 4)()
    ocip.check(ocip.lib.ocipGetProximityBand(height, tmpl_height, part, parts, rows),
               "ocipGetProximityBand")
    return tuple(int(r) for r in rows)


def bands(height, tmpl_height, parts):
    """Every part's band, in part order."""
    return [band(height, tmpl_height, p, parts) for p in range(parts)]


class BandMatch:
    """One part's share of a measure over a whole image, on the current context.

    `src` is the whole host image (only rows s0..s1 are sent to the GPU: a
    numpy row slice, no host copy); the map of the source band stays on the
    device. `owned()` returns the part's destination rows, `device_view()`
    the same rows as a CUDA array (pitch-strided, no copy) for a collective.
    The destination has a host buffer of the band's size for owned().
    """

    def __init__(self, src, tmpl, part, parts, out_dtype=None):
        self.y0, self.y1, self.s0, self.s1 = band(src.shape[0], tmpl.shape[0], part, parts)
        self.out_dtype = np.dtype(out_dtype or (np.float64 if src.dtype == np.float64
                                                else np.float32))
        self.width = src.shape[1]
        self.nch = 1 if src.ndim == 2 else src.shape[2]
        self.src = self.tmpl = self.dst = None
        if self.y1 == self.y0:
            return
        shape = (self.s1 - self.s0,) + src.shape[1:]
        self.src = ocip.Image(src[self.s0:self.s1])
        self.tmpl = ocip.Image(tmpl)
        self.dst = ocip.Image(np.zeros(shape, self.out_dtype))

    def run(self, measure):
        """Queues ocip<measure> on the band (asynchronous, like the measure call)."""
        if self.dst is not None:
            ocip.check(ocip.proximity(measure, self.src, self.tmpl, self.dst), "ocip" + measure)

    def owned(self):
        """The owned destination rows as a host array (a blocking read of the
        band map, as ocipReadImage is)."""
        if self.dst is None:
            shape = (0, self.width) + ((self.nch,) if self.nch > 1 else ())
            return np.zeros(shape, self.out_dtype)
        full = self.dst.read()
        return full[self.y0 - self.s0:self.y1 - self.s0].copy()

    def device_view(self):
        """The owned rows of the band map as an object with
        __cuda_array_interface__ (torch.as_tensor(view, device="cuda") wraps it
        without a copy), or None for a part that owns no rows. The map is
        written on the context's stream (ocip_stream()): order reads after it."""
        if self.dst is None:
            return None
        ptr, pitch = self.dst.device_ptr()
        return _CudaRows(ptr + (self.y0 - self.s0) * pitch, self.y1 - self.y0,
                         self.width * self.nch, pitch, self.out_dtype.itemsize,
                         self.out_dtype.str)

    def release(self):
        for im in (self.src, self.tmpl, self.dst):
            if im is not None:
                im.release()
        self.src = self.tmpl = self.dst = None


class _CudaRows:
    def __init__(self, ptr, rows, cols, pitch, item, typestr):
        self.__cuda_array_interface__ = {
            "shape": (rows, cols), "typestr": typestr, "data": (ptr, False),
            "strides": (pitch, item), "version": 2}


def ocip_stream():
    """The current context's CUDA stream handle."""
    s = ctypes.c_void_p()
    ocip.check(ocip.lib.ocipGetStream(ctypes.byref(s)), "ocipGetStream")
    return s.value or 0


def gather_rows(owned, height, tmpl_height, rank, world, dst=0):
    """Gathers every part's owned rows into the whole map on rank `dst`.

    `owned` is this rank's rows (a torch tensor of shape (rows, cols): CUDA
    under NCCL, host under gloo). The bands are padded to the largest one so
    that one all-gather moves them; rank `dst` returns the (height, cols) map,
    the other ranks None. Every rank must call it (a collective)."""
    import torch
    import torch.distributed as dist
    parts = bands(height, tmpl_height, world)
    most = max(y1 - y0 for y0, y1, _, _ in parts)
    cols = owned.shape[1]
    y0, y1 = parts[rank][0], parts[rank][1]
    if owned.shape[0] != y1 - y0:
        raise ValueError(f"rank {rank} owns {y1 - y0} rows, got {owned.shape[0]}")
    padded = torch.zeros((most, cols), dtype=owned.dtype, device=owned.device)
    padded[:y1 - y0] = owned
    out = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(out, padded)
    if rank != dst:
        return None
    full = torch.empty((height, cols), dtype=owned.dtype, device=owned.device)
    for (a, b, _, _), t in zip(parts, out):
        full[a:b] = t[:b - a]
    return full
