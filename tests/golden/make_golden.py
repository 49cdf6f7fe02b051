"""Generates the golden fixtures in this directory from the reference itself.

The reference ships no golden vectors or known-answer tests for this path
(its only checks compare against Intel IPP, Bench/src/benchImageProximity.hpp
:57-58). These fixtures are outputs of the reference's own kernel sources,
cl-files/ImageProximity.cl and cl-files/Integral.cl, compiled unmodified for
the host through oracle/ref_shim.h (oracle/Makefile, `make -C oracle ref`),
on small seeded inputs:

  proximity.npz  every pixel type x {1, 2, 4} channels x 5 measures, with the
                 reference's own dispatch (_Cached kernel for templates up to
                 16x16, the plain kernel otherwise), in both arithmetic forms
                 (each operation rounded; every acc += a*b contracted to fma);
  integral.npz   Integral and SqrIntegral into F32 and F64 destinations.

Run from the repository root: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# (image W, H, template tw, th): odd and even template sides, a 1x1 template,
# a template as large as the image, one over 16 wide (plain kernel).
SHAPES = [(19, 13, 4, 3), (23, 17, 16, 16), (21, 9, 17, 5), (7, 5, 7, 5), (11, 10, 1, 1)]


def make_inputs(rng, dtype, shape_img, shape_t):
    if np.dtype(dtype).kind == "f":
        S = rng.standard_normal(shape_img).astype(dtype)
        T = rng.standard_normal(shape_t).astype(dtype)
    else:
        info = np.iinfo(dtype)
        lo, hi = max(int(info.min), -40000), min(int(info.max), 40000)
        S = rng.integers(lo, hi + 1, shape_img).astype(dtype)
        T = rng.integers(lo, hi + 1, shape_t).astype(dtype)
    return S, T


def main():
    rng = np.random.default_rng(20140301)
    prox = {}
    case = 0
    for ti, dt in enumerate(O.NP_TYPES):
        for c in (1, 2, 4):
            for (W, H, tw, th) in SHAPES:
                if c == 4 and (W, H) != (19, 13):
                    continue
                si = (H, W) if c == 1 else (H, W, c)
                st = (th, tw) if c == 1 else (th, tw, c)
                S, T = make_inputs(rng, dt, si, st)
                key = f"c{case:03d}"
                prox[key + "_S"] = S
                prox[key + "_T"] = T
                for m in range(5):
                    prox[f"{key}_m{m}"] = O.proximity_reference(m, S, T, mode=0)
                    prox[f"{key}_m{m}_fma"] = O.proximity_reference(m, S, T, mode=0, fused=True)
                case += 1
    np.savez_compressed(os.path.join(HERE, "proximity.npz"), **prox)

    integ = {}
    for i, (dt, W, H) in enumerate([(np.uint8, 70, 11), (np.uint8, 64, 8), (np.float32, 130, 17),
                                    (np.uint16, 5, 3), (np.int16, 65, 9), (np.float64, 66, 10)]):
        if np.dtype(dt).kind == "f":
            S = rng.standard_normal((H, W)).astype(dt)
        else:
            info = np.iinfo(dt)
            S = rng.integers(max(int(info.min), -3000), min(int(info.max), 3000) + 1, (H, W)).astype(dt)
        integ[f"i{i}_S"] = S
        for sqr in (0, 1):
            for f64 in (0, 1):
                if dt == np.float64 and not f64:
                    continue  # the reference's F64-source, F32-dest case is not reproduced
                integ[f"i{i}_sqr{sqr}_f64{f64}"] = O.integral_reference(S, sqr, f64)
    np.savez_compressed(os.path.join(HERE, "integral.npz"), **integ)
    print("proximity cases:", case, "integral cases:", len(integ))


if __name__ == "__main__":
    main()
