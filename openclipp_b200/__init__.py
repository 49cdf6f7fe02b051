"""OpenCLIPP template matching on NVIDIA B200 (sm_100a).

The product is the C shared library libopenclipp_b200.so (C ABI declared in
include/OpenCLIPP.h and include/OpenCLIPP_B200.h). This package locates it
and offers a thin ctypes mirror of that interface (openclipp_b200.ocip) for
Python callers, the tests and the benchmark.
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(HERE, "libopenclipp_b200.so")
INCLUDE_DIR = os.path.join(os.path.dirname(HERE), "include")

__all__ = ["LIBRARY_PATH", "INCLUDE_DIR"]
