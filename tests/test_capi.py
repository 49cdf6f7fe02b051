"""The C-ABI library: loads, exports every declared entry point, and behaves
on hosts without a GPU (no compute is attempted here)."""
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "openclipp_b200")


def declared_symbols():
    names = set()
    for f in os.listdir(INCLUDE):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, f)).read()
        for stmt in text.split(";"):
            if "ocip_API" not in stmt or "#define" in stmt:
                continue
            m = re.search(r"\b(ocip[A-Z]\w*)\s*\(", stmt)
            if m:
                names.add(m.group(1))
    return names


def exported_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(LIBDIR, "libopenclipp_b200.so")],
                         capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


def test_every_declared_symbol_is_exported():
    decl = declared_symbols()
    assert len(decl) >= 30
    missing = decl - exported_symbols()
    assert not missing, missing


def test_only_ocip_symbols_are_exported():
    extra = {s for s in exported_symbols() if not s.startswith("ocip")}
    assert not extra, extra


def test_error_names(ocip):
    assert ocip.error_name(0) == "SUCCESS"
    assert ocip.error_name(-30) == "CL_INVALID_VALUE"
    assert ocip.error_name(-40) == "CL_INVALID_IMAGE_SIZE"
    assert ocip.error_name(-34) == "CL_INVALID_CONTEXT"
    assert ocip.error_name(12345) == "Unknown CL error"


def test_calls_without_context(ocip):
    """Before any context exists every call reports CL_INVALID_CONTEXT, as the
    reference's GetList() (OpenCLIPP/OpenCLIPP.cpp:717-728)."""
    import ctypes
    h = ctypes.c_void_p()
    assert ocip.lib.ocipFinish() == ocip.CL_INVALID_CONTEXT
    desc = ocip.SImage(4, 4, 4, 1, ocip.U8)
    assert ocip.lib.ocipCreateImage(ctypes.byref(h), desc, None, 1) == ocip.CL_INVALID_CONTEXT
    assert ocip.lib.ocipCrossCorr(None, None, None) == ocip.CL_INVALID_CONTEXT
    assert ocip.lib.ocipUninitialize(None) == ocip.CL_INVALID_CONTEXT
    assert ocip.lib.ocipChangeContext(None) == ocip.CL_INVALID_CONTEXT
    assert ocip.lib.ocipSetProximityPath(1) == ocip.CL_INVALID_CONTEXT


def test_cpu_device_type_is_not_found(ocip):
    import ctypes
    h = ctypes.c_void_p()
    CL_DEVICE_TYPE_CPU = 1 << 1
    assert ocip.lib.ocipInitialize(ctypes.byref(h), None, CL_DEVICE_TYPE_CPU) == ocip.CL_DEVICE_NOT_FOUND


def test_c_program_compiles_and_links_against_the_header():
    """A C caller written against include/OpenCLIPP.h builds and links with
    -lopenclipp_b200, as a reference user's program would."""
    src = r'''
#include <stdio.h>
#include "OpenCLIPP.h"
#include "OpenCLIPP_B200.h"
int main(void) {
  ocipContext ctx = 0;
  ocipError e = ocipInitialize(&ctx, NULL, CL_DEVICE_TYPE_ALL);
  printf("%s\n", ocipGetErrorName(e));
  if (e == CL_SUCCESS) {
    unsigned char img[64] = {0}, tpl[4] = {1, 2, 3, 4};
    float out[64];
    SImage si = {8, 8, 8, 1, U8}, st = {2, 2, 2, 1, U8}, so = {8, 8, 32, 1, F32};
    ocipImage S, T, D;
    ocipCreateImage(&S, si, img, CL_MEM_READ_WRITE);
    ocipCreateImage(&T, st, tpl, CL_MEM_READ_WRITE);
    ocipCreateImage(&D, so, out, CL_MEM_READ_WRITE);
    e = ocipCrossCorr(S, T, D);
    if (e == CL_SUCCESS) e = ocipReadImage(D);
    printf("%s %g\n", ocipGetErrorName(e), out[0]);
    ocipReleaseImage(S); ocipReleaseImage(T); ocipReleaseImage(D);
    ocipUninitialize(ctx);
  }
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "caller.c")
        exe = os.path.join(d, "caller")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", INCLUDE, c, "-o", exe,
                        "-L", LIBDIR, "-lopenclipp_b200", f"-Wl,-rpath,{LIBDIR}"],
                       check=True, capture_output=True)
        r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        first = r.stdout.split()[0]
        assert first in ("SUCCESS", "CL_DEVICE_NOT_FOUND")
        if first == "SUCCESS":
            assert r.stdout.split()[1] == "SUCCESS"


def test_no_alloc_scratch_limit_is_checked_on_the_host(ocip):
    """ocipIntegralNoAlloc refuses an image whose scan scratch exceeds its fixed
    16 MiB array before any device work: one channel fits up to 7307 x 7307
    (8 bytes per 128-pixel row segment and per column of each 32-row band),
    7308 x 7308 does not. Only refused sizes are passed here, so the dummy
    pointers are never used."""
    import ctypes
    for w, h in ((7308, 7308), (100000, 1000), (1000, 100000)):
        src = ocip.SImage(w, h, w, 1, ocip.U8)
        dst = ocip.SImage(w, h, w * 8, 1, ocip.F64)
        rc = ocip.lib.ocipIntegralNoAlloc(1, src, ctypes.c_void_p(16), w, dst,
                                          ctypes.c_void_p(16), w * 8, None)
        assert rc == ocip.CL_INVALID_IMAGE_SIZE, (w, h, rc)
        assert b"fixed limit" in ocip.lib.ocipGetLastErrorMessage()


C_MATCHER = r'''
/* A reference user's program: reads a U8 image and template from files,
 * computes CrossCorr and SqrDistance_Norm through the drop-in header, and
 * writes the score maps. */
#include <stdio.h>
#include <stdlib.h>
#include "OpenCLIPP.h"
#include "OpenCLIPP_B200.h"
static int load(const char* path, void* buf, size_t n) {
  FILE* f = fopen(path, "rb");
  if (!f) return 1;
  size_t got = fread(buf, 1, n, f);
  fclose(f);
  return got != n;
}
int main(int argc, char** argv) {
  const int W = 300, H = 200, TW = 21, TH = 17;
  unsigned char* img = malloc(W * H);
  unsigned char* tpl = malloc(TW * TH);
  float* cc = malloc(sizeof(float) * W * H);
  float* sqn = malloc(sizeof(float) * W * H);
  if (argc < 5 || load(argv[1], img, W * H) || load(argv[2], tpl, TW * TH)) return 2;
  ocipContext ctx = 0;
  ocipError e = ocipInitialize(&ctx, NULL, CL_DEVICE_TYPE_GPU);
  if (e != CL_SUCCESS) { printf("%s\n", ocipGetErrorName(e)); return 3; }
  SImage si = {W, H, W, 1, U8}, st = {TW, TH, TW, 1, U8}, so = {W, H, W * 4, 1, F32};
  ocipImage S, T, D1, D2;
  ocipCreateImage(&S, si, img, CL_MEM_READ_WRITE);
  ocipCreateImage(&T, st, tpl, CL_MEM_READ_WRITE);
  ocipCreateImage(&D1, so, cc, CL_MEM_READ_WRITE);
  ocipCreateImage(&D2, so, sqn, CL_MEM_READ_WRITE);
  e = ocipCrossCorr(S, T, D1);
  if (e == CL_SUCCESS) e = ocipSetProximityPath(OCIP_PATH_TENSOR);
  if (e == CL_SUCCESS) e = ocipSqrDistance_Norm(S, T, D2);
  if (e == CL_SUCCESS) e = ocipReadImage(D1);
  if (e == CL_SUCCESS) e = ocipReadImage(D2);
  printf("%s\n", ocipGetErrorName(e));
  FILE* f = fopen(argv[3], "wb");
  fwrite(cc, sizeof(float), W * H, f);
  fclose(f);
  f = fopen(argv[4], "wb");
  fwrite(sqn, sizeof(float), W * H, f);
  fclose(f);
  ocipReleaseImage(S); ocipReleaseImage(T); ocipReleaseImage(D1); ocipReleaseImage(D2);
  ocipUninitialize(ctx);
  return e == CL_SUCCESS ? 0 : 1;
}
'''


@pytest.mark.gpu
def test_c_program_computes_maps_on_the_gpu():
    """The C caller above, built against the headers and linked with
    -lopenclipp_b200, computes a CrossCorr map (plain path) and a
    SqrDistance_Norm map (tensor path) of a U8 image; both equal the exact
    integer oracle rounded once (the sums stay below 2^24)."""
    import numpy as np

    from oracle import oracle as O
    rng = np.random.default_rng(12)
    S = rng.integers(0, 256, (200, 300), dtype=np.uint8)
    T = S[50:67, 100:121].copy()
    with tempfile.TemporaryDirectory() as d:
        c, exe = os.path.join(d, "matcher.c"), os.path.join(d, "matcher")
        open(c, "w").write(C_MATCHER)
        subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", INCLUDE, c, "-o", exe,
                        "-L", LIBDIR, "-lopenclipp_b200", f"-Wl,-rpath,{LIBDIR}"],
                       check=True, capture_output=True)
        paths = [os.path.join(d, n) for n in ("S.bin", "T.bin", "cc.bin", "sqn.bin")]
        S.tofile(paths[0])
        T.tofile(paths[1])
        r = subprocess.run([exe] + paths, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (r.stdout, r.stderr)
        cc = np.fromfile(paths[2], np.float32).reshape(S.shape)
        sqn = np.fromfile(paths[3], np.float32).reshape(S.shape)
    assert np.array_equal(cc, O.proximity_exact(3, S, T).astype(np.float32))
    ex = O.proximity_exact(1, S, T)
    assert np.abs(sqn - ex).max() <= 1e-6 * np.abs(ex).max()
    assert np.unravel_index(np.argmin(sqn), sqn.shape) == (50 + 8, 100 + 10)
