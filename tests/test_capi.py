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
