"""CPU checks of the C-ABI library: it loads without a GPU, exports every
entry point include/galaxy_gpu.h declares, and the ctypes structs match the
C layouts (sizes and field offsets measured by compiling the header)."""
import os
import re
import subprocess
import tempfile

import ctypes as C
import pytest

from galaxy_b200 import LIB_PATH, lib
from galaxy_b200._abi import GxConfig, GxDiag, GxGeometry

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "galaxy_gpu.h")


def declared():
    txt = open(HDR).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(gx_\w+)\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB_PATH)
    names = declared()
    assert len(names) >= 15
    L = lib()
    for n in names:
        assert hasattr(L, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True,
                         text=True).stdout
    for n in names:
        assert re.search(r"\bT " + n + r"\b", out), n


def test_struct_layouts_match_header():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "galaxy_gpu.h"
int main(void){
 printf("%zu %zu %zu\n", sizeof(GxConfig), sizeof(GxGeometry), sizeof(GxDiag));
 printf("%zu %zu %zu %zu\n", offsetof(GxConfig, rmap), offsetof(GxConfig, pmass),
        offsetof(GxConfig, device), offsetof(GxGeometry, lg));
 return 0;}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        lines = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    s = [int(v) for v in lines[0].split()]
    o = [int(v) for v in lines[1].split()]
    assert s == [C.sizeof(GxConfig), C.sizeof(GxGeometry), C.sizeof(GxDiag)]
    assert o == [GxConfig.rmap.offset, GxConfig.pmass.offset, GxConfig.device.offset,
                 GxGeometry.lg.offset]


def test_grdset_rejects_bad_cards_without_gpu():
    """setgrd's checks run before any CUDA call (setgrd.f:57-76, p3dset.f:99-100)."""
    from galaxy_b200 import Galaxy, GxError, make_config
    with pytest.raises(GxError, match="ngz must be a multiple of 3 & 5"):
        Galaxy(make_config(3, 16, 32, ngz=14, dzg=0.1, ng=4, softl=0.5))
    with pytest.raises(GxError, match="Softening length cannot be less"):
        Galaxy(make_config(3, 16, 128, ngz=15, dzg=0.5, ng=4, softl=0.4))
    with pytest.raises(GxError, match="Unrecognized softening rule"):
        Galaxy(make_config(2, 16, 32, ng=4, softl=0.5, tsoft=3))


def test_python_constants_match_the_header():
    """every GX_* integer constant the Python side defines has the header's value"""
    from galaxy_b200 import _abi
    hdr = dict(re.findall(r"^#define\s+(GX_\w+)\s+(-?\d+)\b", open(HDR).read(), re.M))
    py = {k: v for k, v in vars(_abi).items() if k.startswith("GX_") and isinstance(v, int)}
    assert len(py) >= 20
    for k, v in py.items():
        assert k in hdr and int(hdr[k]) == v, k
