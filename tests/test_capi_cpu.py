"""The C-ABI boundary without a GPU: the library loads, exports exactly what
include/fasp_b200.h declares, and its defaults mirror SOLParams (src/Param.hxx:68-79)."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fasp_b200.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(fasp_gpu_[a-z0-9_]+)\s*\(",
                                 txt, re.M)))


def test_library_exports_every_declared_symbol():
    from faspxx_b200 import capi
    names = declared()
    assert len(names) >= 40
    for n in names:
        assert hasattr(capi.lib, n), n
    assert sorted(capi.SIGNATURES) == names


def test_exported_symbols_are_exactly_the_header():
    lib = os.path.join(ROOT, "faspxx_b200", "libfasp_b200.so")
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True).stdout
    exported = sorted({l.split()[-1] for l in out.splitlines() if " T fasp_gpu_" in l})
    assert exported == declared()


def test_defaults_mirror_solparams():
    from faspxx_b200 import capi
    cfg = capi.default_config(capi.CG)
    assert (cfg.prm.maxIter, cfg.prm.minIter, cfg.prm.savIter, cfg.prm.restart) == (1, 0, 100000, 30)
    assert (cfg.prm.relTol, cfg.prm.absTol) == (1e-6, 1e-8)
    assert cfg.useGraph == 1 and cfg.precision == capi.FP64


def test_struct_layouts_match_header():
    """Compile a C probe against the header and compare sizeof/offsetof with ctypes."""
    from faspxx_b200 import capi
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "fasp_b200.h"
int main(void){printf("%zu %zu %zu %zu %zu\n", sizeof(fasp_gpu_config), sizeof(fasp_gpu_info),
 offsetof(fasp_gpu_config, useGraph), offsetof(fasp_gpu_info, launches), sizeof(fasp_gpu_params));return 0;}
'''
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "p.c"), "w") as f:
            f.write(src)
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), os.path.join(d, "p.c"), "-o",
                        os.path.join(d, "p")], check=True)
        got = list(map(int, subprocess.run([os.path.join(d, "p")], capture_output=True,
                                           text=True).stdout.split()))
    assert got == [C.sizeof(capi.Config), C.sizeof(capi.Info), capi.Config.useGraph.offset,
                   capi.Info.launches.offset, C.sizeof(capi.Params)]


def test_no_device_is_reported_not_faked():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from faspxx_b200 import capi
    assert capi.lib.fasp_gpu_init(0) == capi.ERROR_NO_DEVICE
    with pytest.raises(capi.FaspError):
        from faspxx_b200 import sol
        sol.DVec(4)


def test_strerror_covers_retcodes():
    from faspxx_b200 import capi
    for code in (0, -12, -15, -17, -18, -20, -30, -32, -33, -34, -39, -101, -102):
        assert capi.lib.fasp_gpu_strerror(code).decode() != "Unknown error"
