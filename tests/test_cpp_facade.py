"""The C++ façade (include/faspxx_b200.hxx): a driver in the shape of the reference's
example/TestPCG.cxx compiles against it, links to libfasp_b200.so and solves on the GPU."""
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "faspxx_b200", "examples", "test_pcg.cxx")
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "faspxx_b200")


def _compile(out):
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{INC}", SRC, "-o", out, f"-L{LIBDIR}",
                    "-l:libfasp_b200.so", f"-Wl,-rpath,{LIBDIR}"], check=True)


def test_driver_compiles_and_links():
    with tempfile.TemporaryDirectory() as d:
        _compile(os.path.join(d, "t"))


def test_header_is_plain_c():
    """fasp_b200.h is usable from C (the binding other languages' FFIs read)."""
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "c.c")
        with open(p, "w") as f:
            f.write('#include "fasp_b200.h"\nint main(void){fasp_gpu_config c;'
                    'fasp_gpu_default_config(&c, FASP_GPU_CG);return c.alg == 1 ? 0 : 1;}\n')
        subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", f"-I{INC}", p, "-o",
                        os.path.join(d, "c"), f"-L{LIBDIR}", "-l:libfasp_b200.so",
                        f"-Wl,-rpath,{LIBDIR}"], check=True)


@pytest.mark.gpu
def test_driver_runs_on_gpu():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "t")
        _compile(exe)
        out = subprocess.run([exe, "48", "2000"], capture_output=True, text=True, check=True).stdout
    rows = [l.split() for l in out.strip().splitlines()]
    assert rows[0][0] == "pcg" and rows[0][1] == "0" and int(rows[0][2]) > 10
    for name, code, err in rows[1:]:
        assert code == "0", name
        assert float(err) < 1e-5, (name, err)


FEATURES = os.path.join(ROOT, "faspxx_b200", "examples", "test_features.cxx")


def _compile_features(out):
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", f"-I{INC}", FEATURES, "-o", out,
                    f"-L{LIBDIR}", "-l:libfasp_b200.so", f"-Wl,-rpath,{LIBDIR}"], check=True)


def test_feature_driver_compiles():
    with tempfile.TemporaryDirectory() as d:
        _compile_features(os.path.join(d, "f"))


@pytest.mark.gpu
def test_feature_driver_runs_on_gpu():
    """StencilLOP (the matrix-free example at dim 64: 121 CG iterations and the L2 error the
    reference prints, 1.0041e-04), MAT::Mult/Add/MultTransposeAdd, ReadMat of a MatrixMarket
    file, and
    MG-preconditioned CG through the façade."""
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "f")
        _compile_features(exe)
        out = subprocess.run([exe], capture_output=True, text=True, check=True, cwd=d).stdout
    r = {l.split()[0]: l.split()[1:] for l in out.strip().splitlines()}
    assert r["matfree_cg"][0] == "0" and abs(int(r["matfree_cg"][1]) - 121) <= 1
    assert abs(float(r["matfree_cg"][2]) - 1.0041e-04) <= 2e-8
    assert r["mult"] == ["0", "352", "36"]  # the 13-point square of the 5-point stencil
    assert r["add"] == ["0", "156", "36"]   # 2A - A keeps A's pattern
    # MultTransposeAdd on a symmetric matrix equals Apply + v2 (within rounding)
    assert float(r["mta"][0]) > 0 and float(r["mta"][1]) <= 1e-13
    assert r["readmat"] == ["0", "3", "5"]  # every row has its diagonal: nothing inserted
    assert r["mg_pcg"][0] == "0" and int(r["mg_pcg"][1]) <= 12
