"""The CarpetLib side of the drop-in, built against CarpetLib's own headers
(the reference sources, with the oracle's stand-ins for the Cactus flesh):

* carpet_b200/carpet/data_cgx.cc -- data<CCTK_REAL8>::transfer_from_innerloop
  through cgx_transfer -- compiles, with the compile-time checks that
  CarpetLib's operator_type and centering values are the C-ABI's;
* tests/carpet_shim_check.cc runs the marshalling (carpet_b200/carpet/
  cgx_carpet.hh) on CarpetLib's bbox / vect / islab with a stand-in for
  cgx_transfer that records its arguments: boxes arrive as the memory layout
  of bbox<int,3> (what data.cc:212-214 hands the Fortran operators), the
  slab offset as islab::offset, arrays as (storage, padded shape, extent).

Needs the reference sources (CGX_REFERENCE, else the default location) and
the reference build's objects (make -C oracle ref); skipped without them.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("CGX_REFERENCE", "/root/reference")
SRC = os.path.join(REF, "CarpetLib", "src")
OBJ = os.path.join(ROOT, "oracle", "_ref", "nofma")


def _flags():
    return ["-std=c++17", "-w", "-fopenmp", "-I" + os.path.join(ROOT, "oracle", "shim"), "-I" + SRC,
            "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(ROOT, "carpet_b200", "carpet")]


@pytest.fixture(scope="module")
def tmp(tmp_path_factory):
    if not os.path.isdir(SRC):
        pytest.skip("reference sources not present")
    return tmp_path_factory.mktemp("shim")


def test_transfer_from_innerloop_compiles_against_carpetlib(tmp):
    out = tmp / "data_cgx.o"
    r = subprocess.run(["g++", *_flags(), "-c", os.path.join(ROOT, "carpet_b200", "carpet", "data_cgx.cc"),
                        "-o", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    nm = subprocess.run(["nm", "-C", str(out)], capture_output=True, text=True).stdout
    assert "data<double>::transfer_from_innerloop" in nm
    assert " U cgx_transfer" in nm


def test_marshalling_matches_what_carpetlib_hands_its_operators(tmp):
    objs = [os.path.join(OBJ, f) for f in ("bbox.o", "vect.o", "shim_support.o")]
    if not all(os.path.exists(o) for o in objs):
        pytest.skip("reference build objects missing (make -C oracle ref)")
    exe = tmp / "check"
    r = subprocess.run(["g++", *_flags(), os.path.join(ROOT, "tests", "carpet_shim_check.cc"), *objs,
                        "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "marshalling ok" in r.stdout
