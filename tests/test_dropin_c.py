"""The drop-in C API as a C program sees it: programs compiled against
include/parasail.h and include/parasail/matrices/*.h and linked with
libparasail_b200.so.

- tests/c/dropin_kat.c: this project's own C check of the API (static
  matrix objects, direct/profile/serial forms, statistics accessors, _sat
  chains, name lookups, parasail_nw_banded).
- oracle/_ref/test_basic.o: the reference's own known-answer program
  (tests/test_basic.c:22-80, scores 20, 27, 4, 20), compiled unchanged
  against these headers by oracle/Makefile where the reference sources are
  present; the object travels with the repository.

On CPU both are linked (the headers and the library's exported symbols
agree); on a GPU both are run and must exit 0.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "parasail_b200")
KAT_SRC = os.path.join(ROOT, "tests", "c", "dropin_kat.c")
REF_OBJ = os.path.join(ROOT, "oracle", "_ref", "test_basic.o")


def _link(tmp_path, name, inputs):
    exe = str(tmp_path / name)
    cmd = ["gcc", "-O1", "-std=gnu99", "-I" + INC, "-o", exe] + inputs + \
          ["-L" + LIBDIR, "-lparasail_b200", "-Wl,-rpath," + LIBDIR]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def _run(exe):
    p = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    return p.returncode, p.stdout + p.stderr


def test_dropin_programs_link(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libparasail_b200.so")):
        pytest.skip("libparasail_b200.so not built")
    _link(tmp_path, "kat", [KAT_SRC])
    if os.path.exists(REF_OBJ):
        _link(tmp_path, "test_basic", [REF_OBJ])


@pytest.mark.gpu
def test_own_c_program_runs(tmp_path):
    rc, out = _run(_link(tmp_path, "kat", [KAT_SRC]))
    assert rc == 0, out
    assert "pass (0 failures)" in out


@pytest.mark.gpu
def test_reference_test_basic_unchanged_runs(tmp_path):
    if not os.path.exists(REF_OBJ):
        pytest.skip("oracle/_ref/test_basic.o not built (reference sources absent at build time)")
    rc, out = _run(_link(tmp_path, "test_basic", [REF_OBJ]))
    assert rc == 0, out
    assert out.count("pass") == 4, out
