"""The C ABI surface and the host-side logic, without a GPU.

Checks that the shared library loads and exports every function that
include/imageproc_b200.h declares, and that the argument checks (which run on
the host before any device work) reproduce the reference's panics and their
messages (src/template_matching.rs:395-402, :433-437, :483-486) in the
reference's order.
"""

import re

import numpy as np
import pytest

from conftest import ROOT
from imageproc_b200 import _lib
from imageproc_b200 import template_matching as tm

HEADER = ROOT / "include" / "imageproc_b200.h"
EXTREMES_SUFFIXES = ["u8", "u16", "u32", "u64", "i8", "i16", "i32", "i64", "f32", "f64"]
SUPPRESS_SUFFIXES = ["u8", "u16", "u32", "u64", "i8", "i16", "i32", "i64", "f32"]


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"#define.*?(?<!\\)\n", "", text, flags=re.S)
    names = set(re.findall(r"\b(ipb_[a-z0-9_]+)\s*\(", text))
    # the find_extremes family is declared through a macro
    for s in EXTREMES_SUFFIXES:
        names.add(f"ipb_find_extremes_{s}")
        names.add(f"ipb_find_extremes_{s}_device")
    # and so is suppress_non_maximum's
    for s in SUPPRESS_SUFFIXES:
        names.add(f"ipb_suppress_non_maximum_{s}")
        names.add(f"ipb_suppress_non_maximum_{s}_device")
    names = {n for n in names if not n.startswith("ipb_extremes_")}
    return sorted(names)


def test_library_exports_every_declared_function():
    L = _lib.lib()
    names = declared_functions()
    assert "ipb_match_template" in names and "ipb_match_template_device" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_string():
    assert b"sm_100a" in _lib.lib().ipb_version()


def img(w, h, v=0):
    return np.full((h, w), v, np.uint8)


@pytest.mark.parametrize("fn", [tm.match_template, tm.match_template_parallel])
def test_template_wider_than_image_panics_with_reference_message(fn):
    with pytest.raises(tm.Panic, match="^image width must be greater than or equal to template width$"):
        fn(img(5, 5), img(6, 5), tm.MatchTemplateMethod.SumOfSquaredErrors)


@pytest.mark.parametrize("fn", [tm.match_template, tm.match_template_parallel])
def test_template_taller_than_image_panics_with_reference_message(fn):
    with pytest.raises(tm.Panic, match="^image height must be greater than or equal to template height$"):
        fn(img(5, 5), img(5, 6), tm.MatchTemplateMethod.SumOfSquaredErrors)


@pytest.mark.parametrize("fn", [tm.match_template_with_mask, tm.match_template_with_mask_parallel])
def test_mask_size_is_checked_first(fn):
    # the template is also too wide: the reference asserts the mask first
    with pytest.raises(tm.Panic, match="^the template and mask must be the same size$"):
        fn(img(5, 5), img(6, 5), tm.MatchTemplateMethod.CrossCorrelation, img(5, 5))
    with pytest.raises(tm.Panic, match="^image width must be greater than or equal to template width$"):
        fn(img(5, 5), img(6, 5), tm.MatchTemplateMethod.CrossCorrelation, img(6, 5))


def test_find_extremes_of_empty_image_panics():
    for dtype in (np.uint8, np.float32, np.int64):
        with pytest.raises(tm.Panic, match="^image must be non-empty$"):
            tm.find_extremes(np.zeros((0, 3), dtype))
        with pytest.raises(tm.Panic, match="^image must be non-empty$"):
            tm.find_extremes(np.zeros((3, 0), dtype))


def test_bad_method_and_precision_are_rejected():
    with pytest.raises(ValueError):
        tm.match_template(img(5, 5), img(2, 2), 7)
    with pytest.raises(ValueError):
        tm.set_precision(9)


def test_precision_round_trip():
    old = tm.get_precision()
    try:
        for p in tm.Precision:
            tm.set_precision(p)
            assert tm.get_precision() == p
    finally:
        tm.set_precision(old)


def test_non_gray_inputs_are_type_errors():
    with pytest.raises(TypeError):
        tm.match_template(np.zeros((4, 4), np.float32), img(2, 2), 0)
    with pytest.raises(TypeError):
        tm.match_template(np.zeros((4, 4, 3), np.uint8), img(2, 2), 0)


def test_method_enum_matches_reference_order():
    assert [m.name for m in tm.MatchTemplateMethod] == [
        "SumOfSquaredErrors", "SumOfSquaredErrorsNormalized", "CrossCorrelation",
        "CrossCorrelationNormalized"]


def test_cpp_mirror_raises_reference_panics(tmp_path):
    import shutil
    import subprocess
    if not shutil.which("g++"):
        pytest.skip("no C++ compiler")
    exe = tmp_path / "hpp_panics"
    lib_dir = _lib.LIB_PATH.parent
    subprocess.run(["g++", "-std=c++17", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "hpp_panics.cpp"), "-L", str(lib_dir),
                    "-limageproc_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"


def test_kernel_path_round_trip():
    # host-side switch only: no kernel runs
    old = tm.get_path()
    try:
        for p in tm.Path:
            tm.set_path(p)
            assert tm.get_path() == p
        assert int(tm.Path.RowOperand) == 3
        with pytest.raises(ValueError):
            tm.set_path(4)
    finally:
        tm.set_path(old)
