"""Extract the reference's known-answer tests for integral images and
non-maximum suppression as fixtures.

Reads imageproc's ``src/integral_image.rs`` (tests :471-567),
``src/suppress.rs`` (tests :209-270) and ``src/filter/mod.rs`` (tests
:479-513, :615-693) as TEXT and writes
``reference_next_tests.json`` beside this script. Nothing of the reference is
compiled or run: the ``gray_image!`` / ``rgb_image!`` literals, the
``sum_image_pixels`` assertions, the ``put_pixel`` calls and the ``T::new``
point lists are parsed.

Usage: python tests/golden/make_golden_next.py path/to/imageproc/src
(or set IMAGEPROC_SRC to that directory)
"""

from __future__ import annotations

import json
import re
import os
import sys
from pathlib import Path

OUT = Path(__file__).with_name("reference_next_tests.json")


def macro_body(text: str, name: str, start: int = 0) -> tuple[str, int]:
    i = text.index(name + "!(", start) + len(name) + 1
    depth = 0
    for k in range(i, len(text)):
        if text[k] == "(":
            depth += 1
        elif text[k] == ")":
            depth -= 1
            if depth == 0:
                return text[i + 1 : k], k + 1
    raise ValueError("unbalanced")


def parse_image(body: str) -> dict:
    body = body.strip()
    dtype = "u8"
    m = re.match(r"type:\s*(\w+)\s*,", body)
    if m:
        dtype, body = m.group(1), body[m.end():]
    rows = [r.strip() for r in body.split(";") if r.strip()]
    if "[" in body:  # rgb rows of [a, b, c] pixels
        px = [[[int(v) for v in p.split(",")] for p in re.findall(r"\[([^\]]*)\]", r)] for r in rows]
        return {"type": dtype, "channels": 3, "rows": px}
    return {"type": dtype, "channels": 1, "rows": [[int(v) for v in r.split(",") if v.strip()] for r in rows]}


def test_body(text: str, name: str) -> tuple[str, int]:
    i = text.index(f"fn {name}(")
    j = text.index("\n    }\n", i)
    line = text.count("\n", 0, i) + 1
    return text[i:j], line


def integral_tests(src: str) -> list[dict]:
    cases = []
    for name, square in (("test_integral_image_gray", False), ("test_integral_squared_image_gray", True),
                         ("test_integral_image_rgb", False)):
        body, line = test_body(src, name)
        macro = "rgb_image" if "rgb" in name else "gray_image"
        img, end = macro_body(body, macro)
        exp, _ = macro_body(body, macro, end)
        cases.append({"name": name, "line": line, "square": square, "image": parse_image(img),
                      "expected": parse_image(exp)})
    for name in ("test_sum_image_pixels", "test_sum_image_pixels_rgb"):
        body, line = test_body(src, name)
        macro = "rgb_image" if "rgb" in name else "gray_image"
        img, _ = macro_body(body, macro)
        sums = []
        for m in re.finditer(r"sum_image_pixels\(&integral,\s*(\d+),\s*(\d+),\s*(\d+),\s*(\d+)\)(\[0\])?,\s*"
                             r"(\[[^\]]*\]|\d+)\)", body):
            exp = m.group(6)
            exp = [int(v) for v in exp.strip("[]").split(",")] if exp.startswith("[") else [int(exp)]
            sums.append({"ltrb": [int(m.group(k)) for k in range(1, 5)], "expected": exp})
        cases.append({"name": name, "line": line, "image": parse_image(img), "sums": sums})
    return cases


def put_pixels(block: str, var: str) -> list[list[int]]:
    return [[int(a), int(b), int(c)] for a, b, c in
            re.findall(var + r"\.put_pixel\((\d+),\s*(\d+),\s*Luma\(\[(\d+)u8\]\)\)", block)]


def suppress_tests(src: str) -> list[dict]:
    cases = []
    body, line = test_body(src, "test_suppress_non_maximum")
    size = [int(v) for v in re.search(r"GrayImage::new\((\d+),\s*(\d+)\)", body).groups()]
    radius = int(re.search(r"suppress_non_maximum\(&image,\s*(\d+)\)", body).group(1))
    cases.append({"name": "test_suppress_non_maximum", "line": line, "size": size, "radius": radius,
                  "pixels": put_pixels(body, "image"), "expected": put_pixels(body, "expected")})
    body, line = test_body(src, "test_suppress_non_maximum_handles_radius_greater_than_image_side")
    sizes = [[int(a), int(b)] for a, b in re.findall(r"GrayImage::new\((\d+),\s*(\d+)\)", body)]
    radius = int(re.search(r"suppress_non_maximum\(&image,\s*(\d+)\)", body).group(1))
    cases.append({"name": "test_suppress_non_maximum_handles_radius_greater_than_image_side", "line": line,
                  "sizes": sizes, "radius": radius})
    body, line = test_body(src, "test_local_maxima")
    ts_block = body[body.index("let ts"):body.index("let expected")]
    ex_block = body[body.index("let expected"):]
    pt = r"T::new\((\d+),\s*(\d+),\s*([0-9.]+)f32\)"
    radius = int(re.search(r"local_maxima\(&ts,\s*(\d+)\)", body).group(1))
    cases.append({"name": "test_local_maxima", "line": line, "radius": radius,
                  "points": [[int(a), int(b), float(c)] for a, b, c in re.findall(pt, ts_block)],
                  "expected": [[int(a), int(b), float(c)] for a, b, c in re.findall(pt, ex_block)]})
    return cases


def filter_tests(src: str) -> list[dict]:
    """filter_clamped's known answers: the Sobel test (i32 kernel -> i16) and the
    horizontal / vertical 1/3 box tests, which are filter_clamped with 1 x 3 and
    3 x 1 f32 kernels into u8."""
    cases = []
    body, line = test_body(src, "test_filter_clamped_with_results_outside_input_channel_range")
    kbody = body[body.index("Kernel::new(&[") + len("Kernel::new(&["):]
    kvals = [int(v) for v in kbody[:kbody.index("]")].replace("\n", " ").split(",") if v.strip()]
    kw, kh = (int(v) for v in re.search(r"\],\s*(\d+),\s*(\d+)\)", kbody).groups())
    img, end = macro_body(body, "gray_image")
    exp, _ = macro_body(body, "gray_image", end)
    cases.append({"name": "test_filter_clamped_with_results_outside_input_channel_range", "line": line,
                  "kernel_type": "i32", "kernel": kvals, "kernel_width": kw, "kernel_height": kh,
                  "image": parse_image(img), "expected": parse_image(exp)})
    for name, horizontal in (("test_horizontal_filter", True), ("test_vertical_filter", False)):
        body, line = test_body(src, name)
        img, end = macro_body(body, "gray_image")
        exp, _ = macro_body(body, "gray_image", end)
        m = re.search(r"\[1f32 / (\d+)f32; (\d+)\]", body)
        n = int(m.group(2))
        cases.append({"name": name, "line": line, "kernel_type": "f32", "kernel_one_over": int(m.group(1)),
                      "kernel_width": n if horizontal else 1, "kernel_height": 1 if horizontal else n,
                      "image": parse_image(img), "expected": parse_image(exp)})
    # separable_filter_equal = vertical_filter(horizontal_filter(.)) with a 3-tap kernel
    for name in ("test_separable_filter", "test_separable_filter_integer_kernel"):
        body, line = test_body(src, name)
        img, end = macro_body(body, "gray_image")
        exp, _ = macro_body(body, "gray_image", end)
        m = re.search(r"let kernel = \[1(f32 / (\d+)f32|i32); (\d+)\]", body)
        case = {"name": name, "line": line, "separable": True, "taps": int(m.group(3)),
                "image": parse_image(img), "expected": parse_image(exp)}
        if m.group(2):
            case.update(kernel_type="f32", kernel_one_over=int(m.group(2)))
        else:
            case.update(kernel_type="i32", kernel_value=1)
        cases.append(case)
    return cases


def main() -> None:
    if len(sys.argv) > 1:
        src = Path(sys.argv[1])
    elif os.environ.get("IMAGEPROC_SRC"):
        src = Path(os.environ["IMAGEPROC_SRC"])
    else:
        sys.exit(__doc__)
    data = {
        "reference": "image-rs/imageproc 0.27.0",
        "integral_image": {"file": "src/integral_image.rs",
                           "cases": integral_tests((src / "integral_image.rs").read_text())},
        "suppress": {"file": "src/suppress.rs", "cases": suppress_tests((src / "suppress.rs").read_text())},
        "filter": {"file": "src/filter/mod.rs", "cases": filter_tests((src / "filter" / "mod.rs").read_text())},
    }
    OUT.write_text(json.dumps(data, indent=1))
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
