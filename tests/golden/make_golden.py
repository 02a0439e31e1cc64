"""Extract the reference's template-matching known-answer tests as fixtures.

Reads imageproc's ``src/template_matching.rs`` (the ``mod tests`` block,
lines 513-834 of imageproc 0.27.0) as TEXT and writes
``reference_unit_tests.json`` beside this script. Nothing of the reference is
compiled or run: the ``gray_image!`` literals are parsed, and the expected
values that the tests build with f32 expressions such as
``14.0 / (22.0 * tss).sqrt()`` are evaluated with numpy float32 arithmetic,
which rounds each operation like Rust's f32.

Usage: python tests/golden/make_golden.py path/to/imageproc/src/template_matching.rs
(or set IMAGEPROC_SRC to the imageproc source directory)
"""

from __future__ import annotations

import json
import re
import os
import sys
from pathlib import Path

import numpy as np

OUT = Path(__file__).with_name("reference_unit_tests.json")
REL = "src/template_matching.rs"

METHODS = {
    "SumOfSquaredErrors": 0,
    "SumOfSquaredErrorsNormalized": 1,
    "CrossCorrelation": 2,
    "CrossCorrelationNormalized": 3,
}


def macro_args(text: str, start: int) -> tuple[str, int]:
    """Return the text inside the balanced parentheses opening at ``start``."""
    assert text[start] == "("
    depth = 0
    for k in range(start, len(text)):
        if text[k] == "(":
            depth += 1
        elif text[k] == ")":
            depth -= 1
            if depth == 0:
                return text[start + 1 : k], k + 1
    raise ValueError("unbalanced parentheses")


def f32_expr(expr: str, env: dict[str, np.float32]) -> np.float32:
    """Evaluate a float literal or ``A / (B * name).sqrt()`` in f32."""
    expr = expr.strip()
    m = re.fullmatch(r"([0-9.]+)\s*/\s*\(\s*([0-9.]+)\s*\*\s*(\w+)\s*\)\.sqrt\(\)", expr)
    if m:
        a = np.float32(float(m.group(1)))
        b = np.float32(float(m.group(2)))
        prod = np.float32(b * env[m.group(3)])
        return np.float32(a / np.sqrt(prod, dtype=np.float32))
    return np.float32(float(expr.rstrip(".") if expr.endswith(".") else expr))


def parse_gray_image(args: str, env: dict[str, np.float32]) -> dict:
    args = args.strip()
    dtype = "u8"
    m = re.match(r"type:\s*(\w+)\s*,", args)
    if m:
        dtype = m.group(1)
        args = args[m.end() :]
    rows = [r for r in (s.strip() for s in args.split(";")) if r]
    if dtype == "f32":
        vals = [[f32_expr(v, env) for v in r.split(",") if v.strip()] for r in rows]
        return {
            "type": "f32",
            "rows": [[float(v) for v in r] for r in vals],
            "bits": [[int(np.float32(v).view(np.uint32)) for v in r] for r in vals],
        }
    vals = [[int(v) for v in r.split(",") if v.strip()] for r in rows]
    return {"type": dtype, "rows": vals}


def image_expr(text: str, env) -> dict:
    text = text.strip().lstrip("&")
    m = re.fullmatch(r"GrayImage::new\(\s*(\d+)\s*,\s*(\d+)\s*\)", text)
    if m:
        w, h = int(m.group(1)), int(m.group(2))
        return {"type": "u8", "rows": [[0] * w for _ in range(h)]}
    k = text.index("gray_image!")
    args, _ = macro_args(text, text.index("(", k))
    return parse_gray_image(args, env)


def split_top_level(args: str) -> list[str]:
    parts, depth, cur = [], 0, []
    for ch in args:
        if ch in "([":
            depth += 1
        elif ch in ")]":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    if "".join(cur).strip():
        parts.append("".join(cur))
    return [p.strip() for p in parts]


def main(src: Path) -> None:
    text = src.read_text()
    lines = text.splitlines()
    tests_start = next(i for i, l in enumerate(lines) if l.startswith("mod tests"))
    cases = []
    fn_re = re.compile(r"^\s*fn (\w+)\(\) \{")
    for i in range(tests_start, len(lines)):
        m = fn_re.match(lines[i])
        if not m:
            continue
        name = m.group(1)
        # function body: up to the matching closing brace
        depth, j = 0, i
        while True:
            depth += lines[j].count("{") - lines[j].count("}")
            if depth == 0 and j > i:
                break
            j += 1
        attrs_from = i
        while attrs_from > 0 and lines[attrs_from - 1].strip().startswith("#["):
            attrs_from -= 1
        attrs = " ".join(lines[attrs_from:i])
        body = "\n".join(lines[i : j + 1])
        case = {"name": name, "source": f"{REL}:{attrs_from + 1}-{j + 1}",
                "should_panic": "should_panic" in attrs}
        env = {}
        for tm in re.finditer(r"let (\w+) = ([0-9.]+)f32;", body):
            env[tm.group(1)] = np.float32(float(tm.group(2)))
        bindings = {}
        for bm in re.finditer(r"let (\w+) = gray_image!", body):
            args, _ = macro_args(body, body.index("(", bm.end() - 1))
            bindings[bm.group(1)] = parse_gray_image(args, env)
        if name == "test_find_extremes":
            ex = re.search(r"max_value: (\d+),\s*min_value: (\d+),\s*max_value_location: "
                           r"\((\d+), (\d+)\),\s*min_value_location: \((\d+), (\d+)\)", body)
            case.update(kind="find_extremes", image=bindings["image"],
                        expected={"max_value": int(ex.group(1)), "min_value": int(ex.group(2)),
                                  "max_value_location": [int(ex.group(3)), int(ex.group(4))],
                                  "min_value_location": [int(ex.group(5)), int(ex.group(6))]})
            cases.append(case)
            continue
        call = re.search(r"(match_template_with_mask|match_template)\(", body)
        args, _ = macro_args(body, call.end() - 1)
        parts = split_top_level(args)
        masked = call.group(1) == "match_template_with_mask"
        resolve = lambda p: bindings[p.lstrip("&")] if p.lstrip("&") in bindings else image_expr(p, env)
        case["kind"] = "match_template_with_mask" if masked else "match_template"
        case["image"] = resolve(parts[0])
        case["template"] = resolve(parts[1])
        case["method"] = METHODS[parts[2].split("::")[-1]]
        if masked:
            case["mask"] = resolve(parts[3])
        if "expected" in bindings:
            case["expected"] = bindings["expected"]
        elif not case["should_panic"]:
            em = re.search(r"assert_pixels_eq!\(\s*match_template", body)
            tail = body[em.end():]
            _, after = macro_args(tail, tail.index("("))
            k = tail.index("gray_image!", after)
            eargs, _ = macro_args(tail, tail.index("(", k))
            case["expected"] = parse_gray_image(eargs, env)
        case["parallel_variant_checked"] = "_parallel(" in body
        cases.append(case)
    OUT.write_text(json.dumps({"reference": "imageproc 0.27.0", "file": REL,
                               "cases": cases}, indent=1) + "\n")
    print(f"wrote {len(cases)} cases to {OUT}")


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(Path(sys.argv[1]))
    elif os.environ.get("IMAGEPROC_SRC"):
        main(Path(os.environ["IMAGEPROC_SRC"]) / "template_matching.rs")
    else:
        sys.exit(__doc__)
