"""imageproc's examples/template_matching.rs on the GPU.

    python -m imageproc_b200.examples.template_matching input_path output_dir \\
        template_x template_y template_w template_h [parallel]

Loads the image at input_path (PNG or 8-bit netpbm) as Luma, extracts the
region (template_x, template_y, template_w, template_h) as the template,
matches it with SumOfSquaredErrors and SumOfSquaredErrorsNormalized, and
writes template.png, image.png (the image with the region outlined in green),
result_sse.png and result_sse_norm.png (each score map rescaled to 0..255,
padded to the image size and outlined) to output_dir, as the reference
example does (:136-190). Decoding and encoding run on the host; cropping,
matching, rescaling, padding and drawing run in one device pipeline
(ipb_example_template_matching). The optional `parallel` flag ("true" or
"false") is accepted as the reference's is; the device path gives the same
scores either way, as match_template_parallel does.

A failed check ends the program as a Rust panic does: the message on stderr
and exit status 101.
"""

from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

from .. import _lib, png
from .._lib import Panic, check

USAGE = """
Usage:

    python -m imageproc_b200.examples.template_matching input_path output_dir template_x template_y \\
        template_w template_h [parallel]

Reads input_path, cuts the template_w x template_h region at (template_x, template_y) out of it as the
template, scores every placement of that template with the squared-error and normalised squared-error
methods, and writes the template, the outlined image and both rescaled score maps to output_dir.
parallel ("true" or "false", default false) picks the parallel entry point; the scores do not change.
"""


def _u32(s: str) -> int:
    """`str::parse::<u32>().unwrap()`."""
    digits = s[1:] if s.startswith("+") else s
    if not digits.isdigit() or int(digits) >= 2**32:
        raise Panic(f"called `Result::unwrap()` on an `Err` value: ParseIntError for {s!r}")
    return int(digits)


def parse_args(args: list[str]) -> dict:
    """TemplateMatchingArgs::parse (examples/template_matching.rs:27-59)."""
    if len(args) < 7:
        raise Panic(USAGE)
    parallel = False
    if len(args) > 7:
        if args[7] not in ("true", "false"):  # bool::from_str
            raise Panic("called `Result::unwrap()` on an `Err` value: ParseBoolError")
        parallel = args[7] == "true"
    return {"input_path": Path(args[1]), "output_dir": Path(args[2]), "template_x": _u32(args[3]),
            "template_y": _u32(args[4]), "template_w": _u32(args[5]), "template_h": _u32(args[6]),
            "parallel": parallel}


def run_pipeline(image: np.ndarray, x: int, y: int, w: int, h: int) -> dict[str, np.ndarray]:
    """The example's images for a Luma image: template (h, w), image (H, W, 3)
    with the region outlined, result_sse and result_sse_norm (H, W, 3)."""
    a = np.ascontiguousarray(image, np.uint8)
    if a.ndim != 2:
        raise TypeError("the example works on (H, W) uint8 Luma images")
    H, W = a.shape
    if not (x + w < W and y + h < H):  # copy_sub_image (:79-82)
        raise Panic("invalid sub-image")
    out = {"template": _lib.host_empty((h, w), np.uint8), "image": _lib.host_empty((H, W, 3), np.uint8),
           "result_sse": _lib.host_empty((H, W, 3), np.uint8),
           "result_sse_norm": _lib.host_empty((H, W, 3), np.uint8)}
    L = _lib.lib()
    L.ipb_example_template_matching.argtypes = [C.c_void_p] + [C.c_uint32] * 6 + [C.c_void_p] * 4
    L.ipb_example_template_matching.restype = C.c_int
    check(L.ipb_example_template_matching(a.ctypes.data, W, H, x, y, w, h, out["template"].ctypes.data,
                                          out["image"].ctypes.data, out["result_sse"].ctypes.data,
                                          out["result_sse_norm"].ctypes.data))
    return out


def main(argv: list[str]) -> None:
    args = parse_args(argv)
    out_dir = args["output_dir"]
    if not out_dir.is_dir():
        try:
            out_dir.mkdir()  # fs::create_dir: the parent must exist
        except OSError as e:
            raise Panic(f"Failed to create output directory: {e}") from e
    if not args["input_path"].is_file():
        raise Panic("Input file does not exist")
    try:
        image = png.to_luma8(png.read_image(args["input_path"]))
    except (OSError, png.ImageFormatError) as e:
        raise Panic(f"Could not load image at {str(args['input_path'])!r}: {e}") from e
    res = run_pipeline(image, args["template_x"], args["template_y"], args["template_w"], args["template_h"])
    png.write_png(out_dir / "template.png", res["template"])
    png.write_png(out_dir / "image.png", res["image"])
    png.write_png(out_dir / "result_sse.png", res["result_sse"])
    png.write_png(out_dir / "result_sse_norm.png", res["result_sse_norm"])


if __name__ == "__main__":
    try:
        main(sys.argv)
    except Panic as e:
        print(f"thread 'main' panicked:\n{e}", file=sys.stderr)
        sys.exit(101)
