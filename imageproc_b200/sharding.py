"""Splitting one matching query over several GPUs (one process per GPU).

Output positions are independent, so a query shards without any exchange on
the data path; the only collectives are the final gathers:

* Row bands of one large score map: rank r computes output rows
  [y0, y1) from image rows [y0, y1 + h - 1) (an (h - 1)-row halo read from
  the rank's own copy of the image), and the bands are gathered in rank order.
* Templates of a many-template query (an (n, h, w) bank against one image):
  each rank scores a contiguous slice of the templates against its own copy
  of the image; the per-template results are gathered in rank order.
* find_extremes (src/template_matching.rs:479-511) of a map split in bands:
  each rank reduces its band to two packed 64-bit keys, (value order, global
  row-major index) for the minimum and (value order, complemented index) for
  the maximum, and one MIN and one MAX all-reduce combine them. Comparing
  values first and then the lower index is the reference's first-occurrence
  rule (strict < and > in row-major order), so the reduced result equals the
  single-map one for maps without NaN (every exact score map here).

`compute` arguments are callables so the same host logic drives the CUDA
library (the product: `imageproc_b200.template_matching` /
`imageproc_b200.device`) and, in the CPU tests, the oracle. Collectives use
torch.distributed (NCCL on GPUs, gloo in the tests); every rank takes the same
collective steps in the same order.
"""

from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def split_range(n: int, parts: int) -> list[tuple[int, int]]:
    """[0, n) in `parts` contiguous slices whose sizes differ by at most one."""
    base, extra = divmod(n, parts)
    out, start = [], 0
    for r in range(parts):
        size = base + (1 if r < extra else 0)
        out.append((start, start + size))
        start += size
    return out


def band_rows(H: int, h: int, parts: int) -> list[tuple[int, int, int, int]]:
    """Per rank: output rows [y0, y1) of a (H - h + 1)-row map and the image rows
    [y0, y1 + h - 1) they read (the band plus its (h - 1)-row halo)."""
    return [(y0, y1, y0, y1 + h - 1 if y1 > y0 else y0) for y0, y1 in split_range(H - h + 1, parts)]


def order_keys_f32(a: np.ndarray) -> np.ndarray:
    """u32 keys that order like the f32 values (no NaN)."""
    b = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    return np.where(b >> np.uint64(31), ~b & np.uint64(0xFFFFFFFF), b | np.uint64(0x80000000))


def _value_of_key(k: int) -> np.float32:
    k = int(k) & 0xFFFFFFFF
    b = (k & 0x7FFFFFFF) if k & 0x80000000 else (~k & 0xFFFFFFFF)
    return np.array([b], np.uint32).view(np.float32)[0]


def band_extremes_keys(band: np.ndarray, y0: int, Wo: int) -> tuple[int, int]:
    """(min key, max key) of a band of score rows starting at map row y0:
    (order key << 32) | global index for the minimum, (order key << 32) |
    (2^32 - 1 - global index) for the maximum. An empty band gives the
    identities (2^64 - 1, 0)."""
    if band.size == 0:
        return (1 << 64) - 1, 0
    keys = order_keys_f32(band.reshape(-1))
    idx = np.arange(band.size, dtype=np.uint64) + np.uint64(y0 * Wo)
    kmin = int(np.min((keys << np.uint64(32)) | idx))
    kmax = int(np.max((keys << np.uint64(32)) | (np.uint64(0xFFFFFFFF) - idx)))
    return kmin, kmax


def decode_extremes(kmin: int, kmax: int, Wo: int):
    """(max_value, min_value, (max_x, max_y), (min_x, min_y)) from the keys."""
    imin = kmin & 0xFFFFFFFF
    imax = 0xFFFFFFFF - (kmax & 0xFFFFFFFF)
    return (_value_of_key(kmax >> 32), _value_of_key(kmin >> 32), (imax % Wo, imax // Wo),
            (imin % Wo, imin // Wo))


def _to_i64(k: int) -> int:
    v = k ^ (1 << 63)
    return v - (1 << 64) if v >= (1 << 63) else v


def _from_i64(v: int) -> int:
    return ((v + (1 << 64)) if v < 0 else v) ^ (1 << 63)


def allreduce_extremes_keys(kmin: int, kmax: int, group=None) -> tuple[int, int]:
    """MIN of the min keys and MAX of the max keys over the ranks. Unsigned
    64-bit keys travel as signed int64 with the top bit flipped, which keeps
    their order."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    lo = torch.tensor([_to_i64(kmin)], dtype=torch.int64, device=dev)
    hi = torch.tensor([_to_i64(kmax)], dtype=torch.int64, device=dev)
    dist.all_reduce(lo, op=dist.ReduceOp.MIN, group=group)
    dist.all_reduce(hi, op=dist.ReduceOp.MAX, group=group)
    return _from_i64(int(lo.item())), _from_i64(int(hi.item()))


def _gather_objects(obj, group=None) -> list:
    import torch.distributed as dist
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, obj, group=group)
    return out


def match_template_bands(image: np.ndarray, template: np.ndarray, method: int,
                         compute: Callable[[np.ndarray, np.ndarray, int], np.ndarray], *,
                         gather_map: bool = True, group=None):
    """One score map split in output-row bands over the ranks of `group`.

    compute(image_rows, template, method) scores one band (the library's
    match_template on this rank's GPU, or the oracle in tests). Returns
    (map or None, extremes): the full map on every rank when gather_map, and
    find_extremes of the whole map from the packed-key reduction."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    H, W = image.shape
    h, w = template.shape
    Wo = W - w + 1
    y0, y1, r0, r1 = band_rows(H, h, world)[rank]
    band = compute(np.ascontiguousarray(image[r0:r1]), template, method) if y1 > y0 else \
        np.zeros((0, Wo), np.float32)
    kmin, kmax = allreduce_extremes_keys(*band_extremes_keys(band, y0, Wo), group=group)
    full = np.concatenate(_gather_objects(band, group), axis=0) if gather_map else None
    return full, decode_extremes(kmin, kmax, Wo)


def match_templates_split(image: np.ndarray, templates: np.ndarray, method: int,
                          compute: Callable[[np.ndarray, np.ndarray, int], Sequence], *, group=None) -> list:
    """The templates of an (n, h, w) bank split in contiguous slices over the
    ranks, each scored against the rank's own copy of the image by
    compute(image, template_slice, method) -> one result per template
    (extremes records); the results come back in template order on every rank."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    t0, t1 = split_range(templates.shape[0], world)[rank]
    mine = list(compute(image, np.ascontiguousarray(templates[t0:t1]), method)) if t1 > t0 else []
    out = []
    for part in _gather_objects(mine, group):
        out.extend(part)
    return out
