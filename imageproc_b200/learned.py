"""Learned proposals for many-template matching (ipb_proposal_net_*,
ipb_propose_and_match_device).

No counterpart in the reference: imageproc scores every window
(match_template, src/template_matching.rs:78-92) and takes find_extremes
(:479-511). Here a small convolutional network proposes where each 48 x 48
template matches a large image; the proposals are scored exactly, certified
by a lower bound on every other window, and templates that cannot be
certified fall back to the exhaustive kernel, so every answer equals the
exhaustive SumOfSquaredErrors minimum (first occurrence in row-major order).

Training data are seeded synthetic scenes (value noise plus flat rectangles,
as the 8192 x 8192 workload); each (crop, template) pair is labelled by the
exhaustive kernel: the template's best window in its crop.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _lib, synthetic
from ._lib import check

N_PARAMS = 37312
TPL = 48
CENTRE = 5
WEIGHTS = Path(__file__).resolve().parent / "proposal_net_weights.npy"

PATH_PROPOSED, PATH_LOW_MARGIN, PATH_NOT_CERTIFIED = 0, 1, 2


class ProposeOptions(C.Structure):
    _fields_ = [("top_k", C.c_uint32), ("min_margin", C.c_float), ("certify", C.c_int)]


class ProposalResult(C.Structure):
    _fields_ = [("value", C.c_float), ("x", C.c_uint32), ("y", C.c_uint32), ("margin", C.c_float),
                ("path", C.c_uint32), ("uncertified", C.c_uint32)]


@dataclass(frozen=True)
class Answer:
    value: float          # minimum SumOfSquaredErrors score (f32)
    location: tuple       # (x, y) of its first occurrence
    margin: float         # heatmap confidence margin
    path: int             # 0 proposals, 1 fallback (low margin), 2 fallback (not certified)
    uncertified: int = 0  # 4 x 4 position blocks the certificate could not exclude


def _bind():
    L = _lib.lib()
    if getattr(L, "_learned_bound", False):
        return L
    vp, u32 = C.c_void_p, C.c_uint32
    L.ipb_proposal_net_create.argtypes = [vp, C.POINTER(vp)]
    L.ipb_proposal_net_destroy.argtypes = [vp]
    L.ipb_proposal_net_get_params.argtypes = [vp, vp]
    L.ipb_proposal_net_gradients.argtypes = [vp, vp, u32, u32, u32, vp, u32, vp, C.POINTER(C.c_float), vp, vp]
    L.ipb_proposal_net_train_step.argtypes = [vp, vp, u32, u32, u32, vp, u32, vp, C.c_float,
                                              C.POINTER(C.c_float), vp]
    L.ipb_propose_and_match_device.argtypes = [vp, vp, u32, u32, vp, u32, u32, u32, C.c_int,
                                               C.POINTER(ProposeOptions), C.POINTER(ProposalResult), vp]
    L.ipb_proposal_net_features.argtypes = [vp, vp, u32, u32, C.c_int, vp, vp]
    L.ipb_match_proposals_device.argtypes = [vp, u32, u32, vp, u32, u32, u32, C.c_int, vp, u32,
                                             C.POINTER(ProposeOptions), C.POINTER(ProposalResult), vp]
    for f in ("ipb_proposal_net_create", "ipb_proposal_net_destroy", "ipb_proposal_net_get_params",
              "ipb_proposal_net_gradients", "ipb_proposal_net_train_step", "ipb_propose_and_match_device",
              "ipb_proposal_net_features", "ipb_match_proposals_device"):
        getattr(L, f).restype = C.c_int
    L._learned_bound = True
    return L


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights (std sqrt(2 / fan_in)), zero biases, from `seed`."""
    g = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    off = 0
    for cin in (1, 32, 32, 32, 32):
        n = 32 * cin * 9
        p[off:off + n] = g.normal(0.0, np.sqrt(2.0 / (cin * 9)), n).astype(np.float32)
        off += n + 32
    assert off == N_PARAMS
    return p


def _stream(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream) if stream.cuda_stream else None


def _u8(t: torch.Tensor, what: str) -> torch.Tensor:
    if t.dtype != torch.uint8 or not t.is_cuda or not t.is_contiguous():
        raise TypeError(f"{what} must be a contiguous uint8 CUDA tensor")
    return t


class ProposalNet:
    """The proposal network on the current CUDA device."""

    def __init__(self, params: np.ndarray | None = None, *, seed: int = 0):
        L = _bind()
        p = np.ascontiguousarray(init_params(seed) if params is None else params, np.float32)
        if p.shape != (N_PARAMS,):
            raise ValueError(f"expected {N_PARAMS} parameters")
        self._h = C.c_void_p()
        check(L.ipb_proposal_net_create(p.ctypes.data_as(C.c_void_p), C.byref(self._h)))

    @classmethod
    def trained(cls) -> "ProposalNet":
        """The network with the weights shipped with the package."""
        return cls(np.load(WEIGHTS))

    def close(self):
        if self._h:
            _bind().ipb_proposal_net_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.empty(N_PARAMS, np.float32)
        check(_bind().ipb_proposal_net_get_params(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def save(self, path):
        np.save(path, self.params())

    @staticmethod
    def _batch_args(scenes, templates, positives):
        _u8(scenes, "scenes")
        _u8(templates, "templates")
        if scenes.dim() != 3 or templates.dim() != 3 or tuple(templates.shape[1:]) != (TPL, TPL):
            raise ValueError("scenes (n, h, w) and templates (t, 48, 48) expected")
        if positives.dtype != torch.int64 or not positives.is_cuda or positives.numel() != templates.shape[0]:
            raise ValueError("one int64 CUDA positive per template expected")
        n, h, w = scenes.shape
        return n, h, w

    def gradients(self, scenes, templates, positives, stream=None):
        """(loss, gradients) of a batch; gradients in the parameter layout."""
        n, h, w = self._batch_args(scenes, templates, positives)
        loss = C.c_float()
        grads = np.empty(N_PARAMS, np.float32)
        check(_bind().ipb_proposal_net_gradients(
            self._h, scenes.data_ptr(), n, h, w, templates.data_ptr(), templates.shape[0],
            positives.data_ptr(), C.byref(loss), grads.ctypes.data_as(C.c_void_p), _stream(stream)))
        return float(loss.value), grads

    def train_step(self, scenes, templates, positives, lr: float, stream=None) -> float:
        n, h, w = self._batch_args(scenes, templates, positives)
        loss = C.c_float()
        check(_bind().ipb_proposal_net_train_step(
            self._h, scenes.data_ptr(), n, h, w, templates.data_ptr(), templates.shape[0],
            positives.data_ptr(), C.c_float(lr), C.byref(loss), _stream(stream)))
        return float(loss.value)

    def features(self, image: torch.Tensor, kernel: int = 0, stream=None) -> torch.Tensor:
        """The network's 32-channel features of one image (sides multiples of 4),
        as a (32, H/4, W/4) float32 tensor. kernel 0: tcgen05 (the query path),
        1: mma.sync (the training path)."""
        _u8(image, "image")
        H, W = image.shape
        raw = torch.empty((H // 4, 4, W // 4, 8), dtype=torch.bfloat16, device=image.device)
        check(_bind().ipb_proposal_net_features(self._h, image.data_ptr(), W, H, int(kernel), raw.data_ptr(),
                                                _stream(stream)))
        return raw.permute(1, 3, 0, 2).reshape(32, H // 4, W // 4).float()

    def propose_and_match(self, image: torch.Tensor, templates: torch.Tensor, *, top_k: int = 16,
                          min_margin: float = 0.1, certify: bool = True, stream=None) -> list[Answer]:
        """SumOfSquaredErrors minimum of every 48 x 48 template (a (t, 48, 48)
        uint8 CUDA tensor) in `image` (sides multiples of 32)."""
        _u8(image, "image")
        _u8(templates, "templates")
        H, W = image.shape
        n = templates.shape[0]
        res = (ProposalResult * max(n, 1))()
        opt = ProposeOptions(top_k, min_margin, int(certify))
        if templates.dim() != 3:
            raise ValueError("templates must be a (t, h, w) tensor")
        th, tw = templates.shape[1], templates.shape[2]
        check(_bind().ipb_propose_and_match_device(
            self._h, image.data_ptr(), W, H, templates.data_ptr(), tw, th, n, 0, C.byref(opt), res,
            _stream(stream)))
        return [Answer(float(r.value), (int(r.x), int(r.y)), float(r.margin), int(r.path), int(r.uncertified))
                for r in res[:n]]


def match_proposals(image: torch.Tensor, templates: torch.Tensor, origins: torch.Tensor, *,
                    certify: bool = True, stream=None) -> list[Answer]:
    """The verification, certification and fallback stages with proposals
    from elsewhere (ipb_match_proposals_device): `origins` is a (t, k) int32
    CUDA tensor of template origins y * (W - 47) + x, k <= 16 per template,
    each the centre of a 32 x 32 window scored exactly. Same answers as
    propose_and_match (exact SumOfSquaredErrors minima); margin is +inf."""
    _u8(image, "image")
    _u8(templates, "templates")
    if templates.dim() != 3:
        raise ValueError("templates must be a (t, h, w) tensor")
    if origins.dtype != torch.int32 or not origins.is_cuda or origins.dim() != 2 or \
            origins.shape[0] != templates.shape[0] or not origins.is_contiguous():
        raise ValueError("origins must be a contiguous (t, k) int32 CUDA tensor")
    H, W = image.shape
    n, k = origins.shape
    res = (ProposalResult * max(n, 1))()
    opt = ProposeOptions(k, 0.1, int(certify))
    check(_bind().ipb_match_proposals_device(
        image.data_ptr(), W, H, templates.data_ptr(), templates.shape[2], templates.shape[1], n, 0,
        origins.data_ptr(), k, C.byref(opt), res, _stream(stream)))
    return [Answer(float(r.value), (int(r.x), int(r.y)), float(r.margin), int(r.path), int(r.uncertified))
            for r in res[:n]]


def pyramid_origins(image: torch.Tensor, templates: torch.Tensor, k: int = 16) -> torch.Tensor:
    """Coarse-pyramid proposals, the baseline the network is compared with
    (computed with torch operators; not a query path): SumOfSquaredErrors of
    the 4x box-downsampled templates over the 4x box-downsampled image, the
    best position of each 8 x 8 cell of that map, the k best cells per
    template. Returns (t, k) int32 origins for match_proposals: 4x each
    downsampled position, y * (W - 47) + x."""
    import torch.nn.functional as F
    H, W = image.shape
    ds = F.avg_pool2d(image.float()[None, None], 4)
    tds = F.avg_pool2d(templates.float()[:, None], 4)
    cross = F.conv2d(ds, tds)[0]
    sq = F.avg_pool2d(ds * ds, tds.shape[-1], stride=1)[0, 0] * float(tds.shape[-1] * tds.shape[-2])
    sse = sq[None] - 2.0 * cross + (tds * tds).sum((1, 2, 3))[:, None, None]
    T, Hm, Wm = sse.shape
    vals, idx = F.max_pool2d(-sse[:, None], 8, stride=8, ceil_mode=True, return_indices=True)
    top = vals.reshape(T, -1).topk(k, dim=1).indices
    pos = idx.reshape(T, -1).gather(1, top)
    qy, qx = pos // Wm, pos % Wm
    Wo, Ho = W - templates.shape[2] + 1, H - templates.shape[1] + 1
    ox, oy = (4 * qx).clamp(max=Wo - 1), (4 * qy).clamp(max=Ho - 1)
    return (oy * Wo + ox).to(torch.int32).contiguous()


# ---- training data ----------------------------------------------------------------

def training_scene(seed: int, side: int = 8192) -> np.ndarray:
    """A training scene drawn like the 8192 x 8192 workload (value noise plus
    500 flat rectangles), from seeds the benchmark does not use."""
    image, _, _ = synthetic.rect_scene(W=side, H=side, n_templates=0, seed=seed)
    return image


def training_batch(scenes: torch.Tensor, n: int, g: np.random.Generator, crop: int = 96):
    """n (crop, template, positive) triples from the (k, S, S) uint8 CUDA
    scenes: crops at multiples of 4, a 48 x 48 template cut from each crop with
    a brightness offset in [-10, 10] and noise in [-6, 6] (clamped), and the
    positive from the exhaustive kernel: the template's best window in its
    crop (find_extremes' minimum of the SumOfSquaredErrors map), downsampled
    to the nearest position, plus 5."""
    from . import device
    k, S, _ = scenes.shape
    si = g.integers(0, k, n)
    cy = g.integers(0, (S - crop) // 4 + 1, n) * 4
    cx = g.integers(0, (S - crop) // 4 + 1, n) * 4
    ty = g.integers(0, crop - TPL + 1, n)
    tx = g.integers(0, crop - TPL + 1, n)
    dev = scenes.device
    ar = torch.arange(crop, device=dev)
    rows = torch.as_tensor(cy, device=dev)[:, None] + ar[None, :]
    cols = torch.as_tensor(cx, device=dev)[:, None] + ar[None, :]
    crops = scenes[torch.as_tensor(si, device=dev)[:, None, None], rows[:, :, None], cols[:, None, :]].contiguous()
    ta = torch.arange(TPL, device=dev)
    trows = torch.as_tensor(ty, device=dev)[:, None] + ta[None, :]
    tcols = torch.as_tensor(tx, device=dev)[:, None] + ta[None, :]
    base = crops[torch.arange(n, device=dev)[:, None, None], trows[:, :, None], tcols[:, None, :]].to(torch.int16)
    off = torch.as_tensor(g.integers(-10, 11, n), device=dev, dtype=torch.int16)[:, None, None]
    noise = torch.as_tensor(g.integers(-6, 7, (n, TPL, TPL)), device=dev, dtype=torch.int16)
    templates = (base + off + noise).clamp(0, 255).to(torch.uint8).contiguous()
    # labels from the exhaustive kernel
    batch = device.Batch([(crops[i], templates[i], 0) for i in range(n)], extremes=True)
    batch.run()
    ex = batch.extremes_host()
    ds = crop // 4
    pos = np.empty(n, np.int64)
    for i, e in enumerate(ex):
        ax, ay = e.min_value_location
        px, py = (ax + 2) // 4 + CENTRE, (ay + 2) // 4 + CENTRE
        pos[i] = (i * ds + py) * ds + px
    return crops, templates, torch.as_tensor(pos, device=dev)


def train(net: ProposalNet, scenes: torch.Tensor, *, pairs: int = 200_000, batch: int = 128,
          lr: float = 1e-3, seed: int = 0, log_every: int = 100, crop: int = 96, epochs: int = 1,
          log=print) -> list[float]:
    """Adam over `pairs` seeded (crop, template) pairs in batches of `batch`,
    `epochs` passes over the same pairs (the generator restarts from `seed`
    each pass); returns the per-step losses."""
    steps = (pairs + batch - 1) // batch
    total = steps * epochs
    losses = []
    for e in range(epochs):
        g = np.random.default_rng(seed)
        for s in range(steps):
            crops, templates, pos = training_batch(scenes, batch, g, crop)
            k = e * steps + s
            # cosine decay to a tenth over all passes
            lr_s = lr * (0.1 + 0.9 * 0.5 * (1.0 + np.cos(np.pi * k / max(1, total))))
            losses.append(net.train_step(crops, templates, pos, lr_s))
            if log and (k % log_every == 0 or k == total - 1):
                log(f"step {k}/{total} loss {np.mean(losses[-log_every:]):.4f} lr {lr_s:.2e}")
    return losses


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="train the proposal network on the GPU")
    ap.add_argument("--pairs", type=int, default=200_000)
    ap.add_argument("--batch", type=int, default=128)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--scenes", type=int, default=4)
    ap.add_argument("--side", type=int, default=8192)
    ap.add_argument("--crop", type=int, default=96)
    ap.add_argument("--epochs", type=int, default=1)
    ap.add_argument("--out", default=str(WEIGHTS))
    args = ap.parse_args(argv)
    torch.cuda.set_device(0)
    imgs = [training_scene(1000 + k, args.side) for k in range(args.scenes)]
    scenes = torch.from_numpy(np.stack(imgs)).cuda()
    net = ProposalNet(seed=args.seed)
    losses = train(net, scenes, pairs=args.pairs, batch=args.batch, lr=args.lr, seed=args.seed,
                   crop=args.crop, epochs=args.epochs)
    net.save(args.out)
    print(f"saved {args.out}; loss {np.mean(losses[:50]):.4f} -> {np.mean(losses[-50:]):.4f}")


if __name__ == "__main__":
    main()
