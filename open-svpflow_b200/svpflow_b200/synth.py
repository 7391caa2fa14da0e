"""Seeded synthetic YUV420P8 clips for tests and benchmarks.

Stands in for real video (the reference publishes no dataset for this path):
frame 0 is uniform noise in 0..255 blurred by a separable Gaussian (sigma 2 luma,
1 chroma; radius ceil(3 sigma); float accumulation, rounded). Each following clean
frame is the previous one shifted by an integer global motion drawn uniformly from
[-R, R]^2 (edges replicated), with `objects` textured rectangles (32-96 px sides)
pasted on top, each moving with its own constant velocity from [-M, M]^2. Every
output frame adds fresh Gaussian noise (sigma `noise`) to its clean frame, rounded
and clamped to 0..255. Chroma planes move by half the luma motion.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def _kernel(sigma: float) -> np.ndarray:
    r = int(math.ceil(3 * sigma))
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-(x * x) / (2 * sigma * sigma))
    return (k / k.sum()).astype(np.float32)


def _blur(img: np.ndarray, sigma: float) -> np.ndarray:
    k = _kernel(sigma)
    r = len(k) // 2
    a = np.pad(img.astype(np.float32), ((0, 0), (r, r)), mode="edge")
    h = sum(k[i] * a[:, i:i + img.shape[1]] for i in range(len(k)))
    a = np.pad(h, ((r, r), (0, 0)), mode="edge")
    v = sum(k[i] * a[i:i + img.shape[0], :] for i in range(len(k)))
    return v


def _shift(img: np.ndarray, dy: int, dx: int) -> np.ndarray:
    h, w = img.shape
    ys = np.clip(np.arange(h) - dy, 0, h - 1)
    xs = np.clip(np.arange(w) - dx, 0, w - 1)
    return img[ys][:, xs]


@dataclass
class _Obj:
    h: int
    w: int
    y: float
    x: float
    vy: int
    vx: int
    tex: list  # per plane textures


def make_clip(width: int, height: int, frames: int, seed: int, motion: int = 8, objects: int = 4,
              object_motion: int = 16, noise: float = 2.0) -> np.ndarray:
    """Returns uint8 [frames, w*h + 2*(w/2*h/2)] packed I420 frames."""
    assert width % 2 == 0 and height % 2 == 0
    rng = np.random.default_rng(seed)
    cw, ch = width // 2, height // 2
    dims = [(height, width, 2.0), (ch, cw, 1.0), (ch, cw, 1.0)]
    clean = [_blur(rng.integers(0, 256, size=(h, w)).astype(np.float32), s) for h, w, s in dims]
    objs = []
    for _ in range(objects):
        oh = int(rng.integers(32, 97))
        ow = int(rng.integers(32, 97))
        tex = [_blur(rng.integers(0, 256, size=(oh, ow)).astype(np.float32), 2.0)]
        tex += [_blur(rng.integers(0, 256, size=(max(oh // 2, 1), max(ow // 2, 1))).astype(np.float32), 1.0)
                for _ in range(2)]
        objs.append(_Obj(oh, ow, float(rng.integers(0, max(height - oh, 1))), float(rng.integers(0, max(width - ow, 1))),
                         int(rng.integers(-object_motion, object_motion + 1)),
                         int(rng.integers(-object_motion, object_motion + 1)), tex))
    ysz, csz = width * height, cw * ch
    out = np.empty((frames, ysz + 2 * csz), dtype=np.uint8)
    for f in range(frames):
        if f > 0:
            dy = int(rng.integers(-motion, motion + 1))
            dx = int(rng.integers(-motion, motion + 1))
            clean = [_shift(clean[0], dy, dx), _shift(clean[1], dy // 2, dx // 2), _shift(clean[2], dy // 2, dx // 2)]
        planes = [p.copy() for p in clean]
        for o in objs:
            oy = int(o.y + f * o.vy) % max(height - o.h, 1)
            ox = int(o.x + f * o.vx) % max(width - o.w, 1)
            planes[0][oy:oy + o.h, ox:ox + o.w] = o.tex[0][:min(o.h, height - oy), :min(o.w, width - ox)]
            for p in (1, 2):
                t = o.tex[p]
                cy, cx = oy // 2, ox // 2
                planes[p][cy:cy + t.shape[0], cx:cx + t.shape[1]] = t[:min(t.shape[0], ch - cy), :min(t.shape[1], cw - cx)]
        for i, p in enumerate(planes):
            noisy = p + rng.normal(0.0, noise, size=p.shape).astype(np.float32)
            q = np.clip(np.rint(noisy), 0, 255).astype(np.uint8)
            if i == 0:
                out[f, :ysz] = q.reshape(-1)
            else:
                out[f, ysz + (i - 1) * csz: ysz + i * csz] = q.reshape(-1)
    return out


def make_clip_device(width: int, height: int, frames: int, seed: int, motion: int = 8, objects: int = 4,
                     object_motion: int = 16, noise: float = 2.0, device="cuda", chunk: int = 32, bits: int = 8):
    """The recipe of make_clip, run with torch on the device and vectorised over frames (for
    the large batched and served workloads, where the host generator would take minutes).
    Differences: its own random stream, and frame k's background is frame 0's shifted once
    by the accumulated global motion (edges replicated) rather than shifted frame by frame.
    Returns a uint8 tensor [frames, w*h + 2*(w/2*h/2)] on `device`; with bits=10 the textures
    span 0..1023 (uniform noise before the blur), `noise` is in 10-bit units and the tensor
    is int16 holding the uint16 samples."""
    import torch

    assert width % 2 == 0 and height % 2 == 0
    F = torch.nn.functional
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    cw, ch = width // 2, height // 2

    def blur(img, sigma):
        k = torch.from_numpy(_kernel(sigma)).to(device)
        r = k.numel() // 2
        x = F.pad(img[None, None], (r, r, 0, 0), mode="replicate")
        x = F.conv2d(x, k.view(1, 1, 1, -1))
        x = F.pad(x, (0, 0, r, r), mode="replicate")
        return F.conv2d(x, k.view(1, 1, -1, 1))[0, 0]

    top = (1 << bits) - 1

    def noise_img(h, w):
        return torch.randint(0, top + 1, (h, w), generator=g, device=device).float()

    rng = np.random.default_rng(int(seed))
    base = [blur(noise_img(height, width), 2.0), blur(noise_img(ch, cw), 1.0), blur(noise_img(ch, cw), 1.0)]
    objs = []
    for _ in range(objects):
        oh, ow = int(rng.integers(32, 97)), int(rng.integers(32, 97))
        tex = [blur(noise_img(oh, ow), 2.0), blur(noise_img(max(oh // 2, 1), max(ow // 2, 1)), 1.0),
               blur(noise_img(max(oh // 2, 1), max(ow // 2, 1)), 1.0)]
        objs.append((oh, ow, int(rng.integers(0, max(height - oh, 1))), int(rng.integers(0, max(width - ow, 1))),
                     int(rng.integers(-object_motion, object_motion + 1)),
                     int(rng.integers(-object_motion, object_motion + 1)), tex))
    steps = rng.integers(-motion, motion + 1, size=(frames, 2))
    steps[0] = 0
    cum = np.cumsum(steps, axis=0)  # accumulated (dy, dx) of every frame
    ysz, csz = width * height, cw * ch
    out = torch.empty((frames, ysz + 2 * csz), dtype=torch.uint8 if bits == 8 else torch.int16, device=device)
    dims = [(height, width, 1), (ch, cw, 2), (ch, cw, 2)]
    for f0 in range(0, frames, chunk):
        f1 = min(frames, f0 + chunk)
        n = f1 - f0
        fidx = torch.arange(n, device=device)
        for pi, (h, w, div) in enumerate(dims):
            dy = torch.from_numpy(cum[f0:f1, 0] // div).to(device)
            dx = torch.from_numpy(cum[f0:f1, 1] // div).to(device)
            ys = (torch.arange(h, device=device)[None, :] - dy[:, None]).clamp(0, h - 1)  # [n, h]
            xs = (torch.arange(w, device=device)[None, :] - dx[:, None]).clamp(0, w - 1)  # [n, w]
            planes = base[pi][ys[:, :, None], xs[:, None, :]]                               # [n, h, w]
            for oh, ow, y0, x0, vy, vx, tex in objs:
                t = tex[pi]
                th, tw = t.shape
                for k in range(n):  # per-frame rectangle paste (position wraps like make_clip's)
                    f = f0 + k
                    oy = (y0 + f * vy) % max(height - oh, 1)
                    ox = (x0 + f * vx) % max(width - ow, 1)
                    if div == 2:
                        oy, ox = oy // 2, ox // 2
                    hh, ww = min(th, h - oy), min(tw, w - ox)
                    planes[k, oy:oy + hh, ox:ox + ww] = t[:hh, :ww]
            q = (planes + noise * torch.randn(planes.shape, generator=g, device=device)).round_().clamp_(0, top)
            q = q.to(out.dtype).reshape(n, -1)
            if pi == 0:
                out[f0:f1, :ysz] = q
            else:
                out[f0:f1, ysz + (pi - 1) * csz: ysz + pi * csz] = q
    return out


def batched_mix(nclips: int = 64, seed: int = 4, min_len: int = 16, max_len: int = 240):
    """The batched workload: clips of uneven size and length. Resolution drawn per clip
    from {640x360, 1280x720, 1920x1080, 2560x1440}, length log-uniform over
    [min_len, max_len] frames, block size from {8, 16}; motion ranges of the 1080p
    configuration. Returns [(width, height, frames, block, clip seed)]."""
    rng = np.random.default_rng(seed)
    res = [(640, 360), (1280, 720), (1920, 1080), (2560, 1440)]
    out = []
    for i in range(nclips):
        w, h = res[int(rng.integers(0, len(res)))]
        n = int(round(math.exp(rng.uniform(math.log(min_len), math.log(max_len)))))
        blk = int(rng.choice([8, 16]))
        out.append((w, h, n, blk, 1000 + 7 * i + seed))
    return out


def served_stream(nclips: int, rate: float, seed: int = 5, min_len: int = 8, max_len: int = 600):
    """The served workload: Poisson arrivals at `rate` clips/s; resolution from {360p,
    720p, 1080p, 1440p, 2160p}, length log-uniform over [min_len, max_len]. Returns
    [(arrival s, width, height, frames, clip seed)]."""
    rng = np.random.default_rng(seed)
    res = [(640, 360), (1280, 720), (1920, 1080), (2560, 1440), (3840, 2160)]
    t = 0.0
    out = []
    for i in range(nclips):
        t += float(rng.exponential(1.0 / rate))
        w, h = res[int(rng.integers(0, len(res)))]
        n = int(round(math.exp(rng.uniform(math.log(min_len), math.log(max_len)))))
        out.append((t, w, h, n, 5000 + 11 * i + seed))
    return out


def analyse_opt_for_block(block: int) -> str:
    """Analyse options of the 1080p configuration with another block size (overlap = half)."""
    return "{block:{w:%d,overlap:3},main:{search:{type:3,distance:16,satd:true}}}" % block


# Workloads of the reference's benchmark configurations (shapes, motion ranges).
CONFIGS = {
    "640x360": dict(width=640, height=360, frames=32, motion=8, objects=4, object_motion=16),
    "1080p": dict(width=1920, height=1080, frames=240, motion=24, objects=8, object_motion=48),
    # 10-bit (uint16 samples 0..1023, noise sigma 8); the object motions keep the 1080p range
    "2160p10": dict(width=3840, height=2160, frames=120, motion=64, objects=8, object_motion=48, noise=8.0, bits=10),
}
# Option strings of those configurations for the reference's Super / Analyse filters.
SUPER_OPT = {"640x360": "{pel:1}", "1080p": "{pel:2}", "2160p10": "{pel:4}"}
ANALYSE_OPT = {
    "640x360": "{block:{w:16,overlap:0},main:{search:{type:2,distance:2,satd:false,coarse:{satd:false}}}}",
    "1080p": "{block:{w:16,overlap:3},main:{search:{type:3,distance:16,satd:true}}}",
    # block 8 overlap 4, exhaustive radius 8 at the finest level, hex2 above it, SATD + chroma
    "2160p10": "{block:{w:8,overlap:3},main:{search:{type:4,distance:8,satd:true,coarse:{type:2}}}}",
}
