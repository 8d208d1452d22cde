"""Seeded synthetic 10-bit frames made on the GPU (torch), for training and evaluating the tile-proposal network.

numpy takes seconds per 3840x2160 frame, so the thousands of frames the network learns from are made on the device.
The recipe is the ``c1`` workload's (es_synth), widened so the network sees the range of content it will score:

* source: the sum of 3 seeded linear or radial gradients over a random code range (its low end in 64-450, its width
  60-450 codes: CAMBI measures banding in the darker codes only), plus Gaussian grain
  (sigma uniform in 1-12 codes), rounded and clipped;
* encode: a Gaussian blur of the source (sigma uniform in 0.8-2.5), with probability 0.3 also a 7x7 box (de-grain),
  then requantised to steps of 4, 8, 16 or 32 codes on the left half (probability 0.5) or on random rectangles
  covering 30% of the picture.

Frame i draws everything from a torch generator seeded with ``seed + i``. Planes are int16 tensors of codes.
"""

from __future__ import annotations

import math


def _gauss_blur(torch, x, sigma: float):
    r = max(1, int(math.ceil(3 * sigma)))
    t = torch.arange(-r, r + 1, device=x.device, dtype=torch.float32)
    k = torch.exp(-0.5 * (t / sigma) ** 2)
    k = (k / k.sum()).view(1, 1, 1, -1)
    y = x.view(1, 1, *x.shape)
    y = torch.nn.functional.pad(y, (r, r, 0, 0), mode="replicate")
    y = torch.nn.functional.conv2d(y, k)
    y = torch.nn.functional.pad(y, (0, 0, r, r), mode="replicate")
    y = torch.nn.functional.conv2d(y, k.view(1, 1, -1, 1))
    return y.view(*x.shape)


def _box7(torch, x):
    y = torch.nn.functional.pad(x.view(1, 1, *x.shape), (3, 3, 3, 3), mode="replicate")
    return torch.nn.functional.avg_pool2d(y, 7, stride=1).view(*x.shape)


def frame_pair(torch, index: int, w: int = 3840, h: int = 2160, seed: int = 50000):
    """(source, encode): int16 CUDA tensors (h, w) of 10-bit codes, and a dict of the drawn parameters."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed + index)

    def u(lo=0.0, hi=1.0):
        return lo + (hi - lo) * float(torch.rand(1, generator=g, device="cuda").item())

    yy = torch.linspace(0, 1, h, device="cuda").view(h, 1).expand(h, w)
    xx = torch.linspace(0, 1, w, device="cuda").view(1, w).expand(h, w)
    field = torch.zeros(h, w, device="cuda")
    for _ in range(3):
        if u() < 0.5:
            a = u(0, 2 * math.pi)
            field += math.cos(a) * xx + math.sin(a) * yy
        else:
            cx, cy = u(), u()
            field += torch.sqrt((xx - cx) ** 2 + (yy - cy) ** 2)
    field -= field.min()
    field /= field.max().clamp_min(1e-6)
    lo = u(64, 450)
    hi = u(lo + 60, min(940.0, lo + 450))
    sigma = u(1, 12)
    noise = torch.randn(h, w, generator=g, device="cuda")
    src = torch.clamp(torch.round(lo + (hi - lo) * field + sigma * noise), 64, 940)
    blur = u(0.8, 2.5)
    enc = _gauss_blur(torch, src, blur)
    degrain = u() < 0.3
    if degrain:
        enc = _box7(torch, enc)
    step = [4, 8, 16, 32][int(u() * 4) % 4]
    region = torch.zeros(h, w, dtype=torch.bool, device="cuda")
    left = u() < 0.5
    if left:
        region[:, : w // 2] = True
    else:
        while region.float().mean().item() < 0.30:
            rw, rh = int(u(0.1, 0.35) * w), int(u(0.1, 0.35) * h)
            x0, y0 = int(u(0, w - rw)), int(u(0, h - rh))
            region[y0:y0 + rh, x0:x0 + rw] = True
    enc = torch.where(region, torch.round(enc / step) * step, torch.round(enc))
    enc = torch.clamp(enc, 64, 940)
    params = {"lo": lo, "hi": hi, "grain": sigma, "blur": blur, "degrain": degrain, "step": step, "left_half": left}
    return src.to(torch.int16), enc.to(torch.int16), params


def c4_pair(torch, index: int, w: int = 3840, h: int = 2160, seed: int = 4000):
    """The precision workload: a bright 10-bit gradient (codes 600-940, 3 seeded linear or radial gradients) with heavy
    Gaussian grain (sigma 20 codes), clipped to 0-1023; the encode blurs it (sigma 1.0). int16 CUDA tensors."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed + index)

    def u(lo=0.0, hi=1.0):
        return lo + (hi - lo) * float(torch.rand(1, generator=g, device="cuda").item())

    yy = torch.linspace(0, 1, h, device="cuda").view(h, 1).expand(h, w)
    xx = torch.linspace(0, 1, w, device="cuda").view(1, w).expand(h, w)
    field = torch.zeros(h, w, device="cuda")
    for _ in range(3):
        if u() < 0.5:
            a = u(0, 2 * math.pi)
            field += math.cos(a) * xx + math.sin(a) * yy
        else:
            cx, cy = u(), u()
            field += torch.sqrt((xx - cx) ** 2 + (yy - cy) ** 2)
    field -= field.min()
    field /= field.max().clamp_min(1e-6)
    noise = torch.randn(h, w, generator=g, device="cuda")
    src = torch.clamp(torch.round(600 + 340 * field + 20 * noise), 0, 1023)
    enc = torch.clamp(torch.round(_gauss_blur(torch, src, 1.0)), 0, 1023)
    return src.to(torch.int16), enc.to(torch.int16)
