"""Seeded synthetic videos generated on the GPU (torch), for benchmarks and tests.

Gaussian spots on a flat background that diffuse by Brownian motion; a
fraction of spots is replaced by new ones every frame (births/deaths).  Spot
widths and peak signal-to-noise ratios are drawn per spot.  Noise is Poisson
shot noise (uint16 videos) or Gaussian read noise (float32 videos).  The
same seed gives the same bytes on every B200.
"""
import math

import torch


def _render(T, H, W, n_spots, g, dev, sigma_range, amp_fn, D, turnover, margin, chunk):
    """Yield (t0, float32 (nf, H*W) noiseless spot images) chunk by chunk."""

    def draw(n):
        p = torch.rand((n, 2), generator=g, device=dev)
        p[:, 0] = margin + p[:, 0] * (H - 2 * margin)
        p[:, 1] = margin + p[:, 1] * (W - 2 * margin)
        sig = sigma_range[0] + torch.rand(n, generator=g, device=dev) * (sigma_range[1] - sigma_range[0])
        return p, sig, amp_fn(n)

    pos, sig, amp = draw(n_spots)
    rad = int(math.ceil(4 * sigma_range[1]))
    off = torch.arange(-rad, rad + 1, device=dev, dtype=torch.float32)
    oy, ox = torch.meshgrid(off, off, indexing="ij")
    oy, ox = oy.reshape(-1), ox.reshape(-1)
    step = math.sqrt(2.0 * D)
    for t0 in range(0, T, chunk):
        nf = min(chunk, T - t0)
        img = torch.zeros((nf, H * W), device=dev)
        for k in range(nf):
            cy = torch.floor(pos[:, 0])[:, None] + oy[None, :]
            cx = torch.floor(pos[:, 1])[:, None] + ox[None, :]
            d2 = (cy - pos[:, 0:1]) ** 2 + (cx - pos[:, 1:2]) ** 2
            val = amp[:, None] * torch.exp(-d2 / (2.0 * sig[:, None] ** 2))
            ok = (cy >= 0) & (cy < H) & (cx >= 0) & (cx < W)
            idx = (cy.long() * W + cx.long())[ok]
            img[k].index_add_(0, idx, val[ok])
            pos = pos + step * torch.randn(pos.shape, generator=g, device=dev)
            dead = torch.rand(n_spots, generator=g, device=dev) < turnover
            nd = int(dead.sum())
            if nd:
                p2, s2, a2 = draw(nd)
                pos[dead], sig[dead], amp[dead] = p2, s2, a2
            pos[:, 0].clamp_(margin, H - margin)
            pos[:, 1].clamp_(margin, W - margin)
        yield t0, img


def _lognormal_snr(g, dev, snr_range):
    lo, hi = snr_range
    mu = 0.5 * (math.log(lo) + math.log(hi))
    s = (math.log(hi) - math.log(lo)) / 4.0

    def f(n):
        return torch.exp(mu + s * torch.randn(n, generator=g, device=dev)).clamp(lo, hi)

    return f


def brownian_video(T, H, W, n_spots, seed=0, device="cuda", sigma_range=(1.2, 2.5), snr_range=(3.0, 20.0),
                   bg=100.0, D=1.0, turnover=0.02, margin=4.0, chunk=16):
    """uint16 (T, H, W) video: peak amplitude = SNR * sqrt(bg) with SNR
    log-normal clipped to snr_range (median at its geometric mean), sigma
    uniform in sigma_range, Poisson noise on bg + signal, per-axis Brownian
    step N(0, 2D) per frame, a fraction `turnover` of spots respawned per frame."""
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))
    snr = _lognormal_snr(g, dev, snr_range)
    out = torch.empty((T, H, W), dtype=torch.uint16, device=dev)
    for t0, img in _render(T, H, W, n_spots, g, dev, sigma_range, lambda n: snr(n) * math.sqrt(bg), D, turnover,
                           margin, chunk):
        nf = img.shape[0]
        noisy = torch.poisson(img + float(bg), generator=g).clamp_(0, 65535)
        out[t0:t0 + nf] = noisy.to(torch.int32).to(torch.uint16).view(nf, H, W)
    return out


def blob_video(T, H, W, n_spots, seed=0, device="cuda", radius_range=(2.0, 8.0), read_noise=5.0, bg=50.0,
               snr_range=(3.0, 20.0), D=1.0, turnover=0.02, chunk=8):
    """float32 (T, H, W) LoG workload: blobs of radius r uniform in
    radius_range drawn as Gaussians of sigma r / sqrt(2), peak = SNR *
    read_noise, Gaussian read noise of sigma read_noise around bg."""
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))
    snr = _lognormal_snr(g, dev, snr_range)
    sr = (radius_range[0] / math.sqrt(2.0), radius_range[1] / math.sqrt(2.0))
    out = torch.empty((T, H, W), dtype=torch.float32, device=dev)
    for t0, img in _render(T, H, W, n_spots, g, dev, sr, lambda n: snr(n) * read_noise, D, turnover,
                           max(4.0, radius_range[1]), chunk):
        nf = img.shape[0]
        noise = torch.randn(img.shape, generator=g, device=dev)
        out[t0:t0 + nf] = (img + bg + read_noise * noise).view(nf, H, W)
    return out
