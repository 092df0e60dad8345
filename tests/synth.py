"""Seeded synthetic videos for the CPU tests (numpy).

Background + Poisson noise with Gaussian spots that move by Brownian motion,
the distributions of the workloads the benchmark names (spots of width
sigma, lognormal amplitudes, diffusion D px^2/frame, births/deaths).
"""
import numpy as np


def video(T, H, W, n_spots, seed, sigma=1.5, amp_mu=np.log(800.0), amp_s=0.5, D=0.5, bg=100.0,
          turnover=0.0, dtype=np.uint16, read_noise=None, sigma_range=None, margin=3.0):
    rng = np.random.default_rng(seed)
    pos = rng.uniform([margin, margin], [H - margin, W - margin], size=(n_spots, 2))
    if sigma_range is not None:
        sig = rng.uniform(sigma_range[0], sigma_range[1], n_spots)
    else:
        sig = np.full(n_spots, sigma)
    amp = rng.lognormal(amp_mu, amp_s, n_spots)
    yy, xx = np.mgrid[0:H, 0:W]
    frames = np.empty((T, H, W), dtype=dtype)
    truth = []
    for t in range(T):
        img = np.full((H, W), bg, np.float64)
        for k in range(n_spots):
            y, x = pos[k]
            r = int(4 * sig[k]) + 1
            y0, y1 = max(0, int(y) - r), min(H, int(y) + r + 2)
            x0, x1 = max(0, int(x) - r), min(W, int(x) + r + 2)
            g = np.exp(-((yy[y0:y1, x0:x1] - y) ** 2 + (xx[y0:y1, x0:x1] - x) ** 2) / (2 * sig[k] ** 2))
            img[y0:y1, x0:x1] += amp[k] * g
        truth.append(pos.copy())
        if read_noise is not None:
            val = img + rng.normal(0.0, read_noise, img.shape)
        else:
            val = rng.poisson(img).astype(np.float64)
        if np.issubdtype(dtype, np.integer):
            info = np.iinfo(dtype)
            frames[t] = np.clip(np.rint(val), info.min, info.max).astype(dtype)
        else:
            frames[t] = val.astype(dtype)
        pos = pos + rng.normal(0.0, np.sqrt(2 * D), pos.shape)
        if turnover > 0:
            dead = rng.random(n_spots) < turnover
            pos[dead] = rng.uniform([margin, margin], [H - margin, W - margin], size=(dead.sum(), 2))
        pos = np.clip(pos, margin, [H - margin, W - margin])
    return frames, truth
