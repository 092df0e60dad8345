"""CPU oracle of the learned proposal network (test infrastructure only).

The reference has no learned component, so this oracle states the network's
mathematics directly and is the checker for the GPU kernels of
gpu_tracking_b200/csrc/gt_cnn.cu (forward convolutions, loss, input and
weight gradients).  It rounds to BF16 where the GPU stores BF16 (inputs,
weights, hidden activations, gradients between layers) and accumulates in
float64; the GPU accumulates in FP32 in the tensor cores' order, so the two
agree to a tolerance, not bit for bit.

Network: input cells of 4x4 pixels as 16 channels, x = bf16((p - mean) * scale);
a_l = bf16(relu(conv3x3(a_{l-1}, W_l) + b_l)) for l = 1..3 (32 channels);
out = conv3x3(a_3, W_4) + b_4 (score logit, row offset, column offset).
Parameters: per layer W[co][ci][ky*3 + kx] then b[co], fp32.
"""
import numpy as np

CIN = (16, 32, 32, 32)
COUT = (32, 32, 32, 3)


def num_params():
    return sum(co * ci * 9 + co for ci, co in zip(CIN, COUT))


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)


def split(params):
    """[(W (co, ci, 9) float32, b (co,) float32)] per layer."""
    out, o = [], 0
    for ci, co in zip(CIN, COUT):
        w = np.asarray(params[o:o + co * ci * 9], np.float32).reshape(co, ci, 9)
        o += co * ci * 9
        b = np.asarray(params[o:o + co], np.float32)
        o += co
        out.append((w, b))
    return out


def cells(frames, mean, scale, crops=None, crop=None):
    """Space-to-depth input (n, Hc, Wc, 16) float32 (BF16 values).

    Without crops every frame is one image of ceil(H/4) x ceil(W/4) cells;
    pixels beyond the frame read as the mean.  A crop (frame, row, column)
    takes crop x crop pixels from that offset."""
    frames = np.asarray(frames)
    T, H, W = frames.shape
    if crops is None:
        imgs = [(t, 0, 0) for t in range(T)]
        ch, cw = (H + 3) // 4, (W + 3) // 4
    else:
        imgs = [tuple(int(v) for v in c) for c in crops]
        ch = cw = crop // 4
    out = np.zeros((len(imgs), ch, cw, 16), np.float32)
    m, s = np.float32(mean), np.float32(scale)
    for i, (f, oy, ox) in enumerate(imgs):
        pad = np.full((4 * ch, 4 * cw), m, np.float32)
        blk = frames[f, oy:oy + 4 * ch, ox:ox + 4 * cw].astype(np.float32)
        pad[:blk.shape[0], :blk.shape[1]] = blk
        v = (pad - m) * s
        out[i] = v.reshape(ch, 4, cw, 4).transpose(0, 2, 1, 3).reshape(ch, cw, 16)
    return bf16(out)


def conv(x, w):
    """'same' 3x3 convolution, x (n, H, W, ci), w (co, ci, 9), float64 sums."""
    n, H, W, _ = x.shape
    xp = np.zeros((n, H + 2, W + 2, x.shape[3]), np.float64)
    xp[:, 1:-1, 1:-1] = x
    out = np.zeros((n, H, W, w.shape[0]), np.float64)
    for t in range(9):
        dy, dx = divmod(t, 3)
        out += xp[:, dy:dy + H, dx:dx + W, :] @ w[:, :, t].astype(np.float64).T
    return out


def _identity(a):
    return np.asarray(a, np.float64)


def forward(params, x, exact=False):
    """Activations [x, a1, a2, a3] and the head (n, H, W, 3).

    exact=True keeps float64 throughout without BF16 rounding (the smooth
    function whose derivative loss_grad(exact=True) returns)."""
    rnd, dt = (_identity, np.float64) if exact else (bf16, np.float32)
    layers = split(params)
    acts = [x]
    a = x
    for l in range(3):
        w, b = layers[l]
        z = conv(a, rnd(w)).astype(dt) + b.astype(dt)
        a = rnd(np.maximum(z, 0.0))
        acts.append(a)
    w, b = layers[3]
    head = conv(a, rnd(w)).astype(dt) + b.astype(dt)
    return acts, head


def targets(label_frame, label_y, label_x, T, Hc, Wc):
    """(T, Hc, Wc, 3): flag, row and column offset from the cell centre; the
    lowest-index label in a cell owns it."""
    t = np.zeros((T, Hc, Wc, 3), np.float32)
    for i in range(len(label_frame)):
        f = int(label_frame[i])
        y, x = np.float32(label_y[i]), np.float32(label_x[i])
        if f < 0 or f >= T or not (y >= 0) or not (x >= 0):
            continue
        cy, cx = int(np.floor(y * np.float32(0.25))), int(np.floor(x * np.float32(0.25)))
        if cy >= Hc or cx >= Wc or t[f, cy, cx, 0] == 1.0:
            continue
        t[f, cy, cx] = (1.0, y - (np.float32(4.0) * cy + np.float32(1.5)), x - (np.float32(4.0) * cx + np.float32(1.5)))
    return t


def wgrad(X, G):
    """dW[co, ci, t] = sum over cells G[cell, co] * X[cell + tap t, ci]; db."""
    n, H, W, ci = X.shape
    xp = np.zeros((n, H + 2, W + 2, ci), np.float64)
    xp[:, 1:-1, 1:-1] = X
    g = G.reshape(-1, G.shape[3]).astype(np.float64)
    dw = np.zeros((G.shape[3], ci, 9))
    for t in range(9):
        dy, dx = divmod(t, 3)
        dw[:, :, t] = g.T @ xp[:, dy:dy + H, dx:dx + W, :].reshape(-1, ci)
    return dw, g.sum(axis=0)


def dgrad(G, w, rnd=bf16):
    """Input gradient of a 'same' 3x3 convolution with weights w (co, ci, 9)."""
    wt = np.transpose(rnd(w), (1, 0, 2))[:, :, ::-1]
    return conv(G, wt)


def loss_grad(params, x, tgt, pos_weight, lam, exact=False):
    """Score and offset losses (means over cells) and the gradient of their sum."""
    rnd, dt = (_identity, np.float64) if exact else (bf16, np.float32)
    acts, head = forward(params, x, exact)
    s, oy, ox = head[..., 0].astype(np.float64), head[..., 1].astype(np.float64), head[..., 2].astype(np.float64)
    y, ty, tx = tgt[..., 0].astype(np.float64), tgt[..., 1].astype(np.float64), tgt[..., 2].astype(np.float64)
    ncell = s.size
    sp_pos = np.maximum(-s, 0) + np.log1p(np.exp(-np.abs(s)))
    sp_neg = np.maximum(s, 0) + np.log1p(np.exp(-np.abs(s)))
    sig = 1.0 / (1.0 + np.exp(-s))
    ls = (pos_weight * y * sp_pos + (1 - y) * sp_neg).sum() / ncell
    lo = (lam * y * ((oy - ty) ** 2 + (ox - tx) ** 2)).sum() / ncell
    gout = np.zeros(head.shape[:3] + (3,), np.float64)
    gout[..., 0] = (pos_weight * y * (sig - 1) + (1 - y) * sig) / ncell
    gout[..., 1] = 2 * lam * y * (oy - ty) / ncell
    gout[..., 2] = 2 * lam * y * (ox - tx) / ncell
    g = rnd(gout.astype(dt))
    layers = split(params)
    grads = [None] * 4
    for l in (3, 2, 1, 0):
        dw, db = wgrad(acts[l], g)
        grads[l] = (dw, db)
        if l > 0:
            g = rnd((dgrad(g, layers[l][0], rnd) * (acts[l] > 0)).astype(dt))
    flat = np.concatenate([np.concatenate([dw.ravel(), db]) for dw, db in grads])
    return (ls, lo), flat.astype(dt)
