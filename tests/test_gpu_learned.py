"""The learned proposal network on the GPU against its CPU oracle, and the
learned seeds against the plain method.

* forward: the tcgen05 convolutions give the oracle's outputs (BF16
  operands, FP32 accumulation; relative tolerance 1e-4 for the accumulation
  order);
* gradients: loss and every parameter gradient of one batch against the
  oracle's backward pass;
* training: the network trained by the engine's own kernels on the plain
  method's detections finds them again from far fewer walk starts, and every
  learned detection whose walk ends where the plain one does is identical to
  it in every column (the seed-patch bandpass reproduces the full-frame one
  bit for bit).
"""
import ctypes

import numpy as np
import pytest

import gpu_tracking_b200 as gt
from gpu_tracking_b200 import _ffi
from gpu_tracking_b200 import learned
from oracle import cnn_oracle as co
from synth import video

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12))


def random_net(seed):
    net = learned.ProposalNet(seed=seed)
    rng = np.random.default_rng(seed)
    p = np.zeros(co.num_params(), np.float32)
    o = 0
    for ci, cout in zip(co.CIN, co.COUT):
        n = cout * ci * 9
        p[o:o + n] = rng.normal(0, np.sqrt(2.0 / (9 * ci)), n)
        o += n
        p[o:o + cout] = rng.normal(0, 0.1, cout)
        o += cout
    net.params = p
    return net, p


@pytest.mark.parametrize("dtype,shape", [(np.uint16, (96, 128)), (np.uint16, (100, 100)), (np.float32, (64, 200)),
                                         (np.uint8, (40, 36))])
def test_forward_matches_oracle(dtype, shape):
    frames, _ = video(2, shape[0], shape[1], 20, seed=shape[1], dtype=np.uint16)
    if dtype == np.float32:
        frames = frames.astype(np.float32) * 0.5
    elif dtype == np.uint8:
        frames = np.clip(frames // 8, 0, 255).astype(np.uint8)
    net, p = random_net(7)
    mean, scale = float(frames.mean()), 1.0 / float(frames.std())
    net.set_normalization(mean, scale)
    got = net.maps(frames)
    x = co.cells(frames, mean, scale)
    _, head = co.forward(p, x)
    assert got.shape == head.shape[:3] + (4,)
    # the oracle rounds at the GPU's BF16 points; what remains is the FP32
    # accumulation order (observed relative errors 1e-7 .. 2e-5)
    for ch in range(3):
        assert rel_err(got[..., ch], head[..., ch]) < 1e-4, ch
    assert np.all(got[..., 3] == 0)


def test_gradients_match_oracle():
    frames, _ = video(3, 96, 160, 30, seed=11)
    plain = gt.batch(frames, 9, minmass=300.0, tqdm=False)
    net, p = random_net(3)
    mean, scale = float(frames.mean()), 1.0 / float(frames.std())
    net.set_normalization(mean, scale)
    crops = np.array([[0, 0, 0], [1, 32, 64], [2, 28, 96], [0, 32, 92], [1, 0, 12]], np.int32)
    crop = 64
    lf = plain["frame"].to_numpy(np.int64)
    ly = plain["y"].to_numpy(np.float32)
    lx = plain["x"].to_numpy(np.float32)
    grad = np.zeros(co.num_params(), np.float32)
    loss = np.zeros(2, np.float32)
    ctx = _ffi.context(0)
    P32, P64, P32i = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
    fr = np.ascontiguousarray(frames)
    ctx.check(_ffi.lib().gt__proposal_loss_grad(ctx.handle, net.handle, ctypes.c_void_p(fr.ctypes.data), 0,
                                                fr.shape[0], fr.shape[1], fr.shape[2], lf.ctypes.data_as(P64),
                                                ly.ctypes.data_as(P32), lx.ctypes.data_as(P32), len(lf),
                                                crops.ctypes.data_as(P32i), len(crops), crop, 8.0, 1.0,
                                                grad.ctypes.data_as(P32), loss.ctypes.data_as(P32)))
    x = co.cells(frames, mean, scale, crops=crops, crop=crop)
    T, H, W = frames.shape
    tmap = co.targets(lf, ly, lx, T, H // 4, W // 4)
    tgt = np.stack([tmap[f, y // 4:y // 4 + crop // 4, xx // 4:xx // 4 + crop // 4] for f, y, xx in crops])
    assert tgt[..., 0].sum() >= 5
    (ls, lo), g = co.loss_grad(p, x, tgt, 8.0, 1.0)
    assert abs(loss[0] - ls) <= 2e-3 * abs(ls) + 1e-6
    assert abs(loss[1] - lo) <= 2e-2 * abs(lo) + 1e-5
    o = 0
    for l, (ci, cout) in enumerate(zip(co.CIN, co.COUT)):
        n = cout * ci * 9
        assert rel_err(grad[o:o + n], g[o:o + n]) < 3e-2, ("W", l)
        o += n
        assert rel_err(grad[o:o + cout], g[o:o + cout]) < 3e-2, ("b", l)
        o += cout


def test_trained_seeds_recover_plain_detections():
    kw = dict(minmass=300.0, separation=10)
    # every frame draws new spot positions: many independent examples
    train, _ = video(24, 256, 256, 150, seed=21, turnover=1.0)
    plain_train = gt.batch(train, 9, tqdm=False, **kw)
    net = learned.ProposalNet(seed=5)
    loss = net.train(train, plain_train, steps=800, batch=64, crop=64, lr=3e-3)
    assert np.isfinite(loss).all()
    assert loss[-40:, 0].mean() < 0.5 * loss[:40, 0].mean()
    thr, curve = learned.calibrate(net, train[:6], 9, recall=0.99, **kw)
    assert curve and thr == net.threshold

    test, _ = video(4, 256, 256, 150, seed=22, turnover=1.0)
    plain = gt.batch(test, 9, tqdm=False, **kw)
    plain_starts = learned.last_walk_starts()
    got = learned.batch_learned(test, 9, net, tqdm=False, **kw)
    seeds = learned.last_walk_starts()
    s = learned.compare(plain, got)
    assert s["recall"] >= 0.975, s
    assert s["precision"] >= 0.95, s
    # a walk that ends where the plain one does gives the plain row exactly
    assert s["identical"] == s["same_position"], s
    assert s["same_position"] >= 0.97 * s["matched"], s
    assert s["mean_position_error"] <= 0.01, s
    # what the network gains: far fewer walks than bandpass local maxima
    assert seeds < 0.7 * plain_starts, (seeds, plain_starts)
    # and an untrained network at the same threshold finds almost nothing
    raw = learned.ProposalNet(seed=5)
    raw.set_normalization(net.mean, net.scale)
    raw.threshold = net.threshold
    s0 = learned.compare(plain, learned.batch_learned(test, 9, raw, tqdm=False, **kw))
    assert s0["recall"] < 0.5 * s["recall"], s0


def test_learned_rejects_unsupported_options():
    frames, _ = video(1, 64, 64, 5, seed=3)
    net = learned.ProposalNet(seed=1)
    with pytest.raises(ValueError):
        learned.batch_learned(frames, 9, net, snr=0.5, tqdm=False)
    with pytest.raises(ValueError):
        learned.batch_learned(frames.astype(np.float32), 9, net, illumination_sigma=4.0, tqdm=False)
