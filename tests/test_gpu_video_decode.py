"""Video files decoded on the GPU (gt_video_read_device) against the host
decoder (gt_video_read), sample for sample: TIFF stacks in every layout the
decoder supports (uncompressed, PackBits, LZW with dictionary resets,
Deflate inflated on the host; strips and tiles; horizontal differencing;
both byte orders; BigTIFF; u8, u16, i16 and f32 samples), Olympus .ets
frames, frame subsets, and batch() on a path decoded on the device.
"""
import numpy as np
import pandas as pd
import pytest
from PIL import Image

import gpu_tracking_b200 as gt
from gpu_tracking_b200 import api
from test_video_files import frames_u16, write_ets, write_tiff

pytestmark = pytest.mark.gpu


def same_on_device(p, **kw):
    host = api._read_video(p, **kw)
    dev = api._read_video(p, device=True, **kw)
    got = dev.cpu().numpy()
    assert got.dtype == host.dtype and got.shape == host.shape
    if host.dtype == np.float32:
        assert np.array_equal(got.view(np.uint32), host.view(np.uint32))
    else:
        assert np.array_equal(got, host)
    return host


@pytest.mark.parametrize("comp", ["raw", "packbits", "tiff_lzw", "tiff_adobe_deflate"])
def test_pillow_stacks(tmp_path, comp):
    rng = np.random.default_rng(11)
    # noise (LZW dictionary resets), a smooth ramp (long LZW strings, PackBits runs)
    noise = rng.integers(0, 65535, size=(3, 61, 173), dtype=np.uint16)
    ramp = np.broadcast_to((np.arange(173) * 7 % 4096).astype(np.uint16), (3, 61, 173)).copy()
    for name, f in (("noise", noise), ("ramp", ramp)):
        p = str(tmp_path / (name + ".tif"))
        imgs = [Image.fromarray(x) for x in f]
        imgs[0].save(p, save_all=True, append_images=imgs[1:], compression=comp)
        host = same_on_device(p)
        assert np.array_equal(host, f)
        same_on_device(p, frames=[2, 0])
        same_on_device(p, as_float=True)


def test_large_lzw_frames(tmp_path):
    """512 x 700 u16 frames in Pillow's LZW strips: many strips per frame,
    several batches of blocks would not be needed, but every strip runs the
    dictionary through its 12-bit limit."""
    rng = np.random.default_rng(12)
    f = (rng.normal(1000, 300, size=(4, 512, 700)).clip(0, 65535)).astype(np.uint16)
    p = str(tmp_path / "big.tif")
    imgs = [Image.fromarray(x) for x in f]
    imgs[0].save(p, save_all=True, append_images=imgs[1:], compression="tiff_lzw")
    assert np.array_equal(same_on_device(p), f)


@pytest.mark.parametrize("mode,dtype,comp", [("L", np.uint8, "tiff_lzw"), ("L", np.uint8, "packbits"),
                                             ("F", np.float32, "raw")])
def test_pillow_u8_and_f32(tmp_path, mode, dtype, comp):
    rng = np.random.default_rng(13)
    f = (rng.integers(0, 255, size=(2, 40, 57)).astype(dtype) if dtype == np.uint8
         else rng.normal(100, 20, size=(2, 40, 57)).astype(np.float32))
    p = str(tmp_path / "v.tif")
    imgs = [Image.fromarray(x, mode=mode) for x in f]
    imgs[0].save(p, save_all=True, append_images=imgs[1:], compression=comp)
    assert np.array_equal(same_on_device(p), f)


@pytest.mark.parametrize("kw", [
    dict(),
    dict(big_endian=True),
    dict(tile=(16, 16)),
    dict(tile=(16, 32), deflate=True, predictor=True, big_endian=True),
    dict(deflate=True, predictor=True),
    dict(predictor=True),
    dict(predictor=True, big_endian=True, tile=(16, 16)),
    dict(bigtiff=True),
    dict(bigtiff=True, tile=(16, 16), deflate=True),
])
def test_written_layouts(tmp_path, kw):
    f = frames_u16(3, T=2, H=45, W=50)
    p = str(tmp_path / "w.tif")
    write_tiff(p, f, **kw)
    assert np.array_equal(same_on_device(p), f)


def test_signed_16bit_and_ets(tmp_path):
    s = np.random.default_rng(4).integers(-30000, 30000, size=(2, 9, 11)).astype(np.int16)
    p = str(tmp_path / "s.tif")
    write_tiff(p, s, sample_format=2)
    assert np.array_equal(same_on_device(p), s.astype(np.float32))
    a, b = frames_u16(5, T=3, H=12, W=17), frames_u16(6, T=2, H=12, W=17)
    ets = str(tmp_path / "frame_t_0.ets")
    write_ets(ets, {0: a, 1: b})
    assert np.array_equal(same_on_device(ets), a)
    assert np.array_equal(same_on_device(ets, channel=1, frames=[1]), b[[1]])


def test_corrupt_lzw_strip_is_an_error(tmp_path):
    """A strip whose codes run past the dictionary: the device decoder stops
    at the bad code (no read or write leaves the strip's buffers) and the
    call raises, as the host decoder does."""
    f = np.random.default_rng(14).integers(0, 65535, size=(1, 20, 30), dtype=np.uint16)
    p = tmp_path / "c.tif"
    Image.fromarray(f[0]).save(str(p), compression="tiff_lzw")
    with Image.open(str(p)) as im:
        off = int(im.tag_v2[273][0])
    data = bytearray(p.read_bytes())
    # all-ones bits after the first codes: a 9-bit code of 511 while the
    # dictionary holds far fewer entries
    for k in range(off + 4, off + 16):
        data[k] = 0xFF
    p.write_bytes(bytes(data))
    with pytest.raises(Exception):
        api._read_video(str(p))
    with pytest.raises(Exception):
        api._read_video(str(p), device=True)


def test_batch_on_a_path_decodes_on_the_device(tmp_path):
    from synth import video
    frames, _ = video(5, 96, 128, 30, seed=92)
    p = str(tmp_path / "stack.tif")
    imgs = [Image.fromarray(x) for x in frames]
    imgs[0].save(p, save_all=True, append_images=imgs[1:], compression="tiff_lzw")
    fr = api._Frames(p)
    assert hasattr(fr.keep, "is_cuda") and fr.keep.is_cuda
    kw = dict(minmass=300.0, search_range=5.0, tqdm=False)
    pd.testing.assert_frame_equal(gt.batch(p, 9, **kw), gt.batch(frames, 9, **kw))
    pd.testing.assert_frame_equal(gt.batch(p, 9, frames=[1, 3, 4], **kw), gt.batch(frames, 9, frames=[1, 3, 4], **kw))
