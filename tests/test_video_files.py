"""Video files through the engine's frame providers (host-side decoding, no
GPU): TIFF stacks in every layout the decoder supports and Olympus .ets /
.vsi chunk tables (src/decoderiter.rs:273-481, src/execute_gpu.rs:1186-1270),
against the arrays that were written.  Pillow writes the compressed TIFFs; a
small writer below makes the layouts Pillow does not (tiles, horizontal
differencing, big endian, BigTIFF) and the .ets files.
"""
import os
import struct
import zlib

import numpy as np
import pytest
from PIL import Image

import gpu_tracking_b200 as gt
from gpu_tracking_b200 import api


def frames_u16(seed, T=3, H=37, W=53):
    return np.random.default_rng(seed).integers(0, 65535, size=(T, H, W), dtype=np.uint16)


@pytest.mark.parametrize("comp", ["raw", "packbits", "tiff_lzw", "tiff_adobe_deflate"])
def test_pillow_tiff_u16_stack(tmp_path, comp):
    f = frames_u16(1)
    p = str(tmp_path / "v.tif")
    imgs = [Image.fromarray(x) for x in f]
    imgs[0].save(p, save_all=True, append_images=imgs[1:], compression=comp)
    got = gt.load(p)
    assert got.dtype == np.float32 and np.array_equal(got, f.astype(np.float32))
    native = api._read_video(p)
    assert native.dtype == np.uint16 and np.array_equal(native, f)
    assert np.array_equal(gt.load(p, frames=[2, 0]), f[[2, 0]].astype(np.float32))


@pytest.mark.parametrize("mode,dtype", [("L", np.uint8), ("F", np.float32)])
def test_pillow_tiff_u8_and_f32(tmp_path, mode, dtype):
    rng = np.random.default_rng(2)
    f = (rng.integers(0, 255, size=(2, 20, 31)).astype(dtype) if dtype == np.uint8
         else rng.normal(100, 20, size=(2, 20, 31)).astype(np.float32))
    p = str(tmp_path / "v.tiff")
    imgs = [Image.fromarray(x, mode=mode) for x in f]
    imgs[0].save(p, save_all=True, append_images=imgs[1:], compression="tiff_lzw" if dtype == np.uint8 else "raw")
    assert np.array_equal(gt.load(p), f.astype(np.float32))
    assert api._read_video(p).dtype == (np.uint8 if dtype == np.uint8 else np.float32)


def write_tiff(path, frames, big_endian=False, bigtiff=False, tile=None, deflate=False, predictor=False,
               sample_format=1):
    """Minimal TIFF writer: one sample per pixel, strips (one per image) or
    tiles, optional Deflate with horizontal differencing."""
    e = ">" if big_endian else "<"
    T, H, W = frames.shape
    bps = frames.dtype.itemsize * 8
    data_blocks = []
    for img in frames:
        if tile:
            th, tw = tile
            blocks = []
            for by in range(0, H, th):
                for bx in range(0, W, tw):
                    b = np.zeros((th, tw), frames.dtype)
                    part = img[by:by + th, bx:bx + tw]
                    b[:part.shape[0], :part.shape[1]] = part
                    blocks.append(b)
        else:
            blocks = [img]
        enc = []
        for b in blocks:
            b = np.ascontiguousarray(b)
            if predictor:
                d = b.copy()
                d[:, 1:] = b[:, 1:] - b[:, :-1]
                b = d
            raw = b.astype(b.dtype.newbyteorder(e)).tobytes()
            enc.append(zlib.compress(raw) if deflate else raw)
        data_blocks.append(enc)
    out = bytearray()
    hdr_len = 16 if bigtiff else 8
    out += b"\0" * hdr_len
    offs = []
    for enc in data_blocks:
        o = []
        for chunk in enc:
            o.append(len(out))
            out += chunk
        offs.append(o)
    cnt_fmt, nxt_fmt = ("Q", "Q") if bigtiff else ("H", "I")
    ifd_pos = []
    for i in range(T):
        o = offs[i]
        cnts = [len(c) for c in data_blocks[i]]
        # arrays of offsets and counts stored out of line (LONG8 / LONG)
        arr_t = 16 if bigtiff else 4
        arr_fmt = "Q" if bigtiff else "I"
        off_arr = len(out)
        out += struct.pack(e + arr_fmt * len(o), *o)
        cnt_arr = len(out)
        out += struct.pack(e + arr_fmt * len(cnts), *cnts)
        tags = [(256, 4, 1, W), (257, 4, 1, H), (258, 3, 1, bps), (259, 3, 1, 8 if deflate else 1),
                (262, 3, 1, 1), (277, 3, 1, 1), (339, 3, 1, sample_format)]
        if predictor:
            tags.append((317, 3, 1, 2))
        if tile:
            tags += [(322, 4, 1, tile[1]), (323, 4, 1, tile[0])]
            tags += [(324, arr_t, len(o), off_arr if len(o) > 1 or not bigtiff else o[0]),
                     (325, arr_t, len(o), cnt_arr if len(o) > 1 or not bigtiff else cnts[0])]
        else:
            tags += [(273, arr_t, 1, o[0]), (278, 4, 1, H), (279, arr_t, 1, cnts[0])]
        tags.sort()
        pos = len(out)
        ifd_pos.append(pos)
        out += struct.pack(e + cnt_fmt, len(tags))
        field = 8 if bigtiff else 4
        for tag, typ, count, val in tags:
            # a single value sits in the entry; arrays are given by offset
            if count > 1:
                vb = struct.pack(e + ("Q" if bigtiff else "I"), val)
            else:
                vb = struct.pack(e + {3: "H", 4: "I", 16: "Q"}[typ], val)
            vb = vb + b"\0" * (field - len(vb))
            out += struct.pack(e + "HH" + ("Q" if bigtiff else "I"), tag, typ, count) + vb
        out += struct.pack(e + nxt_fmt, 0)
    for i in range(T - 1):
        nxt_at = ifd_pos[i] + (8 if bigtiff else 2) + (20 if bigtiff else 12) * \
            struct.unpack(e + cnt_fmt, bytes(out[ifd_pos[i]:ifd_pos[i] + (8 if bigtiff else 2)]))[0]
        out[nxt_at:nxt_at + (8 if bigtiff else 4)] = struct.pack(e + nxt_fmt, ifd_pos[i + 1])
    bom = b"MM" if big_endian else b"II"
    if bigtiff:
        out[0:16] = bom + struct.pack(e + "HHHQ", 43, 8, 0, ifd_pos[0])
    else:
        out[0:8] = bom + struct.pack(e + "HI", 42, ifd_pos[0])
    with open(path, "wb") as fh:
        fh.write(bytes(out))


@pytest.mark.parametrize("kw", [
    dict(),
    dict(big_endian=True),
    dict(tile=(16, 16)),
    dict(tile=(16, 32), deflate=True, predictor=True, big_endian=True),
    dict(deflate=True, predictor=True),
    dict(bigtiff=True),
    dict(bigtiff=True, tile=(16, 16), deflate=True),
])
def test_written_tiff_layouts(tmp_path, kw):
    f = frames_u16(3, T=2, H=45, W=50)
    p = str(tmp_path / "w.tif")
    write_tiff(p, f, **kw)
    assert np.array_equal(api._read_video(p), f)


def test_signed_16bit_tiff_becomes_float(tmp_path):
    f = np.random.default_rng(4).integers(-30000, 30000, size=(2, 9, 11)).astype(np.int16)
    p = str(tmp_path / "s.tif")
    write_tiff(p, f, sample_format=2)
    got = api._read_video(p)
    assert got.dtype == np.float32 and np.array_equal(got, f.astype(np.float32))


def write_ets(path, frames_by_channel, dtype_code=4):
    """An .ets file laid out as the reference's MinimalETSParser reads it:
    SIS header, ETS header (data type, dims), chunk table of
    (4 bytes, 5 coordinates, offset, 8 bytes) with coordinate 2 the frame and
    coordinate 4 the channel, then raw little-endian frames."""
    ndim = 5
    ch0 = next(iter(frames_by_channel.values()))
    H, W = ch0.shape[1:]
    out = bytearray(b"\0" * 64)
    extra = len(out)
    ets = bytearray(b"ETS\0" + b"\0" * 4 + struct.pack("<I", dtype_code) + b"\0" * 16 + struct.pack("<II", W, H))
    out += ets + b"\0" * 16
    entries = []
    for ch, frames in frames_by_channel.items():
        for t, img in enumerate(frames):
            entries.append((ch, t, len(out)))
            out += np.ascontiguousarray(img).astype(img.dtype.newbyteorder("<")).tobytes()
    used = len(out)
    for ch, t, off in entries[::-1]:  # any order
        out += b"\0" * 4 + struct.pack("<5I", 0, 0, t, 0, ch) + struct.pack("<Q", off) + b"\0" * 8
    out[0:4] = b"SIS\0"
    out[12:16] = struct.pack("<I", ndim)
    out[16:24] = struct.pack("<Q", extra)
    out[32:40] = struct.pack("<Q", used)
    out[40:44] = struct.pack("<I", len(entries))
    with open(path, "wb") as fh:
        fh.write(bytes(out))


def test_ets_channels_and_vsi_path(tmp_path):
    a, b = frames_u16(5, T=3, H=12, W=17), frames_u16(6, T=2, H=12, W=17)
    stack = tmp_path / "_exp_" / "stack1"
    stack.mkdir(parents=True)
    write_ets(str(stack / "frame_t_0.ets"), {0: a, 1: b})
    ets = str(stack / "frame_t_0.ets")
    assert np.array_equal(gt.load(ets), a.astype(np.float32))
    assert np.array_equal(gt.load(ets, channel=1), b.astype(np.float32))
    vsi = str(tmp_path / "exp.vsi")
    assert np.array_equal(api._read_video(vsi, channel=1), b)
    assert np.array_equal(gt.load(vsi, frames=[2]), a[[2]].astype(np.float32))
    with pytest.raises(ValueError):
        gt.load(ets, channel=3)


def test_errors(tmp_path):
    with pytest.raises(FileNotFoundError):
        gt.load(str(tmp_path / "missing.tif"))
    with pytest.raises(FileNotFoundError):
        gt.load(str(tmp_path / "missing.vsi"))
    with pytest.raises(ValueError):
        gt.load(str(tmp_path / "x.avi"))
    bad = tmp_path / "bad.tif"
    bad.write_bytes(b"not a tiff at all")
    with pytest.raises(ValueError):
        gt.load(str(bad))
    f = frames_u16(7, T=2, H=8, W=8)
    p = str(tmp_path / "ok.tif")
    write_tiff(p, f)
    with pytest.raises(ValueError):
        gt.load(p, frames=[5])


@pytest.mark.gpu
def test_batch_on_a_tiff_path_equals_the_array(tmp_path):
    """batch(path) decodes the stack in its own dtype (u16) and tracks it:
    the same table as batch on the array, links included."""
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    from synth import video
    frames, _ = video(4, 96, 128, 30, seed=91)
    p = str(tmp_path / "stack.tif")
    imgs = [Image.fromarray(x) for x in frames]
    imgs[0].save(p, save_all=True, append_images=imgs[1:], compression="tiff_lzw")
    kw = dict(minmass=300.0, search_range=5.0, tqdm=False)
    a = gt.batch(p, 9, **kw)
    b = gt.batch(frames, 9, **kw)
    import pandas as pd
    pd.testing.assert_frame_equal(a, b)
    assert np.allclose(gt.mean_from_file(p), frames.mean(0), rtol=1e-6, atol=1e-3)
