// gt_video.cu — video files as frame providers (host code): TIFF stacks and
// Olympus .ets / .vsi, decoded into the engine's frame dtypes.
//
// Replaces path_to_iter and its providers (src/execute_gpu.rs:1186-1270,
// src/decoderiter.rs:64-481): a .tif/.tiff is every image of the file in IFD
// order (the reference's `tiff` crate 0.7.3 decoder), a .ets file is the
// frames of one channel of its chunk table, and a .vsi path names the .ets
// file `_<stem>_/stack1/frame_t_0.ets` beside it.
//
// TIFF support, written from the TIFF 6.0 specification: classic and BigTIFF,
// little and big endian, strips or tiles, one sample per pixel, 8/16-bit
// unsigned or signed integers and 32-bit floats, compression none, PackBits,
// LZW and Deflate (zlib), with or without horizontal differencing.  u8 and
// u16 images keep their type; i8, i16 and f32 images become f32 (the
// reference converts every frame to f32; the values are the same).
#include <zlib.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "gpu_tracking_b200.h"
#include "gt_runtime.cuh"

namespace {

thread_local std::string g_video_err;

gt_status verr(gt_status st, const std::string& msg) {
    g_video_err = msg;
    return st;
}

struct File {
    FILE* f = nullptr;
    int64_t size = 0;
    ~File() {
        if (f) fclose(f);
    }
    bool open(const std::string& path) {
        f = fopen(path.c_str(), "rb");
        if (!f) return false;
        fseeko(f, 0, SEEK_END);
        size = ftello(f);
        return true;
    }
    bool read_at(int64_t off, void* dst, size_t n) const {
        if (off < 0 || off + (int64_t)n > size) return false;
        if (fseeko(f, off, SEEK_SET) != 0) return false;
        return fread(dst, 1, n, f) == n;
    }
};

enum class Kind { Tiff, Ets };

struct TiffImage {
    uint32_t width = 0, height = 0, bits = 0, format = 1, compression = 1, predictor = 1, spp = 1, planar = 1;
    uint32_t rows_per_strip = 0, tile_w = 0, tile_h = 0;
    std::vector<uint64_t> offsets, counts;  // strips or tiles
};

}  // namespace

struct gt_video {
    Kind kind = Kind::Tiff;
    File file;
    bool big_endian = false;
    std::vector<TiffImage> images;    // TIFF: one per frame
    std::vector<uint64_t> ets_frames;  // ETS: byte offset of each frame
    int32_t H = 0, W = 0;
    int32_t src_type = 0;  // sample type of the file (see sample codes below)
    int32_t dtype = GT_DTYPE_U16;
};

namespace {

// sample codes: 1 u8, 2 u16, 3 i8, 4 i16, 5 f32
int sample_code(uint32_t bits, uint32_t format) {
    if (format == 1 && bits == 8) return 1;
    if (format == 1 && bits == 16) return 2;
    if (format == 2 && bits == 8) return 3;
    if (format == 2 && bits == 16) return 4;
    if (format == 3 && bits == 32) return 5;
    return 0;
}
int32_t dtype_of(int code) { return code == 1 ? GT_DTYPE_U8 : code == 2 ? GT_DTYPE_U16 : GT_DTYPE_F32; }
size_t bytes_of(int code) { return code == 1 || code == 3 ? 1 : code == 5 ? 4 : 2; }

struct Reader {
    const File& f;
    bool be;
    bool ok = true;
    uint64_t get(int64_t off, int n) {
        uint8_t b[8] = {};
        if (!f.read_at(off, b, (size_t)n)) {
            ok = false;
            return 0;
        }
        uint64_t v = 0;
        for (int i = 0; i < n; i++) v |= (uint64_t)b[be ? n - 1 - i : i] << (8 * i);
        return v;
    }
};

int type_size(uint32_t t) {
    switch (t) {
        case 1: case 2: case 6: case 7: return 1;  // BYTE ASCII SBYTE UNDEFINED
        case 3: case 8: return 2;                  // SHORT SSHORT
        case 4: case 9: case 11: case 13: return 4;  // LONG SLONG FLOAT IFD
        case 5: case 10: case 12: case 16: case 17: case 18: return 8;  // RATIONAL DOUBLE LONG8 ...
        default: return 0;
    }
}

gt_status parse_tiff(gt_video* v) {
    uint8_t hdr[16] = {};
    if (!v->file.read_at(0, hdr, 8)) return verr(GT_ERR_READ, "not a TIFF file (short header)");
    if (hdr[0] == 'I' && hdr[1] == 'I') v->big_endian = false;
    else if (hdr[0] == 'M' && hdr[1] == 'M') v->big_endian = true;
    else return verr(GT_ERR_READ, "not a TIFF file (byte order mark)");
    Reader r{v->file, v->big_endian};
    const uint64_t magic = r.get(2, 2);
    bool big = false;
    uint64_t ifd;
    if (magic == 42) {
        ifd = r.get(4, 4);
    } else if (magic == 43) {
        big = true;
        if (r.get(4, 2) != 8) return verr(GT_ERR_READ, "unsupported BigTIFF offset size");
        ifd = r.get(8, 8);
    } else {
        return verr(GT_ERR_READ, "not a TIFF file (magic number)");
    }
    const int count_size = big ? 8 : 2, entry_size = big ? 20 : 12, value_size = big ? 8 : 4;
    int guard = 0;
    while (ifd != 0 && r.ok) {
        if (++guard > (1 << 24)) return verr(GT_ERR_READ, "TIFF IFD chain does not end");
        const uint64_t n = r.get((int64_t)ifd, count_size);
        if (!r.ok || n > 100000) return verr(GT_ERR_READ, "corrupt TIFF IFD");
        TiffImage im;
        std::vector<uint64_t> bps;
        for (uint64_t e = 0; e < n; e++) {
            const int64_t eo = (int64_t)ifd + count_size + (int64_t)e * entry_size;
            const uint32_t tag = (uint32_t)r.get(eo, 2), type = (uint32_t)r.get(eo + 2, 2);
            const uint64_t cnt = r.get(eo + 4, value_size);
            const int ts = type_size(type);
            if (ts == 0 || cnt > (1ull << 32)) continue;
            const uint64_t total = (uint64_t)ts * cnt;
            const int64_t vo = total <= (uint64_t)value_size ? eo + 4 + value_size : (int64_t)r.get(eo + 4 + value_size, value_size);
            auto values = [&]() {
                std::vector<uint64_t> out((size_t)cnt);
                for (uint64_t i = 0; i < cnt; i++) out[i] = r.get(vo + (int64_t)i * ts, ts);
                return out;
            };
            switch (tag) {
                case 256: im.width = (uint32_t)values()[0]; break;
                case 257: im.height = (uint32_t)values()[0]; break;
                case 258: bps = values(); break;
                case 259: im.compression = (uint32_t)values()[0]; break;
                case 273: case 324: im.offsets = values(); break;
                case 277: im.spp = (uint32_t)values()[0]; break;
                case 278: im.rows_per_strip = (uint32_t)std::min<uint64_t>(values()[0], 0xFFFFFFFFu); break;
                case 279: case 325: im.counts = values(); break;
                case 284: im.planar = (uint32_t)values()[0]; break;
                case 317: im.predictor = (uint32_t)values()[0]; break;
                case 322: im.tile_w = (uint32_t)values()[0]; break;
                case 323: im.tile_h = (uint32_t)values()[0]; break;
                case 339: im.format = (uint32_t)values()[0]; break;
                default: break;
            }
            if (!r.ok) return verr(GT_ERR_READ, "TIFF tag value outside the file");
        }
        im.bits = bps.empty() ? 1 : (uint32_t)bps[0];
        if (im.rows_per_strip == 0) im.rows_per_strip = im.height;
        v->images.push_back(std::move(im));
        ifd = r.get((int64_t)ifd + count_size + (int64_t)n * entry_size, value_size);
    }
    if (!r.ok) return verr(GT_ERR_READ, "truncated TIFF file");
    if (v->images.empty()) return verr(GT_ERR_EMPTY_ITERATOR, "the TIFF file holds no image");
    const TiffImage& a = v->images[0];
    for (const TiffImage& im : v->images) {
        if (im.width != a.width || im.height != a.height || im.bits != a.bits || im.format != a.format)
            return verr(GT_ERR_DIMENSION_MISMATCH, "TIFF images differ in size or sample type");
        if (im.spp != 1) return verr(GT_ERR_READ, "only one sample per pixel (grayscale) is supported");
        const int code = sample_code(im.bits, im.format);
        if (!code)
            return verr(GT_ERR_READ, "unsupported TIFF sample type (" + std::to_string(im.bits) + "-bit, format " +
                                         std::to_string(im.format) + ")");
        if (im.offsets.empty() || im.offsets.size() != im.counts.size())
            return verr(GT_ERR_READ, "TIFF image without strip or tile offsets");
        if (im.compression != 1 && im.compression != 5 && im.compression != 8 && im.compression != 32946 &&
            im.compression != 32773)
            return verr(GT_ERR_READ, "unsupported TIFF compression " + std::to_string(im.compression));
        if (im.predictor != 1 && !(im.predictor == 2 && code != 5))
            return verr(GT_ERR_READ, "unsupported TIFF predictor " + std::to_string(im.predictor));
    }
    if (a.width == 0 || a.height == 0 || a.width > 1u << 20 || a.height > 1u << 20)
        return verr(GT_ERR_READ, "unsupported TIFF image size");
    v->H = (int32_t)a.height;
    v->W = (int32_t)a.width;
    v->src_type = sample_code(a.bits, a.format);
    v->dtype = dtype_of(v->src_type);
    return GT_OK;
}

// ---- decompression (TIFF 6.0 sections 9 and 13; Deflate through zlib)
bool unpackbits(const std::vector<uint8_t>& in, std::vector<uint8_t>& out, size_t want) {
    out.clear();
    size_t i = 0;
    while (i < in.size() && out.size() < want) {
        const int8_t n = (int8_t)in[i++];
        if (n >= 0) {
            const size_t len = (size_t)n + 1;
            if (i + len > in.size()) return false;
            out.insert(out.end(), in.begin() + i, in.begin() + i + len);
            i += len;
        } else if (n != -128) {
            if (i >= in.size()) return false;
            out.insert(out.end(), (size_t)(1 - n), in[i++]);
        }
    }
    return out.size() >= want;
}

bool unlzw(const std::vector<uint8_t>& in, std::vector<uint8_t>& out, size_t want) {
    out.clear();
    out.reserve(want);
    // dictionary: entry k = (prefix code, last byte, length)
    std::vector<int32_t> prefix(4096);
    std::vector<uint8_t> last(4096), first(4096);
    std::vector<uint32_t> len(4096);
    for (int k = 0; k < 256; k++) {
        prefix[k] = -1;
        last[k] = first[k] = (uint8_t)k;
        len[k] = 1;
    }
    int next = 258, width = 9, prev = -1;
    size_t bitpos = 0;
    const size_t nbits = in.size() * 8;
    std::vector<uint8_t> tmp;
    auto emit = [&](int code) {
        tmp.resize(len[code]);
        int c = code;
        for (int p = (int)len[code] - 1; p >= 0; p--) {
            tmp[p] = last[c];
            c = prefix[c];
        }
        out.insert(out.end(), tmp.begin(), tmp.end());
    };
    while (bitpos + width <= nbits && out.size() < want) {
        uint32_t code = 0;
        for (int b = 0; b < width; b++, bitpos++)
            code = (code << 1) | ((in[bitpos >> 3] >> (7 - (bitpos & 7))) & 1u);
        if (code == 257) break;
        if (code == 256) {
            next = 258;
            width = 9;
            prev = -1;
            continue;
        }
        if (prev < 0) {
            if (code > 255) return false;
            emit((int)code);
            prev = (int)code;
            continue;
        }
        if ((int)code < next) {
            emit((int)code);
            if (next < 4096) {
                prefix[next] = prev;
                last[next] = first[code];
                first[next] = first[prev];
                len[next] = len[prev] + 1;
                next++;
            }
        } else if ((int)code == next && next < 4096) {
            prefix[next] = prev;
            last[next] = first[prev];
            first[next] = first[prev];
            len[next] = len[prev] + 1;
            next++;
            emit((int)code);
        } else {
            return false;
        }
        prev = (int)code;
        // TIFF's LZW widens the code one entry early
        if (next + 1 >= (1 << width) && width < 12) width++;
    }
    return out.size() >= want;
}

bool inflate_all(const std::vector<uint8_t>& in, std::vector<uint8_t>& out, size_t want) {
    out.assign(want, 0);
    z_stream zs;
    std::memset(&zs, 0, sizeof(zs));
    if (inflateInit(&zs) != Z_OK) return false;
    zs.next_in = const_cast<Bytef*>(in.data());
    zs.avail_in = (uInt)in.size();
    zs.next_out = out.data();
    zs.avail_out = (uInt)want;
    const int rc = inflate(&zs, Z_FINISH);
    const size_t got = want - zs.avail_out;
    inflateEnd(&zs);
    return (rc == Z_STREAM_END || rc == Z_OK || rc == Z_BUF_ERROR) && got >= want;
}

// Undo horizontal differencing (predictor 2) on rows of `cols` samples.
void undo_predictor(std::vector<uint8_t>& buf, size_t rows, size_t cols, int code, bool be) {
    const size_t bs = bytes_of(code);
    for (size_t r = 0; r < rows; r++) {
        uint8_t* row = buf.data() + r * cols * bs;
        if (bs == 1) {
            for (size_t c = 1; c < cols; c++) row[c] = (uint8_t)(row[c] + row[c - 1]);
        } else {
            auto get = [&](size_t c) {
                return be ? (uint16_t)((row[2 * c] << 8) | row[2 * c + 1]) : (uint16_t)(row[2 * c] | (row[2 * c + 1] << 8));
            };
            auto put = [&](size_t c, uint16_t x) {
                if (be) {
                    row[2 * c] = (uint8_t)(x >> 8);
                    row[2 * c + 1] = (uint8_t)x;
                } else {
                    row[2 * c] = (uint8_t)x;
                    row[2 * c + 1] = (uint8_t)(x >> 8);
                }
            };
            for (size_t c = 1; c < cols; c++) put(c, (uint16_t)(get(c) + get(c - 1)));
        }
    }
}

// One sample of the decoded (file byte order) buffer as the output type.
template <typename O>
O sample_as(const uint8_t* p, int code, bool be) {
    switch (code) {
        case 1: return (O)p[0];
        case 3: return (O)(float)(int8_t)p[0];
        case 2: return (O)(uint16_t)(be ? (p[0] << 8) | p[1] : p[0] | (p[1] << 8));
        case 4: return (O)(float)(int16_t)(be ? (p[0] << 8) | p[1] : p[0] | (p[1] << 8));
        default: {
            uint32_t u = be ? ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]
                            : (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
            float f;
            std::memcpy(&f, &u, 4);
            return (O)f;
        }
    }
}

template <typename O>
gt_status decode_tiff_frame(const gt_video* v, const TiffImage& im, O* dst) {
    const int code = v->src_type;
    const size_t bs = bytes_of(code);
    const bool tiled = im.tile_w > 0 && im.tile_h > 0;
    const uint32_t bw = tiled ? im.tile_w : im.width;
    const uint32_t bh = tiled ? im.tile_h : im.rows_per_strip;
    const uint32_t across = tiled ? (im.width + bw - 1) / bw : 1;
    std::vector<uint8_t> raw, dec;
    for (size_t b = 0; b < im.offsets.size(); b++) {
        const uint32_t by = (uint32_t)(b / across) * bh, bx = (uint32_t)(b % across) * bw;
        if (by >= im.height) break;
        const uint32_t rows = tiled ? bh : std::min(bh, im.height - by);
        const size_t want = (size_t)rows * bw * bs;
        raw.resize((size_t)im.counts[b]);
        if (im.counts[b] > (uint64_t)v->file.size || !v->file.read_at((int64_t)im.offsets[b], raw.data(), raw.size()))
            return verr(GT_ERR_READ, "TIFF strip or tile outside the file");
        bool ok = true;
        switch (im.compression) {
            case 1:
                dec = raw;
                ok = dec.size() >= want;
                break;
            case 32773: ok = unpackbits(raw, dec, want); break;
            case 5: ok = unlzw(raw, dec, want); break;
            default: ok = inflate_all(raw, dec, want); break;
        }
        if (!ok) return verr(GT_ERR_READ, "corrupt compressed TIFF data");
        if (im.predictor == 2) undo_predictor(dec, rows, bw, code, v->big_endian);
        for (uint32_t y = 0; y < rows && by + y < im.height; y++)
            for (uint32_t x = 0; x < bw && bx + x < im.width; x++)
                dst[(size_t)(by + y) * im.width + bx + x] =
                    sample_as<O>(dec.data() + ((size_t)y * bw + x) * bs, code, v->big_endian);
    }
    return GT_OK;
}

// ---- Olympus .ets (the chunk table of src/decoderiter.rs:329-381)
gt_status parse_ets(gt_video* v, int32_t channel) {
    Reader r{v->file, false};
    uint8_t magic[4];
    if (!v->file.read_at(0, magic, 4) || std::memcmp(magic, "SIS\0", 4) != 0)
        return verr(GT_ERR_READ, "not an ETS file (SIS header)");
    const uint32_t ndim = (uint32_t)r.get(12, 4);
    const uint64_t extra = r.get(16, 8);
    const uint64_t used_off = r.get(32, 8);
    const uint32_t n_used = (uint32_t)r.get(40, 4);
    if (!r.ok || ndim < 5 || ndim > 64) return verr(GT_ERR_READ, "corrupt ETS header");
    if (!v->file.read_at((int64_t)extra, magic, 4) || std::memcmp(magic, "ETS\0", 4) != 0)
        return verr(GT_ERR_READ, "not an ETS file (ETS header)");
    const uint32_t type = (uint32_t)r.get((int64_t)extra + 8, 4);
    const uint32_t d0 = (uint32_t)r.get((int64_t)extra + 28, 4), d1 = (uint32_t)r.get((int64_t)extra + 32, 4);
    int code;
    switch (type) {
        case 2: code = 1; break;  // u8
        case 4: code = 2; break;  // u16
        case 1: code = 3; break;  // i8
        case 3: code = 4; break;  // i16
        case 9: code = 5; break;  // f32
        default: return verr(GT_ERR_READ, "unsupported ETS data type " + std::to_string(type));
    }
    if (!r.ok || d0 == 0 || d1 == 0 || d0 > 1u << 20 || d1 > 1u << 20) return verr(GT_ERR_READ, "corrupt ETS dimensions");
    // entries: 4 bytes, ndim coordinates, the frame's byte offset, 8 bytes
    const int64_t entry = 4 + 4 * (int64_t)ndim + 8 + 8;
    std::vector<int64_t> frames;  // -1: no chunk
    for (uint32_t i = 0; i < n_used; i++) {
        const int64_t eo = (int64_t)used_off + (int64_t)i * entry;
        const uint32_t t = (uint32_t)r.get(eo + 4 + 4 * 2, 4), ch = (uint32_t)r.get(eo + 4 + 4 * 4, 4);
        const uint64_t off = r.get(eo + 4 + 4 * (int64_t)ndim, 8);
        if (!r.ok) return verr(GT_ERR_READ, "truncated ETS chunk table");
        if ((int32_t)ch != channel) continue;
        if (t >= (1u << 24)) return verr(GT_ERR_READ, "corrupt ETS frame index");
        if (frames.size() <= t) frames.resize(t + 1, -1);
        frames[t] = (int64_t)off;
    }
    if (frames.empty()) return verr(GT_ERR_INVALID_ARGUMENT, "the requested channel wasn't found in the file");
    for (int64_t o : frames)
        if (o < 0) return verr(GT_ERR_READ, "an ETS frame has no data chunk");
    v->ets_frames.assign(frames.begin(), frames.end());
    v->W = (int32_t)d0;
    v->H = (int32_t)d1;
    v->src_type = code;
    v->dtype = dtype_of(code);
    return GT_OK;
}

template <typename O>
gt_status decode_ets_frame(const gt_video* v, uint64_t off, O* dst) {
    const size_t bs = bytes_of(v->src_type), n = (size_t)v->H * v->W;
    std::vector<uint8_t> raw(n * bs);
    if (!v->file.read_at((int64_t)off, raw.data(), raw.size())) return verr(GT_ERR_READ, "ETS frame outside the file");
    for (size_t i = 0; i < n; i++) dst[i] = sample_as<O>(raw.data() + i * bs, v->src_type, false);
    return GT_OK;
}

template <typename O>
gt_status read_frames(gt_video* v, const int64_t* keys, int64_t n, O* dst) {
    const int64_t T = v->kind == Kind::Tiff ? (int64_t)v->images.size() : (int64_t)v->ets_frames.size();
    const size_t px = (size_t)v->H * v->W;
    for (int64_t i = 0; i < n; i++) {
        const int64_t k = keys ? keys[i] : i;
        if (k < 0 || k >= T)
            return verr(GT_ERR_FRAME_OUT_OF_BOUNDS, "tried to access frame " + std::to_string(k) +
                                                        " of a video with " + std::to_string(T) + " frames");
        gt_status st = v->kind == Kind::Tiff ? decode_tiff_frame<O>(v, v->images[(size_t)k], dst + (size_t)i * px)
                                             : decode_ets_frame<O>(v, v->ets_frames[(size_t)k], dst + (size_t)i * px);
        if (st != GT_OK) return st;
    }
    return GT_OK;
}

std::string lower_ext(const std::string& p) {
    const size_t slash = p.find_last_of('/');
    const size_t dot = p.find_last_of('.');
    if (dot == std::string::npos || (slash != std::string::npos && dot < slash)) return "";
    std::string e = p.substr(dot + 1);
    for (char& ch : e) ch = (char)std::tolower((unsigned char)ch);
    return e;
}

}  // namespace

// ---- decoding on the GPU
// The compressed strips or tiles of the requested frames are read from the
// file on the host (only I/O), copied to the device in one piece and decoded
// there: one CTA per strip or tile runs its LZW or PackBits stream on one
// thread (both formats are sequential by construction) with the LZW
// dictionary in shared memory, then the CTA undoes horizontal differencing
// row by row and converts the samples into the output frames.  Deflate
// blocks are inflated on the host (zlib) and travel as uncompressed ones.
// The byte sequences, and so the samples, are those of the host decoder.
namespace {

enum BlockComp : uint32_t { kCompNone = 0, kCompPackBits = 1, kCompLzw = 2 };

struct DecodeBlock {
    uint64_t src;       // byte offset of the block's stream in the uploaded buffer
    uint64_t dec;       // byte offset of its decoded bytes in the decode buffer
    uint32_t src_len;   // stream bytes
    uint32_t want;      // decoded bytes the block must yield (rows x bw x sample bytes)
    uint32_t comp;      // BlockComp
    int32_t frame;      // output frame (position in the requested list)
    int32_t by, bx;     // first row / column of the block in the frame
    int32_t rows, bw;   // rows and samples per row of the block
    int32_t pred;       // TIFF predictor (2: horizontal differencing)
    int32_t pad;
};

constexpr int kLzwCodes = 4096;
constexpr int kDecodeThreads = 128;

// TIFF 6.0 section 13 (LZW).  Every dictionary entry's string occurs in the
// output already written: an entry made after code c is the previous code's
// string followed by the first byte of c's string, which the output holds
// contiguously where the previous code was emitted.  So an entry is an
// (offset, length) pair and emitting a code copies bytes the block already
// decoded.  Same codes, same widening rule and same outputs as the host
// decoder; false on a malformed stream or a short result.
__device__ bool lzw_decode_block(const uint8_t* __restrict__ in, uint32_t in_len, uint8_t* __restrict__ out,
                                 uint32_t want, uint32_t* __restrict__ eoff, uint16_t* __restrict__ elen) {
    int next = 258, width = 9, prev = -1;
    uint32_t pos = 0, prev_pos = 0, prev_len = 0;
    uint64_t bitpos = 0;
    const uint64_t nbits = (uint64_t)in_len * 8;
    while (bitpos + width <= nbits && pos < want) {
        uint32_t code = 0;
        for (int b = 0; b < width; b++, bitpos++)
            code = (code << 1) | ((in[bitpos >> 3] >> (7 - (bitpos & 7))) & 1u);
        if (code == 257) break;
        if (code == 256) {
            next = 258;
            width = 9;
            prev = -1;
            continue;
        }
        uint32_t len;
        const bool after_clear = prev < 0;
        if (after_clear) {
            if (code > 255) return false;
            out[pos] = (uint8_t)code;
            len = 1;
        } else if ((int)code < next) {
            if (code < 256) {
                out[pos] = (uint8_t)code;
                len = 1;
            } else {
                const uint32_t o = eoff[code];
                len = elen[code];
                for (uint32_t k = 0; k < len && pos + k < want; k++) out[pos + k] = out[o + k];
            }
            if (next < kLzwCodes) {
                eoff[next] = prev_pos;
                elen[next] = (uint16_t)(prev_len + 1);
                next++;
            }
        } else if ((int)code == next && next < kLzwCodes) {
            // the previous string and its own first byte
            len = prev_len + 1;
            for (uint32_t k = 0; k < prev_len && pos + k < want; k++) out[pos + k] = out[prev_pos + k];
            if (pos + prev_len < want) out[pos + prev_len] = out[prev_pos];
            eoff[next] = prev_pos;
            elen[next] = (uint16_t)len;
            next++;
        } else {
            return false;
        }
        prev = (int)code;
        prev_pos = pos;
        prev_len = len;
        pos += len;
        // TIFF's LZW widens the code one entry early (not after a clear code's first code)
        if (!after_clear && next + 1 >= (1 << width) && width < 12) width++;
    }
    return pos >= want;
}


// TIFF 6.0 section 9 (PackBits), as the host decoder: whole runs, the result
// at least `want` bytes (bytes past it are not stored).
__device__ bool packbits_decode_block(const uint8_t* __restrict__ in, uint32_t in_len, uint8_t* __restrict__ out,
                                      uint32_t want) {
    uint32_t i = 0, pos = 0;
    while (i < in_len && pos < want) {
        const int n = (int)(int8_t)in[i++];
        if (n >= 0) {
            const uint32_t len = (uint32_t)n + 1;
            if (i + len > in_len) return false;
            for (uint32_t k = 0; k < len && pos + k < want; k++) out[pos + k] = in[i + k];
            i += len;
            pos += len;
        } else if (n != -128) {
            if (i >= in_len) return false;
            const uint32_t len = (uint32_t)(1 - n);
            const uint8_t byte = in[i++];
            for (uint32_t k = 0; k < len && pos + k < want; k++) out[pos + k] = byte;
            pos += len;
        }
    }
    return pos >= want;
}

// One sample of a decoded block (file byte order) as the output type (the
// host decoder's sample_as).
template <typename O>
__device__ __forceinline__ O sample_dev(const uint8_t* p, int code, bool be) {
    switch (code) {
        case 1: return (O)p[0];
        case 3: return (O)(float)(int8_t)p[0];
        case 2: return (O)(uint16_t)(be ? (p[0] << 8) | p[1] : p[0] | (p[1] << 8));
        case 4: return (O)(float)(int16_t)(be ? (p[0] << 8) | p[1] : p[0] | (p[1] << 8));
        default: {
            const uint32_t u = be ? ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]
                                  : (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) |
                                        ((uint32_t)p[3] << 24);
            return (O)__uint_as_float(u);
        }
    }
}

// One CTA per block: decode (thread 0), undo horizontal differencing (a
// thread per row, the host decoder's sample arithmetic), store the samples
// into the block's place in its output frame.
template <typename O>
__global__ void __launch_bounds__(kDecodeThreads)
decode_blocks_kernel(const uint8_t* __restrict__ src, const DecodeBlock* __restrict__ blocks, uint8_t* __restrict__ dec,
                     O* __restrict__ dst, int32_t H, int32_t W, int code, int be, uint32_t* __restrict__ bad) {
    __shared__ uint32_t eoff[kLzwCodes];
    __shared__ uint16_t elen[kLzwCodes];
    const DecodeBlock b = blocks[blockIdx.x];
    const uint8_t* in = src + b.src;
    uint8_t* out = dec + b.dec;
    const int tid = threadIdx.x;
    if (b.comp == kCompNone) {
        for (uint32_t i = tid; i < b.want; i += blockDim.x) out[i] = in[i];
    } else if (tid == 0) {
        const bool ok = b.comp == kCompLzw ? lzw_decode_block(in, b.src_len, out, b.want, eoff, elen)
                                           : packbits_decode_block(in, b.src_len, out, b.want);
        if (!ok) atomicExch(bad, 1u);
    }
    __syncthreads();
    const int bs = (code == 1 || code == 3) ? 1 : (code == 5 ? 4 : 2);
    if (b.pred == 2) {
        // TIFF 6.0 section 14: running sums along each row, modulo the sample width
        for (int r = tid; r < b.rows; r += blockDim.x) {
            uint8_t* row = out + (size_t)r * b.bw * bs;
            if (bs == 1) {
                for (int c = 1; c < b.bw; c++) row[c] = (uint8_t)(row[c] + row[c - 1]);
            } else {
                uint32_t prev = be ? ((row[0] << 8) | row[1]) : (row[0] | (row[1] << 8));
                for (int c = 1; c < b.bw; c++) {
                    uint8_t* q = row + 2 * c;
                    const uint32_t cur = be ? ((q[0] << 8) | q[1]) : (q[0] | (q[1] << 8));
                    const uint32_t x = (cur + prev) & 0xFFFFu;
                    if (be) {
                        q[0] = (uint8_t)(x >> 8);
                        q[1] = (uint8_t)x;
                    } else {
                        q[0] = (uint8_t)x;
                        q[1] = (uint8_t)(x >> 8);
                    }
                    prev = x;
                }
            }
        }
        __syncthreads();
    }
    const int64_t n = (int64_t)b.rows * b.bw;
    O* frame = dst + (size_t)b.frame * H * W;
    for (int64_t i = tid; i < n; i += blockDim.x) {
        const int y = (int)(i / b.bw), x = (int)(i - (int64_t)y * b.bw);
        if (b.by + y < H && b.bx + x < W)
            frame[(size_t)(b.by + y) * W + b.bx + x] = sample_dev<O>(out + (size_t)i * bs, code, be != 0);
    }
}

}  // namespace

namespace {

// Reads the streams of the requested frames (host I/O; Deflate inflated on
// the host) and decodes them on the context's device into d_dst, in batches
// of about kDecodeBatchBytes of streams.
constexpr size_t kDecodeBatchBytes = 256u << 20;

template <typename O>
gt_status read_frames_device(gt_video* v, gt_ctx* ctx, const int64_t* keys, int64_t n, O* d_dst) {
    using gt::rt::DBuf;
    const int64_t T = v->kind == Kind::Tiff ? (int64_t)v->images.size() : (int64_t)v->ets_frames.size();
    const int code = v->src_type;
    const size_t bs = bytes_of(code);
    std::vector<uint8_t> hsrc, raw, dec;
    std::vector<DecodeBlock> blocks;
    uint64_t dec_bytes = 0;
    auto flush = [&]() -> gt_status {
        if (blocks.empty()) return GT_OK;
        auto cuda_err = [](cudaError_t e) { return verr(GT_ERR_CUDA, std::string("CUDA error ") + cudaGetErrorString(e)); };
        cudaError_t e;
        if ((e = ctx->vd_src.ensure(std::max<size_t>(hsrc.size(), 16))) != cudaSuccess) return cuda_err(e);
        if ((e = ctx->vd_dec.ensure(std::max<uint64_t>(dec_bytes, 16))) != cudaSuccess) return cuda_err(e);
        if ((e = ctx->vd_blk.ensure(blocks.size() * sizeof(DecodeBlock))) != cudaSuccess) return cuda_err(e);
        if ((e = ctx->vd_bad.ensure(4)) != cudaSuccess) return cuda_err(e);
        if ((e = cudaMemsetAsync(ctx->vd_bad.p, 0, 4, ctx->st)) != cudaSuccess) return cuda_err(e);
        if (!hsrc.empty() &&
            (e = cudaMemcpyAsync(ctx->vd_src.p, hsrc.data(), hsrc.size(), cudaMemcpyHostToDevice, ctx->st)) != cudaSuccess)
            return cuda_err(e);
        if ((e = cudaMemcpyAsync(ctx->vd_blk.p, blocks.data(), blocks.size() * sizeof(DecodeBlock),
                                 cudaMemcpyHostToDevice, ctx->st)) != cudaSuccess)
            return cuda_err(e);
        decode_blocks_kernel<O><<<(unsigned)blocks.size(), kDecodeThreads, 0, ctx->st>>>(
            ctx->vd_src.as<uint8_t>(), ctx->vd_blk.as<DecodeBlock>(), ctx->vd_dec.as<uint8_t>(), d_dst, v->H, v->W,
            code, v->big_endian ? 1 : 0, ctx->vd_bad.as<uint32_t>());
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(e);
        uint32_t bad = 0;
        if ((e = cudaMemcpyAsync(&bad, ctx->vd_bad.p, 4, cudaMemcpyDeviceToHost, ctx->st)) != cudaSuccess)
            return cuda_err(e);
        if ((e = cudaStreamSynchronize(ctx->st)) != cudaSuccess) return cuda_err(e);
        if (bad) return verr(GT_ERR_READ, "corrupt compressed TIFF data");
        hsrc.clear();
        blocks.clear();
        dec_bytes = 0;
        return GT_OK;
    };
    auto add = [&](const uint8_t* stream, size_t len, uint32_t comp, uint32_t want, int32_t frame, int32_t by,
                   int32_t bx, int32_t rows, int32_t bw, int32_t pred) {
        DecodeBlock b;
        b.src = hsrc.size();
        b.dec = dec_bytes;
        b.src_len = (uint32_t)len;
        b.want = want;
        b.comp = comp;
        b.frame = frame;
        b.by = by;
        b.bx = bx;
        b.rows = rows;
        b.bw = bw;
        b.pred = pred;
        b.pad = 0;
        hsrc.insert(hsrc.end(), stream, stream + len);
        hsrc.resize((hsrc.size() + 15) & ~(size_t)15);
        dec_bytes += ((uint64_t)want + 15) & ~(uint64_t)15;
        blocks.push_back(b);
    };
    for (int64_t i = 0; i < n; i++) {
        const int64_t k = keys ? keys[i] : i;
        if (k < 0 || k >= T)
            return verr(GT_ERR_FRAME_OUT_OF_BOUNDS, "tried to access frame " + std::to_string(k) +
                                                        " of a video with " + std::to_string(T) + " frames");
        if (v->kind == Kind::Ets) {
            const size_t want = (size_t)v->H * v->W * bs;
            raw.resize(want);
            if (!v->file.read_at((int64_t)v->ets_frames[(size_t)k], raw.data(), want))
                return verr(GT_ERR_READ, "ETS frame outside the file");
            // ETS samples are little endian: the kernel reads them with the video's byte order flag (false)
            add(raw.data(), want, kCompNone, (uint32_t)want, (int32_t)i, 0, 0, v->H, v->W, 1);
        } else {
            const TiffImage& im = v->images[(size_t)k];
            const bool tiled = im.tile_w > 0 && im.tile_h > 0;
            const uint32_t bw = tiled ? im.tile_w : im.width;
            const uint32_t bh = tiled ? im.tile_h : im.rows_per_strip;
            const uint32_t across = tiled ? (im.width + bw - 1) / bw : 1;
            for (size_t b = 0; b < im.offsets.size(); b++) {
                const uint32_t by = (uint32_t)(b / across) * bh, bx = (uint32_t)(b % across) * bw;
                if (by >= im.height) break;
                const uint32_t rows = tiled ? bh : std::min(bh, im.height - by);
                const size_t want = (size_t)rows * bw * bs;
                if (want >= (1ull << 32)) return verr(GT_ERR_READ, "TIFF strip or tile too large");
                raw.resize((size_t)im.counts[b]);
                if (im.counts[b] > (uint64_t)v->file.size ||
                    !v->file.read_at((int64_t)im.offsets[b], raw.data(), raw.size()))
                    return verr(GT_ERR_READ, "TIFF strip or tile outside the file");
                switch (im.compression) {
                    case 1:
                        if (raw.size() < want) return verr(GT_ERR_READ, "corrupt compressed TIFF data");
                        add(raw.data(), want, kCompNone, (uint32_t)want, (int32_t)i, (int32_t)by, (int32_t)bx,
                            (int32_t)rows, (int32_t)bw, (int32_t)im.predictor);
                        break;
                    case 32773:
                    case 5:
                        add(raw.data(), raw.size(), im.compression == 5 ? kCompLzw : kCompPackBits, (uint32_t)want,
                            (int32_t)i, (int32_t)by, (int32_t)bx, (int32_t)rows, (int32_t)bw, (int32_t)im.predictor);
                        break;
                    default:
                        if (!inflate_all(raw, dec, want)) return verr(GT_ERR_READ, "corrupt compressed TIFF data");
                        add(dec.data(), want, kCompNone, (uint32_t)want, (int32_t)i, (int32_t)by, (int32_t)bx,
                            (int32_t)rows, (int32_t)bw, (int32_t)im.predictor);
                        break;
                }
                if (hsrc.size() >= kDecodeBatchBytes) {
                    gt_status st = flush();
                    if (st != GT_OK) return st;
                }
            }
        }
        if (hsrc.size() >= kDecodeBatchBytes) {
            gt_status st = flush();
            if (st != GT_OK) return st;
        }
    }
    return flush();
}

}  // namespace

// the span check of the context unit (gt_api.cu)
extern "C" gt_status gt__device_span_check(gt_ctx* ctx, const void* p, size_t bytes, const char* what);

extern "C" {

GT_API gt_status gt_video_open(const char* path, int32_t channel, gt_video** out) {
    if (!path || !out) return verr(GT_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    std::string p(path);
    const std::string ext = lower_ext(p);
    if (ext.empty()) return verr(GT_ERR_INVALID_ARGUMENT, "could not determine extension of file '" + p + "'");
    std::unique_ptr<gt_video> v(new gt_video());
    std::string open_path = p;
    if (ext == "tif" || ext == "tiff") {
        v->kind = Kind::Tiff;
    } else if (ext == "ets" || ext == "vsi") {
        v->kind = Kind::Ets;
        if (ext == "vsi") {
            const size_t slash = p.find_last_of('/');
            const std::string dir = slash == std::string::npos ? "." : p.substr(0, slash);
            const std::string name = slash == std::string::npos ? p : p.substr(slash + 1);
            const std::string stem = name.substr(0, name.find_last_of('.'));
            if (stem.empty()) return verr(GT_ERR_FILE_NOT_FOUND, "vsi doesn't have a filename: '" + p + "'");
            open_path = dir + "/_" + stem + "_/stack1/frame_t_0.ets";
        }
    } else {
        return verr(GT_ERR_INVALID_ARGUMENT, "unsupported file format: " + ext);
    }
    if (channel < 0) return verr(GT_ERR_INVALID_ARGUMENT, "channel must be >= 0");
    if (!v->file.open(open_path)) return verr(GT_ERR_FILE_NOT_FOUND, "could not find file '" + open_path + "'");
    gt_status st = v->kind == Kind::Tiff ? parse_tiff(v.get()) : parse_ets(v.get(), channel);
    if (st != GT_OK) return st;
    *out = v.release();
    return GT_OK;
}

GT_API gt_status gt_video_info(const gt_video* v, int64_t* T, int32_t* H, int32_t* W, int32_t* dtype) {
    if (!v) return verr(GT_ERR_INVALID_ARGUMENT, "null video");
    if (T) *T = v->kind == Kind::Tiff ? (int64_t)v->images.size() : (int64_t)v->ets_frames.size();
    if (H) *H = v->H;
    if (W) *W = v->W;
    if (dtype) *dtype = v->dtype;
    return GT_OK;
}

GT_API gt_status gt_video_read(gt_video* v, const int64_t* frames, int64_t n, int32_t dtype, void* dst) {
    if (!v || (!dst && n > 0) || n < 0) return verr(GT_ERR_INVALID_ARGUMENT, "null argument");
    if (dtype == GT_DTYPE_F32) return read_frames<float>(v, frames, n, (float*)dst);
    if (dtype != v->dtype) return verr(GT_ERR_INVALID_ARGUMENT, "frames decode to their own dtype or to f32");
    if (dtype == GT_DTYPE_U16) return read_frames<uint16_t>(v, frames, n, (uint16_t*)dst);
    return read_frames<uint8_t>(v, frames, n, (uint8_t*)dst);
}

GT_API gt_status gt_video_read_device(gt_ctx* ctx, gt_video* v, const int64_t* frames, int64_t n, int32_t dtype,
                                      void* dst) {
    if (!ctx || !v || (!dst && n > 0) || n < 0) return verr(GT_ERR_INVALID_ARGUMENT, "null argument");
    if (dtype != GT_DTYPE_F32 && dtype != v->dtype)
        return verr(GT_ERR_INVALID_ARGUMENT, "frames decode to their own dtype or to f32");
    if (n == 0) return GT_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return verr(GT_ERR_CUDA, "cudaSetDevice failed");
    const size_t eb = dtype == GT_DTYPE_F32 ? 4 : dtype == GT_DTYPE_U16 ? 2 : 1;
    if (gt__device_span_check(ctx, dst, (size_t)n * v->H * v->W * eb, "frames") != GT_OK)
        return verr(GT_ERR_INVALID_ARGUMENT, gt_last_error(ctx));
    if (dtype == GT_DTYPE_F32) return read_frames_device<float>(v, ctx, frames, n, (float*)dst);
    if (dtype == GT_DTYPE_U16) return read_frames_device<uint16_t>(v, ctx, frames, n, (uint16_t*)dst);
    return read_frames_device<uint8_t>(v, ctx, frames, n, (uint8_t*)dst);
}

GT_API void gt_video_close(gt_video* v) { delete v; }

GT_API const char* gt_video_last_error(void) { return g_video_err.c_str(); }

}  // extern "C"
