// wire.cpp -- host-side file formats of the sequence driver.
//
// Output: the reference publishes the fused depth as a sensor_msgs/Image "32FC1" message
// (evaluate.cc:271-276; toImageMsg, src/tools/transport_util.h:103-132: row-major floats with a
// byte step) and shows a colour-mapped view (evaluate.cc:291-307).  Headless, these become
// files: PFM or NPY for the depth and binary PPM for the view.
//
// Input: the reference takes 8-bit frames from a ROS topic.  Here frames come from files:
// binary PGM/PPM, PNG (decoded with zlib's inflate; the PNG filters are undone here) or a
// 2-D uint8 NPY array.  Colour frames become grey with the BT.601 luma weights in 15-bit fixed
// point, round(0.299 * 2^15) = 9798, round(0.587 * 2^15) = 19235 and 2^15 - 9798 - 19235 = 3735,
// which is the integer form cv::cvtColor uses for 8-bit RGB -> GRAY.
#include <zlib.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pm_stereo.h"

namespace {

constexpr int kMaxSide = 1 << 15;

struct File {
    FILE* f;
    explicit File(const char* path, const char* mode) : f(path ? std::fopen(path, mode) : nullptr) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

bool little_endian_host() {
    const uint16_t one = 1;
    uint8_t b;
    std::memcpy(&b, &one, 1);
    return b == 1;
}

inline uint8_t luma(unsigned r, unsigned g, unsigned b) {
    return (uint8_t)((9798u * r + 19235u * g + 3735u * b + 16384u) >> 15);
}

bool read_all(const char* path, std::vector<uint8_t>& out) {
    File f(path, "rb");
    if (!f.f) return false;
    uint8_t buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, f.f)) > 0) out.insert(out.end(), buf, buf + n);
    return !std::ferror(f.f);
}

inline uint32_t be32(const uint8_t* p) {
    return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}

// ---- PNG ---------------------------------------------------------------------------------
bool decode_png(const std::vector<uint8_t>& in, int& W, int& H, std::vector<uint8_t>* grey) {
    static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    if (in.size() < 8 || std::memcmp(in.data(), sig, 8) != 0) return false;
    size_t pos = 8;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<uint8_t> idat, plte;
    bool have_ihdr = false, end = false;
    while (!end && pos + 12 <= in.size()) {
        const uint32_t len = be32(&in[pos]);
        if (len > in.size() - pos - 12) return false;
        const uint8_t* type = &in[pos + 4];
        const uint8_t* data = &in[pos + 8];
        if (!std::memcmp(type, "IHDR", 4)) {
            if (len != 13) return false;
            const uint32_t w = be32(data), h = be32(data + 4);
            if (w == 0 || h == 0 || w > (uint32_t)kMaxSide || h > (uint32_t)kMaxSide) return false;
            W = (int)w;
            H = (int)h;
            depth = data[8];
            ctype = data[9];
            interlace = data[12];
            if (data[10] != 0 || data[11] != 0) return false;
            have_ihdr = true;
        } else if (!std::memcmp(type, "PLTE", 4)) {
            plte.assign(data, data + len);
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), data, data + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            end = true;
        }
        pos += 12 + (size_t)len;
    }
    if (!have_ihdr || interlace != 0) return false;
    int channels;
    switch (ctype) {
        case 0: channels = 1; break;   // grey
        case 2: channels = 3; break;   // RGB
        case 3: channels = 1; break;   // palette index
        case 4: channels = 2; break;   // grey + alpha
        case 6: channels = 4; break;   // RGBA
        default: return false;
    }
    const bool ok_depth = (ctype == 0 && (depth == 1 || depth == 2 || depth == 4 || depth == 8 || depth == 16)) ||
                          (ctype == 3 && (depth == 1 || depth == 2 || depth == 4 || depth == 8)) ||
                          ((ctype == 2 || ctype == 4 || ctype == 6) && (depth == 8 || depth == 16));
    if (!ok_depth || (ctype == 3 && plte.size() < 3)) return false;
    if (!grey) return true;
    const size_t bits = (size_t)W * channels * depth;
    const size_t rowb = (bits + 7) / 8;
    const size_t bpp = (size_t)channels * depth >= 8 ? (size_t)channels * depth / 8 : 1;
    std::vector<uint8_t> raw((rowb + 1) * (size_t)H);
    uLongf rawlen = (uLongf)raw.size();
    if (uncompress(raw.data(), &rawlen, idat.data(), (uLong)idat.size()) != Z_OK || rawlen != raw.size())
        return false;
    // undo the per-row filters (None, Sub, Up, Average, Paeth)
    std::vector<uint8_t> img(rowb * (size_t)H);
    for (int y = 0; y < H; ++y) {
        const uint8_t ft = raw[(size_t)y * (rowb + 1)];
        const uint8_t* src = &raw[(size_t)y * (rowb + 1) + 1];
        uint8_t* cur = &img[(size_t)y * rowb];
        const uint8_t* up = y > 0 ? &img[(size_t)(y - 1) * rowb] : nullptr;
        for (size_t i = 0; i < rowb; ++i) {
            const int a = i >= bpp ? cur[i - bpp] : 0;
            const int b = up ? up[i] : 0;
            const int c = (up && i >= bpp) ? up[i - bpp] : 0;
            int v = src[i];
            switch (ft) {
                case 0: break;
                case 1: v += a; break;
                case 2: v += b; break;
                case 3: v += (a + b) >> 1; break;
                case 4: {
                    const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
                    v += (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
                    break;
                }
                default: return false;
            }
            cur[i] = (uint8_t)v;
        }
    }
    grey->resize((size_t)W * H);
    const size_t step = depth == 16 ? 2 : 1;   // 16-bit samples: keep the high (first) byte
    for (int y = 0; y < H; ++y) {
        const uint8_t* row = &img[(size_t)y * rowb];
        uint8_t* out = &(*grey)[(size_t)y * W];
        for (int x = 0; x < W; ++x) {
            if (depth < 8) {   // grey or palette packed 1, 2 or 4 bits per pixel, high bits first
                const size_t bit = (size_t)x * depth;
                const int v = (row[bit >> 3] >> (8 - depth - (int)(bit & 7))) & ((1 << depth) - 1);
                if (ctype == 0) {
                    out[x] = (uint8_t)(v * (255 / ((1 << depth) - 1)));
                } else {
                    if ((size_t)(3 * v + 2) >= plte.size()) return false;
                    out[x] = luma(plte[3 * v], plte[3 * v + 1], plte[3 * v + 2]);
                }
                continue;
            }
            const uint8_t* p = row + (size_t)x * channels * step;
            switch (ctype) {
                case 0:
                case 4: out[x] = p[0]; break;
                case 3:
                    if ((size_t)(3 * p[0] + 2) >= plte.size()) return false;
                    out[x] = luma(plte[3 * p[0]], plte[3 * p[0] + 1], plte[3 * p[0] + 2]);
                    break;
                default: out[x] = luma(p[0], p[step], p[2 * step]); break;
            }
        }
    }
    return true;
}

// ---- PGM / PPM ---------------------------------------------------------------------------
bool pnm_token(const std::vector<uint8_t>& in, size_t& pos, long& v) {
    for (;;) {
        while (pos < in.size() && (in[pos] == ' ' || in[pos] == '\t' || in[pos] == '\r' || in[pos] == '\n')) ++pos;
        if (pos < in.size() && in[pos] == '#') {
            while (pos < in.size() && in[pos] != '\n') ++pos;
            continue;
        }
        break;
    }
    if (pos >= in.size() || in[pos] < '0' || in[pos] > '9') return false;
    v = 0;
    while (pos < in.size() && in[pos] >= '0' && in[pos] <= '9' && v < (1L << 20)) v = v * 10 + (in[pos++] - '0');
    return true;
}

bool decode_pnm(const std::vector<uint8_t>& in, int& W, int& H, std::vector<uint8_t>* grey) {
    if (in.size() < 3 || in[0] != 'P' || (in[1] != '5' && in[1] != '6')) return false;
    const int channels = in[1] == '5' ? 1 : 3;
    size_t pos = 2;
    long w, h, maxv;
    if (!pnm_token(in, pos, w) || !pnm_token(in, pos, h) || !pnm_token(in, pos, maxv)) return false;
    if (w <= 0 || h <= 0 || w > kMaxSide || h > kMaxSide || maxv <= 0 || maxv > 65535) return false;
    ++pos;   // the single whitespace after maxval
    W = (int)w;
    H = (int)h;
    const size_t step = maxv > 255 ? 2 : 1;   // 16-bit samples are big-endian: keep the high byte
    if (in.size() < pos + (size_t)W * H * channels * step) return false;
    if (!grey) return true;
    grey->resize((size_t)W * H);
    const uint8_t* p = &in[pos];
    for (size_t i = 0; i < (size_t)W * H; ++i, p += channels * step)
        (*grey)[i] = channels == 1 ? p[0] : luma(p[0], p[step], p[2 * step]);
    return true;
}

// ---- NPY ---------------------------------------------------------------------------------
bool decode_npy(const std::vector<uint8_t>& in, int& W, int& H, std::vector<uint8_t>* grey) {
    if (in.size() < 10 || std::memcmp(in.data(), "\x93NUMPY", 6) != 0) return false;
    size_t hlen, off;
    if (in[6] == 1) {
        hlen = in[8] | ((size_t)in[9] << 8);
        off = 10;
    } else {
        if (in.size() < 12) return false;
        hlen = in[8] | ((size_t)in[9] << 8) | ((size_t)in[10] << 16) | ((size_t)in[11] << 24);
        off = 12;
    }
    if (in.size() < off + hlen) return false;
    const std::string hdr(reinterpret_cast<const char*>(&in[off]), hlen);
    if (hdr.find("'|u1'") == std::string::npos && hdr.find("'<u1'") == std::string::npos &&
        hdr.find("'u1'") == std::string::npos)
        return false;
    if (hdr.find("'fortran_order': True") != std::string::npos) return false;
    const size_t sp = hdr.find("'shape': (");
    if (sp == std::string::npos) return false;
    long h = 0, w = 0;
    if (std::sscanf(hdr.c_str() + sp + 10, "%ld, %ld)", &h, &w) != 2) return false;
    if (w <= 0 || h <= 0 || w > kMaxSide || h > kMaxSide) return false;
    W = (int)w;
    H = (int)h;
    if (in.size() < off + hlen + (size_t)W * H) return false;
    if (grey) grey->assign(in.begin() + (long)(off + hlen), in.begin() + (long)(off + hlen + (size_t)W * H));
    return true;
}

template <typename Row>
pm_status write_rows(FILE* f, int H, Row row) {
    for (int y = 0; y < H; ++y)
        if (!row(f, y)) return PM_ERR_INVALID_ARGUMENT;
    return PM_OK;
}

}  // namespace

extern "C" {

PM_API pm_status pm_write_pfm(const char* path, int W, int H, const float* data, size_t pitch) {
    if (W <= 0 || H <= 0 || !data) return PM_ERR_INVALID_ARGUMENT;
    if (pitch == 0) pitch = 4 * (size_t)W;
    if (pitch < 4 * (size_t)W) return PM_ERR_INVALID_ARGUMENT;
    File f(path, "wb");
    if (!f.f) return PM_ERR_INVALID_ARGUMENT;
    std::fprintf(f.f, "Pf\n%d %d\n%s\n", W, H, little_endian_host() ? "-1.0" : "1.0");
    const char* base = reinterpret_cast<const char*>(data);
    return write_rows(f.f, H, [&](FILE* o, int y) {   // PFM stores the bottom row first
        return std::fwrite(base + (size_t)(H - 1 - y) * pitch, 4, (size_t)W, o) == (size_t)W;
    });
}

PM_API pm_status pm_write_npy(const char* path, int W, int H, const float* data, size_t pitch) {
    if (W <= 0 || H <= 0 || !data) return PM_ERR_INVALID_ARGUMENT;
    if (pitch == 0) pitch = 4 * (size_t)W;
    if (pitch < 4 * (size_t)W) return PM_ERR_INVALID_ARGUMENT;
    File f(path, "wb");
    if (!f.f) return PM_ERR_INVALID_ARGUMENT;
    std::string hdr = "{'descr': '" + std::string(little_endian_host() ? "<f4" : ">f4") +
                      "', 'fortran_order': False, 'shape': (" + std::to_string(H) + ", " + std::to_string(W) + "), }";
    while ((10 + hdr.size() + 1) % 64) hdr += ' ';
    hdr += '\n';
    const uint8_t pre[10] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0, (uint8_t)(hdr.size() & 0xff),
                             (uint8_t)(hdr.size() >> 8)};
    if (std::fwrite(pre, 1, 10, f.f) != 10 || std::fwrite(hdr.data(), 1, hdr.size(), f.f) != hdr.size())
        return PM_ERR_INVALID_ARGUMENT;
    const char* base = reinterpret_cast<const char*>(data);
    return write_rows(f.f, H, [&](FILE* o, int y) {
        return std::fwrite(base + (size_t)y * pitch, 4, (size_t)W, o) == (size_t)W;
    });
}

PM_API pm_status pm_write_ppm(const char* path, int W, int H, const uint8_t* bgr, size_t pitch) {
    if (W <= 0 || H <= 0 || !bgr) return PM_ERR_INVALID_ARGUMENT;
    if (pitch == 0) pitch = 3 * (size_t)W;
    if (pitch < 3 * (size_t)W) return PM_ERR_INVALID_ARGUMENT;
    File f(path, "wb");
    if (!f.f) return PM_ERR_INVALID_ARGUMENT;
    std::fprintf(f.f, "P6\n%d %d\n255\n", W, H);
    std::vector<uint8_t> rgb(3 * (size_t)W);
    return write_rows(f.f, H, [&](FILE* o, int y) {
        const uint8_t* p = bgr + (size_t)y * pitch;
        for (int x = 0; x < W; ++x) {
            rgb[3 * x] = p[3 * x + 2];
            rgb[3 * x + 1] = p[3 * x + 1];
            rgb[3 * x + 2] = p[3 * x];
        }
        return std::fwrite(rgb.data(), 1, rgb.size(), o) == rgb.size();
    });
}

PM_API pm_status pm_read_image_u8(const char* path, int* W, int* H, uint8_t* dst, size_t capacity) {
    if (!path || !W || !H) return PM_ERR_INVALID_ARGUMENT;
    std::vector<uint8_t> in;
    if (!read_all(path, in)) return PM_ERR_INVALID_ARGUMENT;
    int w = 0, h = 0;
    bool (*dec[3])(const std::vector<uint8_t>&, int&, int&, std::vector<uint8_t>*) = {decode_png, decode_pnm,
                                                                                    decode_npy};
    for (auto d : dec) {
        if (!d(in, w, h, nullptr)) continue;
        *W = w;
        *H = h;
        if (!dst) return PM_OK;
        if (capacity < (size_t)w * h) return PM_ERR_INVALID_ARGUMENT;
        std::vector<uint8_t> grey;
        if (!d(in, w, h, &grey)) return PM_ERR_INVALID_ARGUMENT;
        std::memcpy(dst, grey.data(), grey.size());
        return PM_OK;
    }
    return PM_ERR_INVALID_ARGUMENT;
}

}  // extern "C"
