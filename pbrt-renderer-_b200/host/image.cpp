// image.cpp — texture images as 8-bit RGBA (what LoadTexture requests from
// its image library, src/gpu/DXRApp_Textures.cpp:34-40): PNG, TGA, BMP and
// binary PPM / PGM, row 0 = top of the image.
//
// PNG follows the PNG specification (RFC 2083 / ISO 15948): chunks IHDR,
// PLTE, tRNS, IDAT, IEND; a zlib stream (RFC 1950) holding DEFLATE data
// (RFC 1951: stored, fixed-Huffman and dynamic-Huffman blocks); scanline
// filters None / Sub / Up / Average / Paeth; colour types grey, RGB,
// palette, grey+alpha, RGBA at every bit depth the format allows; Adam7
// interlacing.  16-bit samples keep their high byte, low bit depths scale to
// 0..255, a tRNS colour key makes matching pixels transparent.  Every read
// is bounds-checked: malformed files raise NoriException.
#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "nori/nori.h"

namespace nori {

namespace {

[[noreturn]] void bad(const std::string &path, const char *what) {
    throw NoriException("image \"" + path + "\": " + what);
}

// ---- DEFLATE (RFC 1951) --------------------------------------------------------------------------
class Inflater {
public:
    // Output beyond `limit` bytes is an error (the image's size bounds it).
    Inflater(const std::string &path, const uint8_t *in, size_t n, size_t limit, std::vector<uint8_t> &out)
        : m_path(path), m_in(in), m_n(n), m_limit(limit), m_out(out) {}

    void run() {
        bool last = false;
        while (!last) {
            last = bits(1) != 0;
            uint32_t type = bits(2);
            if (type == 0) stored();
            else if (type == 1) fixedBlock();
            else if (type == 2) dynamicBlock();
            else bad(m_path, "invalid DEFLATE block type");
        }
    }

private:
    // Canonical code (RFC 1951 section 3.2.2): the codes of length l are the
    // consecutive values first[l] .. first[l] + count[l] - 1, assigned to the
    // symbols of that length in increasing order; base[l] is where those
    // symbols start in `symbol`.
    struct Huffman {
        uint16_t count[16], first[16], base[16];
        uint16_t symbol[320];
    };

    uint32_t bits(int need) {
        while (m_cnt < need) {
            if (m_pos >= m_n) bad(m_path, "DEFLATE stream ends early");
            m_buf |= (uint32_t)m_in[m_pos++] << m_cnt;
            m_cnt += 8;
        }
        uint32_t v = m_buf & ((1u << need) - 1u);
        m_buf >>= need;
        m_cnt -= need;
        return v;
    }

    void build(Huffman &h, const uint8_t *len, int n) {
        std::memset(&h, 0, sizeof(h));
        for (int s = 0; s < n; s++) h.count[len[s]]++;
        h.count[0] = 0;
        uint32_t code = 0, idx = 0;
        for (int l = 1; l < 16; l++) {
            code = (code + h.count[l - 1]) << 1;
            if (code + h.count[l] > (1u << l)) bad(m_path, "over-subscribed Huffman code");
            h.first[l] = (uint16_t)code;
            h.base[l] = (uint16_t)idx;
            idx += h.count[l];
        }
        uint16_t fill[16];
        std::memcpy(fill, h.base, sizeof(fill));
        for (int s = 0; s < n; s++)
            if (len[s]) h.symbol[fill[len[s]]++] = (uint16_t)s;
    }

    // Codes arrive most-significant bit first: extend the code one bit at a
    // time until it falls inside the range of its length.
    int decode(const Huffman &h) {
        uint32_t code = 0;
        for (int l = 1; l < 16; l++) {
            code = (code << 1) | bits(1);
            uint32_t k = code - h.first[l];  // wraps for code < first
            if (k < h.count[l]) return h.symbol[h.base[l] + k];
        }
        bad(m_path, "invalid Huffman code");
    }

    void stored() {
        m_buf = 0;  // skip to a byte boundary
        m_cnt = 0;
        if (m_pos + 4 > m_n) bad(m_path, "truncated stored block");
        uint32_t len = m_in[m_pos] | (m_in[m_pos + 1] << 8);
        uint32_t nlen = m_in[m_pos + 2] | (m_in[m_pos + 3] << 8);
        m_pos += 4;
        if ((len ^ 0xFFFFu) != nlen) bad(m_path, "stored block length check failed");
        if (m_pos + len > m_n) bad(m_path, "truncated stored block");
        if (m_out.size() + len > m_limit) bad(m_path, "more image data than the image holds");
        m_out.insert(m_out.end(), m_in + m_pos, m_in + m_pos + len);
        m_pos += len;
    }

    void codes(const Huffman &lit, const Huffman &dist) {
        static const uint16_t lbase[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                                           31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
        static const uint8_t lextra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                           2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
        static const uint16_t dbase[30] = {1,   2,   3,   4,   5,   7,    9,    13,   17,   25,
                                           33,  49,  65,  97,  129, 193,  257,  385,  513,  769,
                                           1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
        static const uint8_t dextra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6,
                                           6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
        for (;;) {
            int sym = decode(lit);
            if (sym < 256) {
                if (m_out.size() >= m_limit) bad(m_path, "more image data than the image holds");
                m_out.push_back((uint8_t)sym);
            } else if (sym == 256) {
                return;
            } else {
                sym -= 257;
                if (sym >= 29) bad(m_path, "invalid length symbol");
                uint32_t len = lbase[sym] + bits(lextra[sym]);
                int ds = decode(dist);
                if (ds >= 30) bad(m_path, "invalid distance symbol");
                uint32_t d = dbase[ds] + bits(dextra[ds]);
                if (d > m_out.size()) bad(m_path, "distance reaches before the output");
                if (m_out.size() + len > m_limit) bad(m_path, "more image data than the image holds");
                size_t from = m_out.size() - d;
                for (uint32_t k = 0; k < len; k++) m_out.push_back(m_out[from + k]);
            }
        }
    }

    void fixedBlock() {
        uint8_t len[288 + 30];
        for (int s = 0; s < 144; s++) len[s] = 8;
        for (int s = 144; s < 256; s++) len[s] = 9;
        for (int s = 256; s < 280; s++) len[s] = 7;
        for (int s = 280; s < 288; s++) len[s] = 8;
        for (int s = 0; s < 30; s++) len[288 + s] = 5;
        Huffman lit, dist;
        build(lit, len, 288);
        build(dist, len + 288, 30);
        codes(lit, dist);
    }

    void dynamicBlock() {
        static const uint8_t order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
        uint32_t nlen = bits(5) + 257, ndist = bits(5) + 1, ncode = bits(4) + 4;
        if (nlen > 286 || ndist > 30) bad(m_path, "bad dynamic block counts");
        uint8_t lengths[320] = {0};
        for (uint32_t i = 0; i < ncode; i++) lengths[order[i]] = (uint8_t)bits(3);
        Huffman lencode;
        build(lencode, lengths, 19);
        uint32_t i = 0;
        while (i < nlen + ndist) {
            int sym = decode(lencode);
            if (sym < 16) {
                lengths[i++] = (uint8_t)sym;
                continue;
            }
            uint32_t rep = 0;
            uint8_t val = 0;
            if (sym == 16) {
                if (i == 0) bad(m_path, "repeat with no previous length");
                val = lengths[i - 1];
                rep = 3 + bits(2);
            } else if (sym == 17) {
                rep = 3 + bits(3);
            } else {
                rep = 11 + bits(7);
            }
            if (i + rep > nlen + ndist) bad(m_path, "code lengths overflow");
            while (rep--) lengths[i++] = val;
        }
        if (lengths[256] == 0) bad(m_path, "no end-of-block code");
        Huffman lit, dist;
        build(lit, lengths, (int)nlen);
        build(dist, lengths + nlen, (int)ndist);
        codes(lit, dist);
    }

    const std::string &m_path;
    const uint8_t *m_in;
    size_t m_n, m_limit, m_pos = 0;
    uint32_t m_buf = 0;
    int m_cnt = 0;
    std::vector<uint8_t> &m_out;
};

uint32_t be32(const uint8_t *p) { return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]; }

uint8_t paeth(int a, int b, int c) {
    int p = a + b - c, pa = p > a ? p - a : a - p, pb = p > b ? p - b : b - p, pc = p > c ? p - c : c - p;
    if (pa <= pb && pa <= pc) return (uint8_t)a;
    return (uint8_t)(pb <= pc ? b : c);
}

// Reverses the scanline filters of a w x h (sub-)image in place; returns the
// bytes consumed from `data` (rows of 1 + rowBytes).
size_t unfilter(const std::string &path, uint8_t *data, size_t avail, uint32_t w, uint32_t h, uint32_t bitsPerPixel,
                std::vector<uint8_t> &rows) {
    size_t rowBytes = ((size_t)w * bitsPerPixel + 7) / 8;
    size_t need = (rowBytes + 1) * h;
    if (need > avail) bad(path, "image data shorter than the image");
    size_t bpp = std::max<size_t>(1, bitsPerPixel / 8);
    rows.assign(rowBytes * h, 0);
    for (uint32_t y = 0; y < h; y++) {
        uint8_t f = data[y * (rowBytes + 1)];
        const uint8_t *src = data + y * (rowBytes + 1) + 1;
        uint8_t *cur = &rows[y * rowBytes];
        const uint8_t *prev = y ? &rows[(y - 1) * rowBytes] : nullptr;
        for (size_t i = 0; i < rowBytes; i++) {
            int a = i >= bpp ? cur[i - bpp] : 0, b = prev ? prev[i] : 0, c = (prev && i >= bpp) ? prev[i - bpp] : 0;
            int x = src[i];
            switch (f) {
                case 0: cur[i] = (uint8_t)x; break;
                case 1: cur[i] = (uint8_t)(x + a); break;
                case 2: cur[i] = (uint8_t)(x + b); break;
                case 3: cur[i] = (uint8_t)(x + ((a + b) >> 1)); break;
                case 4: cur[i] = (uint8_t)(x + paeth(a, b, c)); break;
                default: bad(path, "invalid PNG filter type");
            }
        }
    }
    return need;
}

struct PngInfo {
    uint32_t w, h, depth, colour;
    std::vector<uint8_t> palette;  // RGBA per entry
    bool hasKey = false;
    uint16_t key[3] = {0, 0, 0};
};

uint32_t channels(uint32_t colour) { return colour == 0 ? 1 : colour == 2 ? 3 : colour == 3 ? 1 : colour == 4 ? 2 : 4; }

// Sample k of a row at the image's bit depth (16-bit: the full value).
uint32_t sample(const uint8_t *row, size_t k, uint32_t depth) {
    if (depth == 8) return row[k];
    if (depth == 16) return ((uint32_t)row[2 * k] << 8) | row[2 * k + 1];
    size_t bit = k * depth;
    return (row[bit >> 3] >> (8 - depth - (bit & 7))) & ((1u << depth) - 1u);
}

// RGBA8 of pixel x of a decoded row.
void pixel(const PngInfo &in, const uint8_t *row, uint32_t x, uint8_t *dst) {
    const uint32_t ch = channels(in.colour), d = in.depth;
    auto to8 = [&](uint32_t v) -> uint8_t {
        if (d == 16) return (uint8_t)(v >> 8);
        if (d == 8) return (uint8_t)v;
        return (uint8_t)(v * (255u / ((1u << d) - 1u)));  // 1, 2, 4 bits: 255, 85, 17
    };
    uint32_t s[4];
    for (uint32_t c = 0; c < ch; c++) s[c] = sample(row, (size_t)x * ch + c, d);
    switch (in.colour) {
        case 0: {
            uint8_t g = to8(s[0]);
            dst[0] = dst[1] = dst[2] = g;
            dst[3] = (in.hasKey && s[0] == in.key[0]) ? 0 : 255;
            break;
        }
        case 2:
            for (int c = 0; c < 3; c++) dst[c] = to8(s[c]);
            dst[3] = (in.hasKey && s[0] == in.key[0] && s[1] == in.key[1] && s[2] == in.key[2]) ? 0 : 255;
            break;
        case 3: {
            size_t e = s[0];
            if (4 * e + 3 >= in.palette.size()) {
                dst[0] = dst[1] = dst[2] = 0;  // index past the palette: black, opaque
                dst[3] = 255;
            } else {
                std::memcpy(dst, &in.palette[4 * e], 4);
            }
            break;
        }
        case 4: {
            uint8_t g = to8(s[0]);
            dst[0] = dst[1] = dst[2] = g;
            dst[3] = to8(s[1]);
            break;
        }
        default:
            for (int c = 0; c < 4; c++) dst[c] = to8(s[c]);
    }
}

void loadPNG(const std::string &path, const std::vector<uint8_t> &f, uint32_t &W, uint32_t &H, std::vector<uint8_t> &rgba) {
    PngInfo in{};
    std::vector<uint8_t> z;
    size_t at = 8;
    bool haveHeader = false, interlaced = false;
    while (true) {
        if (at + 12 > f.size()) bad(path, "PNG ends before IEND");
        uint32_t len = be32(&f[at]);
        if (len > f.size() - at - 12) bad(path, "PNG chunk runs past the file");
        const uint8_t *type = &f[at + 4], *data = &f[at + 8];
        if (!std::memcmp(type, "IHDR", 4)) {
            if (len < 13) bad(path, "short IHDR");
            in.w = be32(data);
            in.h = be32(data + 4);
            in.depth = data[8];
            in.colour = data[9];
            interlaced = data[12] == 1;
            if (data[10] != 0 || data[11] != 0 || data[12] > 1) bad(path, "unknown PNG compression, filter or interlace");
            bool ok = (in.colour == 0 && (in.depth == 1 || in.depth == 2 || in.depth == 4 || in.depth == 8 || in.depth == 16)) ||
                      (in.colour == 3 && (in.depth == 1 || in.depth == 2 || in.depth == 4 || in.depth == 8)) ||
                      ((in.colour == 2 || in.colour == 4 || in.colour == 6) && (in.depth == 8 || in.depth == 16));
            if (!ok) bad(path, "invalid PNG colour type / bit depth");
            if (!in.w || !in.h || in.w > 32768 || in.h > 32768 || (uint64_t)in.w * in.h > (1u << 28))
                bad(path, "PNG size outside 1..32768 or above 2^28 pixels");
            haveHeader = true;
        } else if (!std::memcmp(type, "PLTE", 4)) {
            if (len % 3 || len > 768) bad(path, "bad PLTE");
            in.palette.assign(len / 3 * 4, 255);
            for (uint32_t e = 0; e < len / 3; e++)
                for (int c = 0; c < 3; c++) in.palette[4 * e + c] = data[3 * e + c];
        } else if (!std::memcmp(type, "tRNS", 4)) {
            if (in.colour == 3) {
                for (uint32_t e = 0; e < len && 4 * e + 3 < in.palette.size(); e++) in.palette[4 * e + 3] = data[e];
            } else if (in.colour == 0 && len >= 2) {
                in.hasKey = true;
                in.key[0] = (uint16_t)((data[0] << 8) | data[1]);
            } else if (in.colour == 2 && len >= 6) {
                in.hasKey = true;
                for (int c = 0; c < 3; c++) in.key[c] = (uint16_t)((data[2 * c] << 8) | data[2 * c + 1]);
            }
        } else if (!std::memcmp(type, "IDAT", 4)) {
            z.insert(z.end(), data, data + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            break;
        }
        at += 12 + (size_t)len;
    }
    if (!haveHeader) bad(path, "PNG without IHDR");
    if (in.colour == 3 && in.palette.empty()) bad(path, "palette PNG without PLTE");
    if (z.size() < 2 || (z[0] & 0x0F) != 8 || ((z[0] << 8) | z[1]) % 31) bad(path, "bad zlib header");
    if (z[1] & 0x20) bad(path, "zlib preset dictionary");
    static const uint32_t x0[7] = {0, 4, 0, 2, 0, 1, 0}, y0[7] = {0, 0, 4, 0, 2, 0, 1};  // Adam7 passes:
    static const uint32_t dx[7] = {8, 8, 4, 4, 2, 2, 1}, dy[7] = {8, 8, 8, 4, 4, 2, 2};   // (x0 + i dx, y0 + j dy)
    const uint32_t bpp = channels(in.colour) * in.depth;
    W = in.w;
    H = in.h;
    auto passW = [&](int p) { return W > x0[p] ? (W - x0[p] + dx[p] - 1) / dx[p] : 0u; };
    auto passH = [&](int p) { return H > y0[p] ? (H - y0[p] + dy[p] - 1) / dy[p] : 0u; };
    size_t expect = 0;  // filtered bytes: rows of 1 + rowBytes, per pass when interlaced
    if (!interlaced) expect = (((size_t)W * bpp + 7) / 8 + 1) * H;
    else
        for (int p = 0; p < 7; p++)
            if (passW(p) && passH(p)) expect += (((size_t)passW(p) * bpp + 7) / 8 + 1) * passH(p);
    std::vector<uint8_t> raw;
    raw.reserve(expect);
    Inflater(path, z.data() + 2, z.size() - 2, expect, raw).run();
    rgba.assign((size_t)W * H * 4, 0);
    std::vector<uint8_t> rows;
    if (!interlaced) {
        unfilter(path, raw.data(), raw.size(), W, H, bpp, rows);
        size_t rb = ((size_t)W * bpp + 7) / 8;
        for (uint32_t y = 0; y < H; y++)
            for (uint32_t x = 0; x < W; x++) pixel(in, &rows[y * rb], x, &rgba[((size_t)y * W + x) * 4]);
        return;
    }
    size_t off = 0;
    for (int p = 0; p < 7; p++) {
        uint32_t pw = passW(p), ph = passH(p);
        if (!pw || !ph) continue;
        off += unfilter(path, raw.data() + off, raw.size() - off, pw, ph, bpp, rows);
        size_t rb = ((size_t)pw * bpp + 7) / 8;
        for (uint32_t j = 0; j < ph; j++)
            for (uint32_t i = 0; i < pw; i++)
                pixel(in, &rows[j * rb], i, &rgba[(((size_t)y0[p] + j * dy[p]) * W + x0[p] + i * dx[p]) * 4]);
    }
}

uint16_t le16(const uint8_t *p) { return (uint16_t)(p[0] | (p[1] << 8)); }
uint32_t le32(const uint8_t *p) { return p[0] | (p[1] << 8) | (p[2] << 16) | ((uint32_t)p[3] << 24); }

// TGA: uncompressed or run-length true colour (24/32 bit) and grey (8 bit).
void loadTGA(const std::string &path, const std::vector<uint8_t> &f, uint32_t &W, uint32_t &H, std::vector<uint8_t> &rgba) {
    if (f.size() < 18) bad(path, "short TGA header");
    uint32_t idlen = f[0], cmap = f[1], type = f[2];
    W = le16(&f[12]);
    H = le16(&f[14]);
    uint32_t bits = f[16], desc = f[17];
    bool rle = type == 10 || type == 11, grey = type == 3 || type == 11;
    if (cmap || !(type == 2 || type == 3 || type == 10 || type == 11)) bad(path, "unsupported TGA type");
    if ((grey && bits != 8) || (!grey && bits != 24 && bits != 32)) bad(path, "unsupported TGA pixel size");
    if (!W || !H) bad(path, "empty TGA");
    const uint32_t bp = bits / 8;
    size_t at = 18 + idlen;
    rgba.assign((size_t)W * H * 4, 255);
    auto put = [&](size_t k, const uint8_t *p) {
        uint8_t *d = &rgba[k * 4];
        if (grey) d[0] = d[1] = d[2] = p[0];
        else { d[0] = p[2]; d[1] = p[1]; d[2] = p[0]; if (bp == 4) d[3] = p[3]; }
    };
    size_t n = (size_t)W * H, k = 0;
    while (k < n) {
        if (!rle) {
            if (at + bp > f.size()) bad(path, "truncated TGA");
            put(k++, &f[at]);
            at += bp;
            continue;
        }
        if (at >= f.size()) bad(path, "truncated TGA");
        uint32_t hdr = f[at++], cnt = (hdr & 0x7F) + 1;
        if (k + cnt > n) bad(path, "TGA run past the image");
        if (hdr & 0x80) {
            if (at + bp > f.size()) bad(path, "truncated TGA");
            for (uint32_t i = 0; i < cnt; i++) put(k++, &f[at]);
            at += bp;
        } else {
            if (at + (size_t)bp * cnt > f.size()) bad(path, "truncated TGA");
            for (uint32_t i = 0; i < cnt; i++, at += bp) put(k++, &f[at]);
        }
    }
    if (!(desc & 0x20)) {  // bottom-up storage: flip to top row first
        for (uint32_t y = 0; y < H / 2; y++)
            std::swap_ranges(&rgba[(size_t)y * W * 4], &rgba[(size_t)(y + 1) * W * 4], &rgba[(size_t)(H - 1 - y) * W * 4]);
    }
}

// BMP: uncompressed 24 / 32-bit (BGR / BGRA), bottom-up or top-down.
void loadBMP(const std::string &path, const std::vector<uint8_t> &f, uint32_t &W, uint32_t &H, std::vector<uint8_t> &rgba) {
    if (f.size() < 54 || le32(&f[14]) < 40) bad(path, "short or unsupported BMP header");
    uint32_t dataAt = le32(&f[10]);
    int32_t w = (int32_t)le32(&f[18]), h = (int32_t)le32(&f[22]);
    uint32_t bits = le16(&f[28]), comp = le32(&f[30]);
    if ((bits != 24 && bits != 32) || (comp != 0 && !(comp == 3 && bits == 32))) bad(path, "unsupported BMP format");
    if (w <= 0 || h == 0 || w > 32768 || h > 32768 || h < -32768) bad(path, "bad BMP size");
    bool topDown = h < 0;
    W = (uint32_t)w;
    H = (uint32_t)(topDown ? -h : h);
    size_t bp = bits / 8, stride = ((size_t)W * bp + 3) & ~(size_t)3;
    if (dataAt + stride * H > f.size()) bad(path, "truncated BMP");
    rgba.assign((size_t)W * H * 4, 255);
    for (uint32_t y = 0; y < H; y++) {
        const uint8_t *row = &f[dataAt + stride * (topDown ? y : H - 1 - y)];
        for (uint32_t x = 0; x < W; x++) {
            uint8_t *d = &rgba[((size_t)y * W + x) * 4];
            d[0] = row[x * bp + 2];
            d[1] = row[x * bp + 1];
            d[2] = row[x * bp];
            if (bp == 4) d[3] = row[x * bp + 3];
        }
    }
}

// Binary PPM (P6) / PGM (P5), maxval <= 255.
void loadPNM(const std::string &path, const std::vector<uint8_t> &f, uint32_t &W, uint32_t &H, std::vector<uint8_t> &rgba) {
    size_t at = 2;
    auto field = [&]() -> uint32_t {
        while (at < f.size()) {
            if (f[at] == '#') { while (at < f.size() && f[at] != '\n') at++; }
            else if (f[at] == ' ' || f[at] == '\t' || f[at] == '\r' || f[at] == '\n') at++;
            else break;
        }
        uint64_t v = 0;
        size_t start = at;
        while (at < f.size() && f[at] >= '0' && f[at] <= '9' && v < 100000) v = v * 10 + (f[at++] - '0');
        if (at == start) bad(path, "bad PNM header");
        return (uint32_t)v;
    };
    bool colour = f[1] == '6';
    W = field();
    H = field();
    uint32_t maxv = field();
    at++;  // the single whitespace byte before the samples
    if (!W || !H || W > 32768 || H > 32768 || !maxv || maxv > 255) bad(path, "unsupported PNM size or maxval");
    size_t ch = colour ? 3 : 1;
    if (at + (size_t)W * H * ch > f.size()) bad(path, "truncated PNM");
    rgba.assign((size_t)W * H * 4, 255);
    for (size_t k = 0; k < (size_t)W * H; k++)
        for (int c = 0; c < 3; c++) {
            uint32_t v = f[at + k * ch + (colour ? c : 0)];
            rgba[k * 4 + c] = (uint8_t)(maxv == 255 ? v : (v * 255 + maxv / 2) / maxv);
        }
}

}  // namespace

void loadImageRGBA8(const std::string &path, uint32_t &width, uint32_t &height, std::vector<uint8_t> &rgba) {
    std::ifstream is(path, std::ios::binary);
    if (!is) throw NoriException("image \"" + path + "\": cannot open");
    std::vector<uint8_t> f((std::istreambuf_iterator<char>(is)), std::istreambuf_iterator<char>());
    static const uint8_t pngSig[8] = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
    if (f.size() >= 8 && !std::memcmp(f.data(), pngSig, 8)) return loadPNG(path, f, width, height, rgba);
    if (f.size() >= 2 && f[0] == 'B' && f[1] == 'M') return loadBMP(path, f, width, height, rgba);
    if (f.size() >= 2 && f[0] == 'P' && (f[1] == '5' || f[1] == '6')) return loadPNM(path, f, width, height, rgba);
    if (f.size() >= 3 && f[0] == 0xFF && f[1] == 0xD8 && f[2] == 0xFF)
        bad(path, "JPEG textures are not supported (convert to PNG)");
    std::string ext = path.size() > 4 ? path.substr(path.size() - 4) : "";
    for (char &c : ext) c = (char)std::tolower((unsigned char)c);
    if (ext == ".tga") return loadTGA(path, f, width, height, rgba);
    bad(path, "unknown image format (PNG, TGA, BMP, PPM/PGM are read)");
}

}  // namespace nori
