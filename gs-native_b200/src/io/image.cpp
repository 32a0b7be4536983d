// gs_native image IO (PPM, PNG writer) and area downscale.
#include "io/image.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <fstream>
#include <limits>

namespace gs_native {

namespace {

// CRC-32 of PNG chunks (ISO 3309 polynomial 0xEDB88320, reflected).
uint32_t Crc32(const uint8_t* data, size_t n, uint32_t crc = 0) {
    static const std::array<uint32_t, 256> table = [] {
        std::array<uint32_t, 256> t{};
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            t[i] = c;
        }
        return t;
    }();
    crc = ~crc;
    for (size_t i = 0; i < n; ++i) crc = table[(crc ^ data[i]) & 0xFFu] ^ (crc >> 8);
    return ~crc;
}

void PutBe32(std::vector<uint8_t>& out, uint32_t v) {
    for (int s = 24; s >= 0; s -= 8) out.push_back(static_cast<uint8_t>(v >> s));
}

void WriteChunk(std::ofstream& f, const char type[4], const std::vector<uint8_t>& payload) {
    std::vector<uint8_t> head;
    PutBe32(head, static_cast<uint32_t>(payload.size()));
    f.write(reinterpret_cast<const char*>(head.data()), 4);
    std::vector<uint8_t> body(type, type + 4);
    body.insert(body.end(), payload.begin(), payload.end());
    f.write(reinterpret_cast<const char*>(body.data()), static_cast<std::streamsize>(body.size()));
    std::vector<uint8_t> crc;
    PutBe32(crc, Crc32(body.data(), body.size()));
    f.write(reinterpret_cast<const char*>(crc.data()), 4);
}

}  // namespace

bool ReadPpm(const std::string& path, ImageU8& image) {
    std::ifstream f(path, std::ios::binary);
    std::string magic;
    int maxval = 0;
    if (!f || !(f >> magic) || magic != "P6") return false;
    auto next_int = [&](int& v) {
        while (f >> std::ws && f.peek() == '#') f.ignore(std::numeric_limits<std::streamsize>::max(), '\n');
        return static_cast<bool>(f >> v);
    };
    if (!next_int(image.width) || !next_int(image.height) || !next_int(maxval) || maxval != 255 || image.width <= 0 ||
        image.height <= 0)
        return false;
    f.get();  // the single whitespace byte after the header
    image.rgb.resize(static_cast<size_t>(image.width) * image.height * 3);
    return static_cast<bool>(f.read(reinterpret_cast<char*>(image.rgb.data()), image.rgb.size()));
}

bool WritePpm(const std::string& path, const ImageU8& image) {
    std::ofstream f(path, std::ios::binary);
    if (!f) return false;
    f << "P6\n" << image.width << " " << image.height << "\n255\n";
    f.write(reinterpret_cast<const char*>(image.rgb.data()), static_cast<std::streamsize>(image.rgb.size()));
    return static_cast<bool>(f);
}

bool WritePng(const std::string& path, const ImageU8& image) {
    if (image.width <= 0 || image.height <= 0 ||
        image.rgb.size() != static_cast<size_t>(image.width) * image.height * 3)
        return false;
    std::ofstream f(path, std::ios::binary);
    if (!f) return false;
    static const uint8_t signature[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
    f.write(reinterpret_cast<const char*>(signature), 8);
    std::vector<uint8_t> ihdr;
    PutBe32(ihdr, static_cast<uint32_t>(image.width));
    PutBe32(ihdr, static_cast<uint32_t>(image.height));
    ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});  // depth 8, RGB, deflate, filter 0, no interlace
    WriteChunk(f, "IHDR", ihdr);

    // Raw scanlines, each led by filter type 0.
    const size_t row = static_cast<size_t>(image.width) * 3;
    std::vector<uint8_t> raw;
    raw.reserve((row + 1) * image.height);
    for (int y = 0; y < image.height; ++y) {
        raw.push_back(0);
        raw.insert(raw.end(), image.rgb.begin() + y * row, image.rgb.begin() + (y + 1) * row);
    }
    // zlib stream: header (deflate, 32K window, no dictionary), stored blocks
    // of at most 65535 bytes, Adler-32 of the raw data.
    std::vector<uint8_t> z = {0x78, 0x01};
    for (size_t pos = 0; pos < raw.size() || raw.empty();) {
        const size_t n = std::min<size_t>(65535, raw.size() - pos);
        const bool last = pos + n == raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back(static_cast<uint8_t>(n & 0xFF));
        z.push_back(static_cast<uint8_t>(n >> 8));
        z.push_back(static_cast<uint8_t>(~n & 0xFF));
        z.push_back(static_cast<uint8_t>((~n >> 8) & 0xFF));
        z.insert(z.end(), raw.begin() + pos, raw.begin() + pos + n);
        pos += n;
        if (last) break;
    }
    uint32_t a = 1, b = 0;
    for (uint8_t v : raw) {
        a = (a + v) % 65521u;
        b = (b + a) % 65521u;
    }
    PutBe32(z, (b << 16) | a);
    WriteChunk(f, "IDAT", z);
    WriteChunk(f, "IEND", {});
    return static_cast<bool>(f);
}

ImageU8 DownscaleArea(const ImageU8& in, int k) {
    if (k <= 1) return in;
    ImageU8 out;
    out.width = std::max(1, static_cast<int>(std::lround(in.width / static_cast<float>(k))));
    out.height = std::max(1, static_cast<int>(std::lround(in.height / static_cast<float>(k))));
    out.rgb.assign(static_cast<size_t>(out.width) * out.height * 3, 0);
    const double sx = in.width / static_cast<double>(out.width), sy = in.height / static_cast<double>(out.height);
    for (int y = 0; y < out.height; ++y) {
        const int y0 = static_cast<int>(y * sy), y1 = std::min(in.height, std::max(y0 + 1, static_cast<int>((y + 1) * sy)));
        for (int x = 0; x < out.width; ++x) {
            const int x0 = static_cast<int>(x * sx),
                      x1 = std::min(in.width, std::max(x0 + 1, static_cast<int>((x + 1) * sx)));
            for (int c = 0; c < 3; ++c) {
                uint64_t s = 0;
                for (int yy = y0; yy < y1; ++yy)
                    for (int xx = x0; xx < x1; ++xx) s += in.rgb[(static_cast<size_t>(yy) * in.width + xx) * 3 + c];
                const uint64_t cnt = static_cast<uint64_t>(y1 - y0) * (x1 - x0);
                out.rgb[(static_cast<size_t>(y) * out.width + x) * 3 + c] = static_cast<uint8_t>((2 * s + cnt) / (2 * cnt));
            }
        }
    }
    return out;
}

ImageU8 ConcatHorizontal(const ImageU8& a, const ImageU8& b) {
    ImageU8 out;
    if (a.height != b.height) return out;
    out.width = a.width + b.width;
    out.height = a.height;
    out.rgb.resize(static_cast<size_t>(out.width) * out.height * 3);
    for (int y = 0; y < out.height; ++y) {
        std::copy_n(a.rgb.begin() + static_cast<size_t>(y) * a.width * 3, a.width * 3,
                    out.rgb.begin() + static_cast<size_t>(y) * out.width * 3);
        std::copy_n(b.rgb.begin() + static_cast<size_t>(y) * b.width * 3, b.width * 3,
                    out.rgb.begin() + (static_cast<size_t>(y) * out.width + a.width) * 3);
    }
    return out;
}

}  // namespace gs_native
