// 8-bit RGB image files without OpenCV: binary PPM (P6) read/write and a PNG
// writer (colour type 2, bit depth 8, filter 0, deflate "stored" blocks with
// zlib Adler-32 and PNG CRC-32). The demo renderer writes its renders, ground
// truths and side-by-side comparisons with it (the reference uses cv::imwrite,
// demo/render.cpp:134-140).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace gs_native {

struct ImageU8 {
    int width = 0, height = 0;
    std::vector<uint8_t> rgb;  // HWC
};

bool ReadPpm(const std::string& path, ImageU8& image);
bool WritePpm(const std::string& path, const ImageU8& image);
bool WritePng(const std::string& path, const ImageU8& image);

// Integer-factor area downscale to (lround(w / k), lround(h / k)): each output
// pixel is the rounded mean of the input pixels its footprint covers.
ImageU8 DownscaleArea(const ImageU8& in, int k);

// [a | b] side by side (equal heights).
ImageU8 ConcatHorizontal(const ImageU8& a, const ImageU8& b);

}  // namespace gs_native
