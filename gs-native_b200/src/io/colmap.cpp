// gs_native::ReadColmapScene and PPM IO.
#include "io/colmap.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <unordered_map>

namespace gs_native {

namespace {

constexpr int32_t kPinholeModel = 1;

template <typename T>
bool Read(std::ifstream& f, T& v) {
    return static_cast<bool>(f.read(reinterpret_cast<char*>(&v), sizeof(T)));
}

// Skips n bytes; false when the file ends first.
bool Skip(std::ifstream& f, uint64_t n) {
    f.ignore(static_cast<std::streamsize>(n));
    return f && static_cast<uint64_t>(f.gcount()) == n;
}

struct ColmapCamera {
    int32_t id = 0;
    int width = 0, height = 0;
    double fx = 0, fy = 0, cx = 0, cy = 0;
};

struct ColmapImage {
    int32_t camera_id = 0;
    float R[9];
    float t[3];
    std::string name;
};

// World-to-camera rotation of a unit quaternion (w, x, y, z).
void QuaternionToMatrix(double w, double x, double y, double z, float R[9]) {
    const double n = std::sqrt(w * w + x * x + y * y + z * z);
    w /= n;
    x /= n;
    y /= n;
    z /= n;
    R[0] = static_cast<float>(1 - 2 * (y * y + z * z));
    R[1] = static_cast<float>(2 * (x * y - w * z));
    R[2] = static_cast<float>(2 * (x * z + w * y));
    R[3] = static_cast<float>(2 * (x * y + w * z));
    R[4] = static_cast<float>(1 - 2 * (x * x + z * z));
    R[5] = static_cast<float>(2 * (y * z - w * x));
    R[6] = static_cast<float>(2 * (x * z - w * y));
    R[7] = static_cast<float>(2 * (y * z + w * x));
    R[8] = static_cast<float>(1 - 2 * (x * x + y * y));
}

bool ReadCameras(const std::string& path, ColmapCamera& cam) {
    std::ifstream f(path, std::ios::binary);
    uint64_t count = 0, w = 0, h = 0;
    int32_t model = 0;
    if (!f || !Read(f, count) || count != 1 || !Read(f, cam.id) || !Read(f, model) || model != kPinholeModel ||
        !Read(f, w) || !Read(f, h) || !Read(f, cam.fx) || !Read(f, cam.fy) || !Read(f, cam.cx) || !Read(f, cam.cy))
        return false;
    cam.width = static_cast<int>(w);
    cam.height = static_cast<int>(h);
    return cam.width > 0 && cam.height > 0;
}

bool ReadImages(const std::string& path, std::vector<ColmapImage>& images) {
    std::ifstream f(path, std::ios::binary);
    uint64_t count = 0;
    if (!f || !Read(f, count)) return false;
    images.clear();
    for (uint64_t i = 0; i < count; ++i) {
        ColmapImage im;
        int32_t id = 0;
        double q[4], t[3];
        if (!Read(f, id) || !Read(f, q[0]) || !Read(f, q[1]) || !Read(f, q[2]) || !Read(f, q[3]) ||
            !Read(f, t[0]) || !Read(f, t[1]) || !Read(f, t[2]) || !Read(f, im.camera_id))
            return false;
        QuaternionToMatrix(q[0], q[1], q[2], q[3], im.R);
        for (int a = 0; a < 3; ++a) im.t[a] = static_cast<float>(t[a]);
        if (!std::getline(f, im.name, '\0')) return false;
        uint64_t points2d = 0;
        if (!Read(f, points2d)) return false;
        if (!Skip(f, points2d * (2 * sizeof(double) + sizeof(int64_t)))) return false;
        images.push_back(std::move(im));
    }
    return true;
}

bool ReadPoints(const std::string& path, std::vector<float>& xyz, std::vector<float>& rgb) {
    std::ifstream f(path, std::ios::binary);
    uint64_t count = 0;
    if (!f || !Read(f, count)) return false;
    xyz.clear();
    rgb.clear();
    for (uint64_t i = 0; i < count; ++i) {
        uint64_t id = 0, track = 0;
        double p[3], error = 0;
        uint8_t c[3];
        if (!Read(f, id) || !Read(f, p[0]) || !Read(f, p[1]) || !Read(f, p[2]) || !Read(f, c[0]) || !Read(f, c[1]) ||
            !Read(f, c[2]) || !Read(f, error) || !Read(f, track))
            return false;
        if (!Skip(f, track * 2 * sizeof(int32_t))) return false;
        for (int a = 0; a < 3; ++a) {
            xyz.push_back(static_cast<float>(p[a]));
            rgb.push_back(c[a] / 255.0f);
        }
    }
    return true;
}

std::string PpmName(const std::string& name) {
    const size_t dot = name.find_last_of('.');
    if (dot != std::string::npos && name.substr(dot) == ".ppm") return name;
    return (dot == std::string::npos ? name : name.substr(0, dot)) + ".ppm";
}

}  // namespace

CameraParams MakeCamera(int width, int height, float fx, float fy, float cx, float cy, const float R_c_w[9],
                        const float t_c_w[3]) {
    CameraParams c{};
    c.fx_ = fx;
    c.fy_ = fy;
    c.cx_ = cx;
    c.cy_ = cy;
    std::memcpy(c.R_c_w_, R_c_w, sizeof(c.R_c_w_));
    std::memcpy(c.t_c_w_, t_c_w, sizeof(c.t_c_w_));
    c.near_depth_ = 0.2f;
    c.far_depth_ = std::numeric_limits<float>::max();
    c.width_ = width;
    c.height_ = height;
    c.tile_count_x_ = (width + 15) / 16;
    c.tile_count_y_ = (height + 15) / 16;
    return c;
}

bool ReadColmapScene(const std::string& scene_dir, int downscale, ColmapScene& scene) {
    const std::string sparse = scene_dir + "/sparse/0/", image_dir = scene_dir + "/images/";
    ColmapCamera cam;
    std::vector<ColmapImage> images;
    if (!ReadCameras(sparse + "cameras.bin", cam) || !ReadImages(sparse + "images.bin", images) ||
        !ReadPoints(sparse + "points3D.bin", scene.point_positions, scene.point_colors))
        return false;
    std::sort(images.begin(), images.end(),
              [](const ColmapImage& a, const ColmapImage& b) { return a.name < b.name; });
    scene.train_cameras.clear();
    scene.test_cameras.clear();
    scene.train_images.clear();
    scene.test_images.clear();
    for (size_t i = 0; i < images.size(); ++i) {
        const ColmapImage& im = images[i];
        if (im.camera_id != cam.id) return false;
        ImageU8 img;
        if (!ReadPpm(image_dir + im.name, img) && !ReadPpm(image_dir + PpmName(im.name), img)) return false;
        img = DownscaleArea(img, std::max(1, downscale));
        const float sx = img.width / static_cast<float>(cam.width), sy = img.height / static_cast<float>(cam.height);
        const CameraParams c =
            MakeCamera(img.width, img.height, static_cast<float>(cam.fx) * sx, static_cast<float>(cam.fy) * sy,
                       static_cast<float>(cam.cx) * sx - 0.5f, static_cast<float>(cam.cy) * sy - 0.5f, im.R, im.t);
        if (i % 8 == 0) {
            scene.test_cameras.push_back(c);
            scene.test_images.push_back(std::move(img));
            scene.test_names.push_back(im.name);
        } else {
            scene.train_cameras.push_back(c);
            scene.train_images.push_back(std::move(img));
            scene.train_names.push_back(im.name);
        }
    }
    return !scene.train_cameras.empty() && !scene.point_positions.empty();
}

}  // namespace gs_native
