// Gaussian PLY IO (see ply.h).
#include "io/ply.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>

#include "core/types/buffers.h"

namespace gs_native {

namespace {

constexpr int kRest = 15;  // SH coefficients per channel beyond DC
constexpr int kRowFloats = 3 + 3 + 3 + 3 * kRest + 1 + 3 + 4;

// Axis-angle -> unit quaternion (w, x, y, z) (data_io.cpp:296-300).
void ToQuaternion(const float w[3], float q[4]) {
    double theta = std::sqrt(double(w[0]) * w[0] + double(w[1]) * w[1] + double(w[2]) * w[2]);
    double k = theta < 1e-8 ? 0.5 : std::sin(0.5 * theta) / theta;
    q[0] = static_cast<float>(std::cos(0.5 * theta));
    q[1] = static_cast<float>(k * w[0]);
    q[2] = static_cast<float>(k * w[1]);
    q[3] = static_cast<float>(k * w[2]);
}

// Unit quaternion -> axis-angle with angle in [0, pi] (the convention of
// Eigen::AngleAxis used by data_io.cpp:519-525).
void FromQuaternion(double qw, double qx, double qy, double qz, float w[3]) {
    double n = std::sqrt(qw * qw + qx * qx + qy * qy + qz * qz);
    qw /= n;
    qx /= n;
    qy /= n;
    qz /= n;
    if (qw < 0) {
        qw = -qw;
        qx = -qx;
        qy = -qy;
        qz = -qz;
    }
    double s = std::sqrt(qx * qx + qy * qy + qz * qz);
    if (s < 1e-12) {
        w[0] = w[1] = w[2] = 0.0f;
        return;
    }
    double angle = 2.0 * std::atan2(s, qw);
    w[0] = static_cast<float>(qx / s * angle);
    w[1] = static_cast<float>(qy / s * angle);
    w[2] = static_cast<float>(qz / s * angle);
}

}  // namespace

std::vector<Gaussian> UnpackGaussians(const float* p, int count) {
    std::vector<Gaussian> out(static_cast<size_t>(std::max(count, 0)));
    const size_t N = static_cast<size_t>(std::max(count, 0));
    for (size_t i = 0; i < N; ++i) {
        Gaussian& g = out[i];
        for (int a = 0; a < 3; ++a) {
            g.position_[a] = p[(kPositionIndex + a) * N + i];
            g.log_scale_[a] = p[(kLogScaleIndex + a) * N + i];
            g.rotation_[a] = p[(kRotationIndex + a) * N + i];
            for (int k = 0; k < 16; ++k) g.sh_[k][a] = p[(kShIndex + a * 16 + k) * N + i];
        }
        g.opacity_logit_ = p[kOpacityIndex * N + i];
    }
    return out;
}

std::vector<float> PackGaussians(const std::vector<Gaussian>& gaussians) {
    const size_t N = gaussians.size();
    std::vector<float> p(N * kMaxParamCount);
    for (size_t i = 0; i < N; ++i) {
        const Gaussian& g = gaussians[i];
        for (int a = 0; a < 3; ++a) {
            p[(kPositionIndex + a) * N + i] = g.position_[a];
            p[(kLogScaleIndex + a) * N + i] = g.log_scale_[a];
            p[(kRotationIndex + a) * N + i] = g.rotation_[a];
            for (int k = 0; k < 16; ++k) p[(kShIndex + a * 16 + k) * N + i] = g.sh_[k][a];
        }
        p[kOpacityIndex * N + i] = g.opacity_logit_;
    }
    return p;
}

bool WriteGaussiansPly(const std::string& path, const std::vector<Gaussian>& gaussians) {
    std::ofstream file(path, std::ios::binary);
    if (!file) return false;
    file << "ply\nformat binary_little_endian 1.0\nelement vertex " << gaussians.size() << "\n";
    for (const char* name : {"x", "y", "z", "nx", "ny", "nz"}) file << "property float " << name << "\n";
    for (int i = 0; i < 3; ++i) file << "property float f_dc_" << i << "\n";
    for (int i = 0; i < 3 * kRest; ++i) file << "property float f_rest_" << i << "\n";
    file << "property float opacity\n";
    for (int i = 0; i < 3; ++i) file << "property float scale_" << i << "\n";
    for (int i = 0; i < 4; ++i) file << "property float rot_" << i << "\n";
    file << "end_header\n";
    std::vector<float> row(kRowFloats);
    for (const Gaussian& g : gaussians) {
        int n = 0;
        for (int a = 0; a < 3; ++a) row[n++] = g.position_[a];
        for (int a = 0; a < 3; ++a) row[n++] = 0.0f;
        for (int c = 0; c < 3; ++c) row[n++] = g.sh_[0][c];
        for (int c = 0; c < 3; ++c)
            for (int k = 1; k <= kRest; ++k) row[n++] = g.sh_[k][c];
        row[n++] = g.opacity_logit_;
        for (int a = 0; a < 3; ++a) row[n++] = g.log_scale_[a];
        float q[4];
        ToQuaternion(g.rotation_, q);
        for (int a = 0; a < 4; ++a) row[n++] = q[a];
        file.write(reinterpret_cast<const char*>(row.data()), sizeof(float) * row.size());
    }
    return static_cast<bool>(file);
}

bool ReadGaussiansPly(const std::string& path, std::vector<Gaussian>& gaussians) {
    std::ifstream file(path, std::ios::binary);
    std::string line;
    if (!file || !std::getline(file, line) || (line != "ply" && line != "ply\r")) return false;
    bool binary = false, complete = false, vertex = false;
    int64_t count = -1;
    std::vector<std::string> props;
    while (std::getline(file, line)) {
        std::istringstream s(line);
        std::string token;
        s >> token;
        if (token == "end_header") {
            complete = true;
            break;
        }
        if (token == "format") {
            std::string format, version;
            s >> format >> version;
            binary = format == "binary_little_endian" && version == "1.0";
        } else if (token == "element") {
            std::string element;
            int64_t elements = -1;
            s >> element >> elements;
            if (!s || elements < 0 || (count < 0 && element != "vertex") || (element == "vertex" && count >= 0))
                return false;
            vertex = element == "vertex";
            if (vertex) count = elements;
        } else if (token == "property" && vertex) {
            std::string type, name;
            s >> type >> name;
            if (!s || (type != "float" && type != "float32") ||
                std::find(props.begin(), props.end(), name) != props.end())
                return false;
            props.push_back(name);
        }
    }
    if (!binary || !complete || count <= 0 || count > std::numeric_limits<int>::max()) return false;
    std::vector<std::string> names = {"x", "y", "z", "opacity", "scale_0", "scale_1", "scale_2",
                                      "rot_0", "rot_1", "rot_2", "rot_3"};
    for (int c = 0; c < 3; ++c) names.push_back("f_dc_" + std::to_string(c));
    for (int j = 0; j < 3 * kRest; ++j) names.push_back("f_rest_" + std::to_string(j));
    std::vector<size_t> idx;
    for (const std::string& name : names) {
        auto it = std::find(props.begin(), props.end(), name);
        if (it == props.end()) return false;
        idx.push_back(static_cast<size_t>(it - props.begin()));
    }
    const std::streampos begin = file.tellg();
    file.seekg(0, std::ios::end);
    const std::streamoff available = file.tellg() - begin;
    const size_t row_bytes = props.size() * sizeof(float);
    if (available < 0 || static_cast<uint64_t>(available) / row_bytes < static_cast<uint64_t>(count)) return false;
    file.seekg(begin);
    std::vector<Gaussian> loaded(static_cast<size_t>(count));
    std::vector<float> row(props.size());
    for (Gaussian& g : loaded) {
        if (!file.read(reinterpret_cast<char*>(row.data()), static_cast<std::streamsize>(row_bytes))) return false;
        for (size_t k : idx)
            if (!std::isfinite(row[k])) return false;
        for (int a = 0; a < 3; ++a) {
            g.position_[a] = row[idx[a]];
            g.log_scale_[a] = row[idx[4 + a]];
        }
        g.opacity_logit_ = row[idx[3]];
        double qw = row[idx[7]], qx = row[idx[8]], qy = row[idx[9]], qz = row[idx[10]];
        double norm = std::sqrt(qw * qw + qx * qx + qy * qy + qz * qz);
        if (!(norm > 0) || !std::isfinite(norm)) return false;
        FromQuaternion(qw, qx, qy, qz, g.rotation_);
        for (int c = 0; c < 3; ++c) {
            g.sh_[0][c] = row[idx[11 + c]];
            for (int j = 1; j <= kRest; ++j) g.sh_[j][c] = row[idx[14 + c * kRest + j - 1]];
        }
    }
    gaussians.swap(loaded);
    return true;
}

}  // namespace gs_native
