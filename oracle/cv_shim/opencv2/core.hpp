// Minimal OpenCV-compatible surface for compiling the reference's CPU
// reference renderer (test/cpu_reference.h) and the headers it pulls in
// (test/test_support.h, src/core/types/{camera,scene}.h) without OpenCV.
//
// TEST INFRASTRUCTURE ONLY (oracle/): only what those headers use is here:
// cv::Mat with 8-bit / 32-bit float / 64-bit float elements and 1-4 channels,
// shared reference-counted storage, at<T>(row, col) / at<T>(i), convertTo with
// a scale, element-wise mul, eye/zeros, the Mat_<float> comma initialiser,
// cv::Size, cv::Scalar, cv::Point, cv::Vec. Semantics follow OpenCV's
// documented behaviour for those calls; the library itself is not used.
#pragma once

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

#define CV_8U 0
#define CV_32F 5
#define CV_64F 6
#define CV_CN_SHIFT 3
#define CV_MAKETYPE(depth, cn) ((depth) + (((cn) - 1) << CV_CN_SHIFT))
#define CV_MAT_DEPTH(t) ((t) & ((1 << CV_CN_SHIFT) - 1))
#define CV_MAT_CN(t) ((((t) >> CV_CN_SHIFT) & 63) + 1)
#define CV_8UC1 CV_MAKETYPE(CV_8U, 1)
#define CV_8UC3 CV_MAKETYPE(CV_8U, 3)
#define CV_32FC1 CV_MAKETYPE(CV_32F, 1)
#define CV_32FC3 CV_MAKETYPE(CV_32F, 3)
#define CV_64FC1 CV_MAKETYPE(CV_64F, 1)
#define CV_64FC3 CV_MAKETYPE(CV_64F, 3)

namespace cv {

typedef unsigned char uchar;

struct Size {
    int width = 0, height = 0;
    Size() = default;
    Size(int w, int h) : width(w), height(h) {}
    bool operator==(const Size& o) const { return width == o.width && height == o.height; }
    bool operator!=(const Size& o) const { return !(*this == o); }
};

struct Point {
    int x = 0, y = 0;
    Point() = default;
    Point(int x_, int y_) : x(x_), y(y_) {}
};

template <typename T, int N>
struct Vec {
    T val[N] = {};
    T& operator[](int i) { return val[i]; }
    const T& operator[](int i) const { return val[i]; }
};
typedef Vec<uchar, 3> Vec3b;
typedef Vec<float, 3> Vec3f;
typedef Vec<double, 3> Vec3d;

struct Scalar {
    double val[4] = {0, 0, 0, 0};
    Scalar() = default;
    Scalar(double v0, double v1 = 0, double v2 = 0, double v3 = 0) : val{v0, v1, v2, v3} {}
    double operator[](int i) const { return val[i]; }
};

inline size_t depth_size(int depth) {
    switch (depth) {
        case CV_8U: return 1;
        case CV_32F: return 4;
        case CV_64F: return 8;
        default: throw std::runtime_error("cv shim: unsupported depth");
    }
}

class Mat {
public:
    int rows = 0, cols = 0;
    uchar* data = nullptr;
    size_t step = 0;  // bytes per row

    Mat() = default;
    Mat(int r, int c, int t) { create(r, c, t); }
    Mat(int r, int c, int t, const Scalar& s) {
        create(r, c, t);
        *this = s;
    }
    Mat(int r, int c, int t, void* external) : rows(r), cols(c), data(static_cast<uchar*>(external)), type_(t) {
        step = static_cast<size_t>(c) * elemSize();
    }

    void create(int r, int c, int t) {
        rows = r;
        cols = c;
        type_ = t;
        step = static_cast<size_t>(c) * elemSize();
        storage_ = std::make_shared<std::vector<uchar>>(static_cast<size_t>(r) * step);
        data = storage_->data();
    }

    int type() const { return type_; }
    int depth() const { return CV_MAT_DEPTH(type_); }
    int channels() const { return CV_MAT_CN(type_); }
    size_t elemSize1() const { return depth_size(depth()); }
    size_t elemSize() const { return elemSize1() * channels(); }
    size_t total() const { return static_cast<size_t>(rows) * cols; }
    bool empty() const { return data == nullptr || total() == 0; }
    Size size() const { return Size(cols, rows); }

    template <typename T> T& at(int r, int c) { return reinterpret_cast<T*>(data + r * step)[c]; }
    template <typename T> const T& at(int r, int c) const {
        return reinterpret_cast<const T*>(data + r * step)[c];
    }
    // single index: element i of a continuous single-row or single-column matrix
    template <typename T> T& at(int i) { return reinterpret_cast<T*>(data)[i]; }
    template <typename T> const T& at(int i) const { return reinterpret_cast<const T*>(data)[i]; }

    // every element's channels set to the scalar's first channels (saturated for 8-bit)
    Mat& operator=(const Scalar& s) {
        const int cn = channels();
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c)
                for (int k = 0; k < cn; ++k) set(r, c, k, s.val[k < 4 ? k : 3]);
        return *this;
    }

    double get(int r, int c, int k) const {
        const uchar* p = data + r * step + (static_cast<size_t>(c) * channels() + k) * elemSize1();
        switch (depth()) {
            case CV_8U: return *p;
            case CV_32F: return *reinterpret_cast<const float*>(p);
            default: return *reinterpret_cast<const double*>(p);
        }
    }
    void set(int r, int c, int k, double v) {
        uchar* p = data + r * step + (static_cast<size_t>(c) * channels() + k) * elemSize1();
        switch (depth()) {
            case CV_8U: {
                double x = v < 0 ? 0 : v > 255 ? 255 : v;
                *p = static_cast<uchar>(static_cast<int>(x + 0.5));  // saturate_cast rounds to nearest
                break;
            }
            case CV_32F: *reinterpret_cast<float*>(p) = static_cast<float>(v); break;
            default: *reinterpret_cast<double*>(p) = v; break;
        }
    }

    // dst = src * alpha + beta in the depth of rtype (channels kept)
    void convertTo(Mat& dst, int rtype, double alpha = 1, double beta = 0) const {
        Mat out(rows, cols, CV_MAKETYPE(CV_MAT_DEPTH(rtype), channels()));
        const int cn = channels();
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c)
                for (int k = 0; k < cn; ++k) {
                    double v = get(r, c, k);
                    out.set(r, c, k, alpha == 1 && beta == 0 ? v : v * alpha + beta);
                }
        dst = out;
    }

    // element-wise product (same type and size)
    Mat mul(const Mat& o) const {
        Mat out(rows, cols, type_);
        const int cn = channels();
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c)
                for (int k = 0; k < cn; ++k) out.set(r, c, k, get(r, c, k) * o.get(r, c, k));
        return out;
    }

    static Mat zeros(int r, int c, int t) { return Mat(r, c, t, Scalar(0, 0, 0, 0)); }
    static Mat eye(int r, int c, int t) {
        Mat m = zeros(r, c, t);
        for (int i = 0; i < r && i < c; ++i) m.set(i, i, 0, 1);
        return m;
    }

private:
    int type_ = 0;
    std::shared_ptr<std::vector<uchar>> storage_;
};

template <typename T> struct MatDepth;
template <> struct MatDepth<uchar> { static constexpr int value = CV_8U; };
template <> struct MatDepth<float> { static constexpr int value = CV_32F; };
template <> struct MatDepth<double> { static constexpr int value = CV_64F; };

template <typename T> class Mat_;

// (Mat_<T>(r, c) << a, b, c, ...): fills the matrix row-major
template <typename T>
struct MatCommaInitializer_ {
    Mat_<T> m;
    int index = 0;
    template <typename U> MatCommaInitializer_& operator,(U v) {
        m.template at<T>(index / m.cols, index % m.cols) = static_cast<T>(v);
        ++index;
        return *this;
    }
    operator Mat() const { return m; }
};

template <typename T>
class Mat_ : public Mat {
public:
    Mat_(int r, int c) : Mat(r, c, MatDepth<T>::value) {}
    template <typename U> MatCommaInitializer_<T> operator<<(U v) const {
        MatCommaInitializer_<T> init{*this, 0};
        init, v;
        return init;
    }
};

}  // namespace cv
