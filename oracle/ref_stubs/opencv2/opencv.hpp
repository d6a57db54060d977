// TEST INFRASTRUCTURE -- stand-in for the few OpenCV names the reference's stereo_mapper.cpp
// uses, so that file compiles unmodified on a host without OpenCV (oracle/build_ref.py, CPU
// fusion variant).  Written for this purpose; not OpenCV's code.  cv::Mat is a reference-
// counted dense matrix (assignment shares the data, clone() copies, as in OpenCV);
// cv::cuda::GpuMat keeps its elements in HOST memory here, so the harness can hand the CPU
// fusion path the maps the GPU stages would have produced; the HighGUI calls do nothing.
#pragma once
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#define CV_8U 0
#define CV_32S 4
#define CV_32F 5
#define CV_64F 6
#define CV_MINMAX 32

typedef unsigned char uchar;   // global, as OpenCV declares it

namespace cv {

using ::uchar;

inline size_t elem_size(int type) { return type == CV_8U ? 1 : type == CV_64F ? 8 : 4; }

template <class T> struct Scalar_ {
    T val[4] = {};
    Scalar_() = default;
    Scalar_(T v0) { val[0] = v0; }
};
typedef Scalar_<double> Scalar;

struct Point {
    int x = 0, y = 0;
    Point() = default;
    Point(int x_, int y_) : x(x_), y(y_) {}
};

struct Vec3b {
    uchar v[3] = {};
    uchar& operator[](int i) { return v[i]; }
    uchar operator[](int i) const { return v[i]; }
};

enum { COLORMAP_RAINBOW = 4 };

class Mat {
public:
    int rows = 0, cols = 0;
    size_t step = 0;          // bytes per row
    unsigned char* data = nullptr;

    Mat() = default;
    Mat(int r, int c, int type) { create(r, c, type); }

    void create(int r, int c, int type) {
        rows = r;
        cols = c;
        type_ = type;
        step = (size_t)c * elem_size(type);
        buf_ = std::make_shared<std::vector<unsigned char>>((size_t)r * step);
        data = buf_->data();
    }
    int type() const { return type_; }

    template <class T> T& at(int r, int c) { return reinterpret_cast<T*>(data + (size_t)r * step)[c]; }
    template <class T> const T& at(int r, int c) const {
        return reinterpret_cast<const T*>(data + (size_t)r * step)[c];
    }

    Mat clone() const {
        Mat m(rows, cols, type_);
        if (data) std::memcpy(m.data, data, (size_t)rows * step);
        return m;
    }
    Mat& setTo(double v) {
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c) set_(r, c, v);
        return *this;
    }
    template <class T> Mat& setTo(const Scalar_<T>& s) { return setTo((double)s.val[0]); }

    void convertTo(Mat& out, int type) const {
        Mat m(rows, cols, type);
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c) m.set_(r, c, get_(r, c));
        out = m;
    }
    Mat t() const {
        Mat m(cols, rows, type_);
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c) m.set_(c, r, get_(r, c));
        return m;
    }
    Mat inv() const {   // 3x3, by the adjugate
        Mat m(3, 3, CV_64F);
        const double a = get_(0, 0), b = get_(0, 1), c = get_(0, 2), d = get_(1, 0), e = get_(1, 1),
                     f = get_(1, 2), g = get_(2, 0), h = get_(2, 1), i = get_(2, 2);
        const double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
        const double adj[9] = {e * i - f * h, c * h - b * i, b * f - c * e, f * g - d * i, a * i - c * g,
                               c * d - a * f, d * h - e * g, b * g - a * h, a * e - b * d};
        for (int k = 0; k < 9; ++k) m.set_(k / 3, k % 3, adj[k] / det);
        return m;
    }

    friend Mat operator*(const Mat& a, const Mat& b) {
        Mat m(a.rows, b.cols, CV_64F);
        for (int r = 0; r < a.rows; ++r)
            for (int c = 0; c < b.cols; ++c) {
                double s = 0.0;
                for (int k = 0; k < a.cols; ++k) s += a.get_(r, k) * b.get_(k, c);
                m.set_(r, c, s);
            }
        return m;
    }
    friend Mat operator-(const Mat& a, const Mat& b) {
        Mat m(a.rows, a.cols, a.type_);
        for (int r = 0; r < a.rows; ++r)
            for (int c = 0; c < a.cols; ++c) m.set_(r, c, a.get_(r, c) - b.get_(r, c));
        return m;
    }
    friend Mat operator*(const Mat& a, double s) {
        Mat m(a.rows, a.cols, a.type_);
        for (int r = 0; r < a.rows; ++r)
            for (int c = 0; c < a.cols; ++c) m.set_(r, c, a.get_(r, c) * s);
        return m;
    }
    friend Mat operator/(const Mat& a, double s) {
        Mat m(a.rows, a.cols, a.type_);
        for (int r = 0; r < a.rows; ++r)
            for (int c = 0; c < a.cols; ++c) m.set_(r, c, a.get_(r, c) / s);
        return m;
    }

private:
    int type_ = CV_32F;
    std::shared_ptr<std::vector<unsigned char>> buf_;

    double get_(int r, int c) const {
        switch (type_) {
            case CV_8U: return at<uchar>(r, c);
            case CV_32S: return at<int32_t>(r, c);
            case CV_64F: return at<double>(r, c);
            default: return at<float>(r, c);
        }
    }
    void set_(int r, int c, double v) {
        switch (type_) {
            case CV_8U: at<uchar>(r, c) = (uchar)v; break;
            case CV_32S: at<int32_t>(r, c) = (int32_t)v; break;
            case CV_64F: at<double>(r, c) = v; break;
            default: at<float>(r, c) = (float)v; break;
        }
    }
};

namespace cuda {
// Host-backed stand-in for a device matrix: `data` and `step` describe host memory.
class GpuMat {
public:
    int rows = 0, cols = 0;
    size_t step = 0;
    unsigned char* data = nullptr;

    GpuMat() = default;
    GpuMat(int r, int c, int type) : rows(r), cols(c), type_(type) {
        step = (size_t)c * elem_size(type);
        buf_.assign((size_t)r * step, 0);
        data = buf_.data();
    }
    template <class T> GpuMat& setTo(const Scalar_<T>& s) {
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c) {
                unsigned char* p = data + (size_t)r * step + (size_t)c * elem_size(type_);
                if (type_ == CV_32F) *reinterpret_cast<float*>(p) = (float)s.val[0];
                else if (type_ == CV_32S) *reinterpret_cast<int32_t*>(p) = (int32_t)s.val[0];
                else if (type_ == CV_64F) *reinterpret_cast<double*>(p) = (double)s.val[0];
                else *p = (unsigned char)s.val[0];
            }
        return *this;
    }
    void upload(const Mat& m) {
        if (rows != m.rows || cols != m.cols || type_ != m.type()) *this = GpuMat(m.rows, m.cols, m.type());
        for (int r = 0; r < rows; ++r) std::memcpy(data + (size_t)r * step, m.data + (size_t)r * m.step, step);
    }
    void download(Mat& m) const {
        Mat out(rows, cols, type_);
        for (int r = 0; r < rows; ++r) std::memcpy(out.data + (size_t)r * out.step, data + (size_t)r * step, step);
        m = out;
    }

private:
    int type_ = CV_32F;
    std::vector<unsigned char> buf_;
};
}  // namespace cuda

// HighGUI and display helpers: no display here.
inline void normalize(const Mat&, Mat&, double, double, int, int) {}
inline void applyColorMap(const Mat&, Mat&, int) {}
inline void imshow(const std::string&, const Mat&) {}
inline int waitKey(int = 0) { return -1; }
inline void circle(Mat&, Point, int, const Scalar&) {}

}  // namespace cv
