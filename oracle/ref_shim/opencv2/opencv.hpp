// Minimal stand-in for the OpenCV surface the reference's route sources use
// (cv::Mat with rows / cols / data / create / clone / ptr / isContinuous /
// empty, imread / imwrite, CV_8U, IMREAD_GRAYSCALE).  Only the checker build
// in oracle/ref_build.py uses it; image files are never read through it.
#pragma once

#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#ifndef CV_8U
#define CV_8U 0
#endif

namespace cv {

enum { IMREAD_GRAYSCALE = 0 };

class Mat {
public:
    int rows = 0;
    int cols = 0;
    unsigned char* data = nullptr;

    Mat() = default;
    Mat(int r, int c, int /*type*/) { create(r, c, CV_8U); }

    void create(int r, int c, int /*type*/) {
        if (storage_ && r * c == rows * cols) {
            rows = r;
            cols = c;
            return;
        }
        storage_ = std::make_shared<std::vector<unsigned char>>(
            static_cast<size_t>(r) * static_cast<size_t>(c));
        rows = r;
        cols = c;
        data = storage_->data();
    }
    Mat clone() const {
        Mat m;
        m.create(rows, cols, CV_8U);
        if (rows * cols > 0) {
            std::memcpy(m.data, data, static_cast<size_t>(rows) * cols);
        }
        return m;
    }
    template <typename T>
    T* ptr(int y) {
        return reinterpret_cast<T*>(data + static_cast<size_t>(y) * cols);
    }
    template <typename T>
    const T* ptr(int y) const {
        return reinterpret_cast<const T*>(data + static_cast<size_t>(y) * cols);
    }
    bool isContinuous() const { return true; }
    bool empty() const { return data == nullptr || rows * cols == 0; }

private:
    std::shared_ptr<std::vector<unsigned char>> storage_;
};

inline Mat imread(const std::string&, int) { return Mat(); }
inline bool imwrite(const std::string&, const Mat&) { return false; }

}  // namespace cv
