// opencv2/opencv.hpp stand-in (TEST INFRASTRUCTURE ONLY): just enough of
// OpenCV's names for the reference's src/wrappers.cuh to compile where OpenCV
// is absent.  Its PNG recorder (src/wrappers.cuh:323-345) is never called by
// the checkers built with it; every function here does nothing.
#pragma once
#include <cstddef>
#include <string>

#define CV_8UC1 0
#define CV_32FC1 5
#define CV_64FC1 6
#define CV_Assert(expr) ((void)0)

namespace cv {
enum { NORM_MINMAX = 32, COLORMAP_VIRIDIS = 16 };
struct Mat {
    Mat() {}
    Mat(std::size_t, std::size_t, int) {}
    template <typename T>
    T &at(std::size_t, std::size_t)
    {
        static T sink;
        return sink;
    }
    int type() const { return CV_32FC1; }
};
inline void normalize(const Mat &, Mat &, double, double, int, int) {}
inline void applyColorMap(const Mat &, Mat &, int) {}
inline bool imwrite(const std::string &, const Mat &) { return true; }
} // namespace cv
