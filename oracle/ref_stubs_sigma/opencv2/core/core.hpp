/* Stand-in: the cv::Mat / cv::Mat_ storage the reference's depth-noise model reads and writes
 * (row-major, element access only). */
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>
namespace cv {
class Mat {
  public:
    int rows = 0, cols = 0;
    std::vector<float> f;  // the one element type used here (distanceTransform's CV_32F output)
    template <class T> T& at(int i, int j) { return f[(std::size_t)i * cols + j]; }
    template <class T> const T& at(int i, int j) const { return f[(std::size_t)i * cols + j]; }
};
template <class T> class Mat_ {
  public:
    int rows = 0, cols = 0;
    std::vector<T> d;
    Mat_() {}
    Mat_(int r, int c) : rows(r), cols(c), d((std::size_t)r * c) {}
    T& operator()(int i, int j) { return d[(std::size_t)i * cols + j]; }
    const T& operator()(int i, int j) const { return d[(std::size_t)i * cols + j]; }
};
}  // namespace cv
