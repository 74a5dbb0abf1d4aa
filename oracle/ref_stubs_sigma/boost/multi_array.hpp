/* Stand-in: a two-dimensional boost::multi_array (extents, resize, num_elements, element access),
 * the parts the reference's depth-noise model is written with. */
#pragma once
#include <cstddef>
#include <vector>
namespace boost {
struct extent_2d { std::size_t rows, cols; };
struct extent_1d {
    std::size_t rows;
    extent_2d operator[](std::size_t c) const { return extent_2d{rows, c}; }
};
struct extent_gen {
    extent_1d operator[](std::size_t r) const { return extent_1d{r}; }
};
static const extent_gen extents = extent_gen();
template <class T, std::size_t N> class multi_array;
template <class T> class multi_array<T, 2> {
    std::vector<T> v_;
    std::size_t cols_ = 0;

  public:
    multi_array() {}
    explicit multi_array(extent_2d e) : v_(e.rows * e.cols), cols_(e.cols) {}
    void resize(extent_2d e) { v_.assign(e.rows * e.cols, T()); cols_ = e.cols; }
    T* data() { return v_.data(); }
    std::size_t num_elements() const { return v_.size(); }
    T* operator[](std::size_t r) { return v_.data() + r * cols_; }
    const T* operator[](std::size_t r) const { return v_.data() + r * cols_; }
};
}  // namespace boost
