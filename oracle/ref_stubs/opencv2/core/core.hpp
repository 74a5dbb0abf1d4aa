/* Stand-in: the reference code compiled here names cv::Mat in declarations, and the 2-D
 * optical-flow sources define helpers (a Hessian of cv::Mat, cv::Mat_ parameters that stay empty)
 * that the 2-D flow path never calls.  These types only let that code compile; none of it runs. */
#pragma once
namespace cv {
template <class T, int N> struct Vec {
    T val[N];
    T& operator[](int i) { return val[i]; }
    const T& operator[](int i) const { return val[i]; }
};
typedef Vec<float, 2> Vec2f;
typedef Vec<float, 3> Vec3f;
typedef Vec<float, 4> Vec4f;
typedef Vec<unsigned char, 3> Vec3b;
template <class T> struct DataType { enum { type = 0 }; };
struct Scalar {
    Scalar(double = 0, double = 0, double = 0, double = 0) {}
};
class Mat {
  public:
    int rows = 0, cols = 0;
    Mat() {}
    Mat(int, int, int, const Scalar& = Scalar()) {}
    Mat& operator=(const Scalar&) { return *this; }
    template <class T> T& at(int, int)
    {
        static T t;
        return t;
    }
    template <class T> const T& at(int, int) const
    {
        static T t;
        return t;
    }
};
template <class T> struct Mat_ {
    int rows = 0, cols = 0;
    template <class U> U at(int, int) const { return U(); }
};
}  // namespace cv
