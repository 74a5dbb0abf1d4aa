/* Stand-in for the reference's Qt/OpenCV image-file IO header: file IO is not built, so
 * loading and saving report failure. */
#ifndef _ImageIO_h
#define _ImageIO_h
class ImageIO
{
public:
    enum ImageType { standard, derivative, normalized };
    template <class T>
    static bool loadImage(const char*, T*&, int&, int&, int&) { return false; }
    template <class T>
    static bool saveImage(const char*, const T*, int, int, int, ImageType = standard) { return false; }
};
#endif
