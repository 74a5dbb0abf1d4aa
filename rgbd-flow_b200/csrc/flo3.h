// flo3.h — the .flo3 scene-flow file format (host code).
//
// The format of readSceneFlow / writeSceneFlow (src/sceneFlowIO.cpp:18-61), in which the
// reference's demo writes its result (src/main.cpp:126):
//   8 bytes   magic number 237 159 43 26 202 94 218 68 (sceneFlowIO.cpp:18)
//   int32     width
//   int32     height
//   float32   width * height (u, v, w) triples, row by row from the top (sceneFlowIO.cpp:32-41)
// The reference writes host byte order; its platforms are little-endian, and so is this build,
// which reads and writes little-endian only.
// The reference reports each failure differently, and these functions keep the distinctions:
//   - a file that cannot be opened (ASSERT_ALWAYS on the stream) -> RGBDFLOW_ERR_IO;
//   - a header or pixel data cut short (std::runtime_error) -> RGBDFLOW_ERR_IO;
//   - a wrong magic number (std::invalid_argument) -> RGBDFLOW_ERR_FORMAT.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>

#include "../../include/rgbdflow.h"

#if !defined(__BYTE_ORDER__) || __BYTE_ORDER__ != __ORDER_LITTLE_ENDIAN__
#error ".flo3 files are little-endian; this build reads and writes them in host order"
#endif

namespace rgbdflow {

constexpr unsigned char kFlo3Magic[8] = {237, 159, 43, 26, 202, 94, 218, 68};

struct Flo3Error {
    int code;
    std::string msg;
};

struct FileCloser {
    void operator()(FILE* f) const
    {
        if (f) std::fclose(f);
    }
};
using File = std::unique_ptr<FILE, FileCloser>;

inline void flo3_write(const char* path, const float* flow, int W, int H)
{
    if (!path || !flow || W < 1 || H < 1) throw Flo3Error{RGBDFLOW_ERR_INVALID_ARG, "flo3 write: bad arguments"};
    FILE* raw = std::fopen(path, "wb");
    if (!raw) throw Flo3Error{RGBDFLOW_ERR_IO, std::string("can't open ") + path + " for writing"};
    File f(raw);
    const int32_t wh[2] = {W, H};
    if (std::fwrite(kFlo3Magic, 1, 8, f.get()) != 8 || std::fwrite(wh, 4, 2, f.get()) != 2)
        throw Flo3Error{RGBDFLOW_ERR_IO, "can't write metadata for flow image"};
    const size_t n = (size_t)W * H * 3;
    if (std::fwrite(flow, 4, n, f.get()) != n) throw Flo3Error{RGBDFLOW_ERR_IO, "can't write pixel values for flow image"};
    if (std::fclose(f.release()) != 0) throw Flo3Error{RGBDFLOW_ERR_IO, "can't write pixel values for flow image"};
}

inline void flo3_read(const char* path, float* flow, size_t n_floats, int* W, int* H)
{
    if (!path || !W || !H) throw Flo3Error{RGBDFLOW_ERR_INVALID_ARG, "flo3 read: bad arguments"};
    FILE* raw = std::fopen(path, "rb");
    if (!raw) throw Flo3Error{RGBDFLOW_ERR_IO, std::string("can't open ") + path};
    File f(raw);
    unsigned char magic[8];
    int32_t wh[2];
    if (std::fread(magic, 1, 8, f.get()) != 8 || std::fread(wh, 4, 2, f.get()) != 2)
        throw Flo3Error{RGBDFLOW_ERR_IO, "can't read metadata for flow image"};
    if (std::memcmp(magic, kFlo3Magic, 8) != 0)
        throw Flo3Error{RGBDFLOW_ERR_FORMAT, "magic number doesn't match .flo3 format"};
    if (wh[0] < 1 || wh[1] < 1) throw Flo3Error{RGBDFLOW_ERR_FORMAT, "flo3 size below 1"};
    *W = wh[0];
    *H = wh[1];
    if (!flow) return;
    const size_t n = (size_t)wh[0] * wh[1] * 3;
    if (n_floats < n) throw Flo3Error{RGBDFLOW_ERR_INVALID_ARG, "flo3 read: the buffer holds fewer than W*H*3 floats"};
    if (std::fread(flow, 4, n, f.get()) != n) throw Flo3Error{RGBDFLOW_ERR_IO, "can't read pixel values for flow image"};
}

// Middlebury .flo, the format the reference's demo writes 2-D flows in (readFlow / writeFlow,
// src/middleburyFlowIO.cpp:15-65; src/main.cpp:125): the 4 bytes "PIEH" (read back as the float
// 202021.25), int32 width, int32 height, then width * height (u, v) float32 pairs, rows top to
// bottom, little-endian; failures classed as for .flo3.
constexpr unsigned char kFloTag[4] = {'P', 'I', 'E', 'H'};

inline void flo_write(const char* path, const float* flow, int W, int H)
{
    if (!path || !flow || W < 1 || H < 1) throw Flo3Error{RGBDFLOW_ERR_INVALID_ARG, "flo write: bad arguments"};
    FILE* raw = std::fopen(path, "wb");
    if (!raw) throw Flo3Error{RGBDFLOW_ERR_IO, std::string("can't open ") + path + " for writing"};
    File f(raw);
    const int32_t wh[2] = {W, H};
    if (std::fwrite(kFloTag, 1, 4, f.get()) != 4 || std::fwrite(wh, 4, 2, f.get()) != 2)
        throw Flo3Error{RGBDFLOW_ERR_IO, "can't write metadata for flow image"};
    const size_t n = (size_t)W * H * 2;
    if (std::fwrite(flow, 4, n, f.get()) != n) throw Flo3Error{RGBDFLOW_ERR_IO, "can't write pixel values for flow image"};
    if (std::fclose(f.release()) != 0) throw Flo3Error{RGBDFLOW_ERR_IO, "can't write pixel values for flow image"};
}

inline void flo_read(const char* path, float* flow, size_t n_floats, int* W, int* H)
{
    if (!path || !W || !H) throw Flo3Error{RGBDFLOW_ERR_INVALID_ARG, "flo read: bad arguments"};
    FILE* raw = std::fopen(path, "rb");
    if (!raw) throw Flo3Error{RGBDFLOW_ERR_IO, std::string("can't open ") + path};
    File f(raw);
    unsigned char tag[4];
    int32_t wh[2];
    if (std::fread(tag, 1, 4, f.get()) != 4 || std::fread(wh, 4, 2, f.get()) != 2)
        throw Flo3Error{RGBDFLOW_ERR_IO, "can't read metadata for flow image"};
    if (std::memcmp(tag, kFloTag, 4) != 0) throw Flo3Error{RGBDFLOW_ERR_FORMAT, "magic number doesn't match .flo format"};
    if (wh[0] < 1 || wh[1] < 1) throw Flo3Error{RGBDFLOW_ERR_FORMAT, "flo size below 1"};
    *W = wh[0];
    *H = wh[1];
    if (!flow) return;
    const size_t n = (size_t)wh[0] * wh[1] * 2;
    if (n_floats < n) throw Flo3Error{RGBDFLOW_ERR_INVALID_ARG, "flo read: the buffer holds fewer than W*H*2 floats"};
    if (std::fread(flow, 4, n, f.get()) != n) throw Flo3Error{RGBDFLOW_ERR_IO, "can't read pixel values for flow image"};
}

}  // namespace rgbdflow
