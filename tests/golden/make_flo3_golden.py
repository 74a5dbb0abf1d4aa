"""Writes tests/golden/flow_3x2.flo3 and tests/golden/flow_3x2.flo.

flow_3x2.flo3 is a 3 x 2 scene flow in the .flo3 format, written with struct from the format's
definition in readSceneFlow / writeSceneFlow (src/sceneFlowIO.cpp):
  8-byte magic number 237 159 43 26 202 94 218 68 (line 18),
  int32 width, int32 height (lines 28, 53-55),
  width * height (u, v, w) float32 triples, row by row from the top (lines 32-41, 56-60),
all in the byte order of a little-endian host.  The values include -0.0, a subnormal and the
largest float, so that a reader or writer that is not bit-exact shows.
flow_3x2.flo holds the first two channels (u, v) of the same values in the Middlebury .flo
format of readFlow / writeFlow (src/middleburyFlowIO.cpp): the 4 bytes "PIEH" (lines 15-16, 55),
int32 width, int32 height, then the (u, v) float32 pairs row by row (lines 56-64).

Run: python tests/golden/make_flo3_golden.py
"""
import os
import struct

import numpy as np

MAGIC = bytes([237, 159, 43, 26, 202, 94, 218, 68])
W, H = 3, 2
VALUES = np.array([
    [[0.0, -0.0, 1.5], [-2.25, 3.0e-3, -0.125], [1.0e-40, -1.0e-40, 3.4028235e38]],
    [[12.5, -7.75, 0.0625], [-0.5, 0.5, -1.0e-3], [640.0, -480.0, 2.0]],
], dtype=np.float32)
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "flow_3x2.flo3")
FLO_OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "flow_3x2.flo")


def encode(values):
    h, w, _ = values.shape
    body = b"".join(struct.pack("<fff", *map(float, values[i, j])) for i in range(h) for j in range(w))
    return MAGIC + struct.pack("<ii", w, h) + body


def encode_flo(values):
    h, w, _ = values.shape
    body = b"".join(struct.pack("<ff", *map(float, values[i, j, :2])) for i in range(h) for j in range(w))
    return b"PIEH" + struct.pack("<ii", w, h) + body


if __name__ == "__main__":
    with open(OUT, "wb") as f:
        f.write(encode(VALUES))
    with open(FLO_OUT, "wb") as f:
        f.write(encode_flo(VALUES))
    print(OUT, os.path.getsize(OUT), "bytes;", FLO_OUT, os.path.getsize(FLO_OUT), "bytes")
