""".flo3 files through the C ABI (rgbdflow_flo3_read / rgbdflow_flo3_write; readSceneFlow /
writeSceneFlow, src/sceneFlowIO.cpp:18-61), host-only: no GPU needed.  The golden file
tests/golden/flow_3x2.flo3 is written by tests/golden/make_flo3_golden.py from the format's
definition with struct, independently of the library."""
import ctypes
import importlib.util
import os

import numpy as np
import pytest

import rgbdflow as rf

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _golden_module():
    spec = importlib.util.spec_from_file_location("make_flo3_golden", os.path.join(GOLDEN_DIR, "make_flo3_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_reads_the_golden_file_bit_for_bit():
    g = _golden_module()
    flow = rf.read_flo3(g.OUT)
    assert flow.shape == (g.H, g.W, 3)
    np.testing.assert_array_equal(_bits(flow), _bits(g.VALUES))


def test_writes_the_golden_bytes(tmp_path):
    g = _golden_module()
    out = tmp_path / "w.flo3"
    rf.write_flo3(str(out), g.VALUES)
    assert out.read_bytes() == open(g.OUT, "rb").read()
    assert out.read_bytes() == g.encode(g.VALUES)


@pytest.mark.parametrize("shape", [(1, 1), (13, 17), (240, 320)])
def test_round_trip(tmp_path, shape):
    rng = np.random.default_rng(shape[0] * 1000 + shape[1])
    flow = rng.normal(scale=5.0, size=shape + (3,)).astype(np.float32)
    flow.flat[::7] = np.float32(-0.0)
    p = tmp_path / "r.flo3"
    rf.write_flo3(str(p), flow)
    assert p.stat().st_size == 16 + flow.size * 4
    np.testing.assert_array_equal(_bits(rf.read_flo3(str(p))), _bits(flow))


def test_bytes_after_the_last_value_are_ignored(tmp_path):
    g = _golden_module()
    p = tmp_path / "t.flo3"
    p.write_bytes(g.encode(g.VALUES) + b"trailing")
    np.testing.assert_array_equal(_bits(rf.read_flo3(str(p))), _bits(g.VALUES))


def _code(fn, *a):
    with pytest.raises(rf.RgbdFlowError) as e:
        fn(*a)
    return e.value.code


def test_errors_keep_the_reference_distinctions(tmp_path):
    g = _golden_module()
    good = g.encode(g.VALUES)
    # a file that cannot be opened (ASSERT_ALWAYS on the stream): IO
    assert _code(rf.read_flo3, str(tmp_path / "missing.flo3")) == -9
    assert _code(rf.write_flo3, str(tmp_path / "no_dir" / "x.flo3"), g.VALUES) == -9
    # a header cut short (runtime_error "can't read metadata"): IO
    p = tmp_path / "short_header.flo3"
    p.write_bytes(good[:12])
    assert _code(rf.read_flo3, str(p)) == -9
    # pixel data cut short (runtime_error "can't read pixel values"): IO
    p = tmp_path / "short_data.flo3"
    p.write_bytes(good[:-4])
    assert _code(rf.read_flo3, str(p)) == -9
    # another magic number (invalid_argument): FORMAT
    p = tmp_path / "magic.flo3"
    p.write_bytes(bytes([good[0] ^ 1]) + good[1:])
    assert _code(rf.read_flo3, str(p)) == -10
    # a size below 1: FORMAT
    p = tmp_path / "zero.flo3"
    p.write_bytes(g.MAGIC + np.array([0, 2], "<i4").tobytes())
    assert _code(rf.read_flo3, str(p)) == -10
    # a flow that is not (H, W, 3): INVALID_ARG
    assert _code(rf.write_flo3, str(tmp_path / "bad.flo3"), np.zeros((4, 4), np.float32)) == -1


def test_read_reports_the_size_and_checks_the_buffer(tmp_path):
    g = _golden_module()
    lib = rf.load()
    W, H = ctypes.c_int(), ctypes.c_int()
    err = ctypes.create_string_buffer(256)
    assert lib.rgbdflow_flo3_read(g.OUT.encode(), None, 0, ctypes.byref(W), ctypes.byref(H), err, len(err)) == 0
    assert (W.value, H.value) == (g.W, g.H)
    small = np.empty(g.W * g.H * 3 - 1, np.float32)
    rc = lib.rgbdflow_flo3_read(g.OUT.encode(), small.ctypes.data, small.size, ctypes.byref(W), ctypes.byref(H),
                                err, len(err))
    assert rc == -1 and b"fewer" in err.value


def test_flow2d_defaults_are_the_demos():
    """rgbdflow_flow2d_params_default (host-only): runFlowTwoFramesCeLiu's iterations
    (src/runFlowTwoFrames.cpp:36-41), the demo's smoothness weight and opticalFlowParams' pyramid."""
    p = rf.flow2d_params()
    assert (p.alpha, p.pyramid_ratio, p.min_width, p.n_outer, p.n_inner, p.n_sor) == (0.02, 0.75, 20, 10, 1, 400)
    assert 2 <= p.sor_ring <= 16


def test_middlebury_flo_golden_both_ways(tmp_path):
    """Middlebury .flo (rgbdflow_flo_read / rgbdflow_flo_write; readFlow / writeFlow,
    src/middleburyFlowIO.cpp): the golden file reads back bit for bit and is rewritten byte for
    byte; its tag reads as the float 202021.25 the reference checks."""
    g = _golden_module()
    data = open(g.FLO_OUT, "rb").read()
    assert np.frombuffer(data[:4], "<f4")[0] == np.float32(202021.25)
    flow = rf.read_flo(g.FLO_OUT)
    assert flow.shape == (g.H, g.W, 2)
    np.testing.assert_array_equal(_bits(flow), _bits(g.VALUES[..., :2]))
    out = tmp_path / "w.flo"
    rf.write_flo(str(out), g.VALUES[..., :2])
    assert out.read_bytes() == data == g.encode_flo(g.VALUES)


def test_middlebury_flo_errors(tmp_path):
    g = _golden_module()
    good = g.encode_flo(g.VALUES)
    assert _code(rf.read_flo, str(tmp_path / "missing.flo")) == -9
    p = tmp_path / "short.flo"
    p.write_bytes(good[:-1])
    assert _code(rf.read_flo, str(p)) == -9
    p = tmp_path / "tag.flo"
    p.write_bytes(b"PIEX" + good[4:])
    assert _code(rf.read_flo, str(p)) == -10
    p = tmp_path / "flo3_as_flo.flo"
    p.write_bytes(g.encode(g.VALUES))
    assert _code(rf.read_flo, str(p)) == -10
    assert _code(rf.write_flo, str(tmp_path / "bad.flo"), g.VALUES) == -1
