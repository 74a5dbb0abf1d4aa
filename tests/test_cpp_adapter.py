"""The C++ adapter (include/rgbdflow.hpp): the reference's call shapes over the C ABI.

tests/cpp/adapter_check.cpp is compiled with g++ against the library and driven like a caller
of the reference: without a device it checks the sceneFlowParams mapping and that errors are
exceptions carrying the status code; on a B200 its flows through
runFlowTwoFramesSceneFlowExperiments, sceneFlowMultiscale and sceneFlowWithInit must equal
(bit for bit) the same solves through the C ABI directly.
"""
import os
import subprocess

import numpy as np
import pytest

import build as rfbuild
import oracle_binding as ob
import rgbdflow as rf
import synthetic as syn

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def adapter_bin(tmp_path_factory):
    lib = rfbuild.build()
    out = str(tmp_path_factory.mktemp("adapter") / "adapter_check")
    libdir = os.path.dirname(lib)
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(HERE, "cpp", "adapter_check.cpp"), "-o", out, "-L" + libdir, "-lrgbdflow",
                    "-Wl,-rpath," + libdir], check=True)
    return out


def test_adapter_without_device(adapter_bin):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("checks the no-device error path")
    except ImportError:
        pass
    r = subprocess.run([adapter_bin, "cpu"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_adapter_matches_c_abi(adapter_bin, ctx, tmp_path):
    p = syn.make_config_pair("320x240", seed=23)
    W, H = p["W"], p["H"]
    c = p["cam"]
    sig = ob.depth_sigma(p["depth1"]).astype(np.float32)
    est = p["gt"].astype(np.float32)
    np.array([W, H, c.f, c.cx, c.cy, 0.5], np.float64).tofile(tmp_path / "meta.bin")
    p["bgr1"].tofile(tmp_path / "bgr1.bin")
    p["bgr2"].tofile(tmp_path / "bgr2.bin")
    p["depth1"].astype(np.float32).tofile(tmp_path / "depth1.bin")
    p["depth2"].astype(np.float32).tofile(tmp_path / "depth2.bin")
    sig.tofile(tmp_path / "sigma1.bin")
    est.tofile(tmp_path / "est.bin")
    r = subprocess.run([adapter_bin, "gpu", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

    cam = rf.CameraParams.make(W, H, c.f, c.cx, c.cy)
    prm = rf.benchmark_params(W)
    two = ctx.scene_flow_two_frames(cam, p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm, stats=False)
    got = np.fromfile(tmp_path / "flow_two_frames.bin", np.float32).reshape(H, W, 3)
    np.testing.assert_array_equal(got, two)

    im1, im2 = p["bgr1"] / 255.0, p["bgr2"] / 255.0
    u, v, w, _ = ctx.scene_flow_multiscale(cam, im1, p["depth1"], im2, p["depth2"], sig, prm)
    got = np.fromfile(tmp_path / "flow_multiscale.bin", np.float64).reshape(H, W, 3)
    np.testing.assert_array_equal(got, np.stack([u, v, w], -1))

    u, v, w, _ = ctx.scene_flow_with_init(cam, im1, p["depth1"], im2, p["depth2"], sig, prm,
                                          est[..., 0], est[..., 1], est[..., 2])
    got = np.fromfile(tmp_path / "flow_with_init.bin", np.float64).reshape(H, W, 3)
    np.testing.assert_array_equal(got, np.stack([u, v, w], -1))
