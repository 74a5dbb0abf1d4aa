"""The C-ABI library (librgbdflow.so): loads, exports every entry point include/*.h declares,
and its host-only functions agree with the oracle.  No GPU compute here."""
import ctypes
import glob
import os
import re

import pytest

import rgbdflow as rf
import oracle_binding as ob

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(rgbdflow_\w+)\s*\(", src, flags=re.M):
            syms.add(m.group(1))
    return syms


@pytest.fixture(scope="module")
def lib():
    import build
    build.build()
    return rf.load()


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ["rgbdflow_scene_flow_two_frames", "rgbdflow_scene_flow_multiscale", "rgbdflow_scene_flow_with_init",
              "rgbdflow_scene_flow_single_scale", "rgbdflow_scene_flow_batch", "rgbdflow_server_submit"]:
        assert s in syms


def test_library_exports_every_declared_symbol(lib):
    raw = ctypes.CDLL(rf.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(raw, s)]
    assert not missing, missing
    # and the binding's signature table covers exactly the declared set
    assert set(rf.SIGNATURES) == declared_symbols()


def test_abi_version_and_defaults(lib):
    assert lib.rgbdflow_abi_version() == 1
    p = rf.Params()
    lib.rgbdflow_params_default(ctypes.byref(p))
    q = rf.default_params()
    for name, _ in rf.Params._fields_:
        assert getattr(p, name) == getattr(q, name), name
    # setUpSceneFlowParams (runFlowTwoFrames.cpp:70-79) and sceneFlowParams() (OpticalFlow.h:107-109)
    assert (p.min_width, p.n_outer, p.n_inner, p.n_sor) == (60, 50, 1, 10000)
    assert p.gamma == 1e-5 and p.pyramid_ratio == 0.75 and p.regularization == rf.REG_HPB


@pytest.mark.parametrize("W,H,ratio,mw", [(640, 480, 0.5, 40), (320, 240, 0.5, 20), (160, 120, 0.5, 10),
                                          (640, 480, 0.75, 60), (97, 61, 0.6, 7), (33, 17, 0.5, 2)])
def test_pyramid_levels_match_oracle(lib, W, H, ratio, mw):
    import numpy as np
    levels = rf.pyramid_levels(W, H, ratio, mw)
    img = np.zeros((H, W))
    pyr = ob.build_pyramid(img, ratio, mw)
    assert levels == [(x.shape[1], x.shape[0]) for x in pyr]


def test_batch_device_bytes_and_validation(lib):
    prm = rf.benchmark_params(640)
    one = rf.batch_device_bytes([(640, 480)], prm)
    two = rf.batch_device_bytes([(640, 480), (640, 480)], prm)
    assert 50e6 < one < 200e6 and two > 1.9 * one
    warm = rf.batch_device_bytes([(640, 480)], prm, warm=[1])
    assert warm < one
    bad = rf.default_params()  # HPB regularisation is not built
    with pytest.raises(rf.RgbdFlowError) as e:
        rf.batch_device_bytes([(640, 480)], bad)
    assert e.value.code == -2


def test_no_device_is_reported_not_faked(lib):
    """Without a CUDA device the library refuses to compute (there is no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert lib.rgbdflow_ctx_create(0, 0, ctypes.byref(h)) == -6
