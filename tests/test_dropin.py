"""Drop-in use through the reference's own, unchanged Python binding (CPU part).

The reference binding (bindings/python/rednoise/__init__.py of the reference tree,
found through oracle.reference_dir(): $RN_REFERENCE_DIR or the tree the oracle was
built from) is imported as it is, with REDNOISE_LIBRARY pointing at this
repository's librednoise_b200.so. Its ctypes declarations (_configure_signatures)
bind every function of the reference C ABI, so loading proves the exports and
their argument lists; scene loading, the triangle count and the version string run
on the host. Rendering needs a GPU: without one the library reports failure and the
binding raises, as it does for any failed rn_render. The GPU half (the reference's
examples/c_consumer.c compiled against include/rednoise/rednoise.h) is
tests/test_dropin_gpu.py. Skipped where the reference tree is absent.
"""
import importlib.util
import os
import sys

import pytest
import torch

import oracle
from rednoise_b200 import _native

REF = oracle.reference_dir()
pytestmark = pytest.mark.skipif(REF is None, reason="reference tree absent")


@pytest.fixture()
def binding(monkeypatch):
    monkeypatch.setenv("REDNOISE_LIBRARY", os.path.abspath(_native.LIB_PATH))
    path = os.path.join(REF, "bindings", "python", "rednoise", "__init__.py")
    spec = importlib.util.spec_from_file_location("rednoise_reference_binding", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    yield mod
    sys.modules.pop("rednoise_reference_binding", None)


def test_reference_binding_drives_this_library(binding):
    lib = binding._load_library()
    assert os.path.samefile(lib._name, _native.LIB_PATH)
    assert binding.version() == "0.1.2"
    scene = binding.Scene.load_obj(os.path.join(REF, "assets", "cornell-box.obj"))
    try:
        assert scene.triangle_count == 32
        if torch.cuda.is_available():
            img = scene.render("pathtraced", 64, 48, 4.0, 4)
            assert img.size == (64, 48) and len(img.rgba) == 64 * 48 * 4
        else:
            with pytest.raises(RuntimeError, match="rn_render failed"):
                scene.render("pathtraced", 64, 48, 4.0, 4)
    finally:
        scene.close()
    with pytest.raises(FileNotFoundError):
        binding.Scene.load_obj(os.path.join(REF, "assets", "no-such-file.obj"))
