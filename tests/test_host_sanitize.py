"""Host code under sanitizers: tests/host_sanitize.cpp built with the loader and
BVH builder (rednoise_b200/csrc/host_scene.cpp) under AddressSanitizer +
UndefinedBehaviorSanitizer (float-cast-overflow included), and under
ThreadSanitizer for the threaded build. CPU only."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = [os.path.join(ROOT, "tests", "host_sanitize.cpp"), os.path.join(ROOT, "rednoise_b200", "csrc", "host_scene.cpp")]
FLAGS = {
    "address,undefined": ["-fsanitize=address,undefined,float-cast-overflow", "-fno-sanitize-recover=all"],
    "thread": ["-fsanitize=thread"],
}


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
@pytest.mark.parametrize("kind", sorted(FLAGS))
def test_host_code_under_sanitizers(tmp_path, kind):
    exe = str(tmp_path / "host_check")
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-fno-omit-frame-pointer", *FLAGS[kind],
           "-I" + os.path.join(ROOT, "rednoise_b200", "csrc"), "-I" + os.path.join(ROOT, "include"),
           *SRC, "-o", exe, "-pthread"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0", TSAN_OPTIONS="halt_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "host checks passed" in r.stdout
