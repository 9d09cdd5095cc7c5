"""The main GPU parity suites again, on the bounds-checked build
(librednoise_b200_debug.so, `make -C rednoise_b200/csrc debug`): every
data-dependent index (tree references, queue slots, sort positions, shading
entries, photon deposits) is checked against its buffer, and a failed check makes
the call return an error -- the stand-in for compute-sanitizer's memory checker,
which is not available here. The results must still equal the references'."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SUITES = ["test_trace_gpu.py", "test_refmode_gpu.py", "test_physical_gpu.py", "test_raytraced_gpu.py",
          "test_photon_gpu.py", "test_gi_gpu.py", "test_lbvh_gpu.py", "test_adjoint_gpu.py"]


def test_parity_suites_on_the_bounds_checked_build():
    lib = os.path.join(ROOT, "rednoise_b200", "librednoise_b200_debug.so")
    assert os.path.isfile(lib), "build it with: make -C rednoise_b200/csrc debug"
    env = dict(os.environ, RN_B200_LIBRARY=lib)
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider",
                        *[os.path.join("tests", f) for f in SUITES]],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
