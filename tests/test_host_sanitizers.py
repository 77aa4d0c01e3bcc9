"""The host preprocessing and writers of the library built alone under
AddressSanitizer / UBSan and under ThreadSanitizer (tests/host_check): mesh
generators, the BVH build with its threaded top levels and the flatten
(Src/bvh.cpp, Src/meshmapping.cpp:62-125), the host surface-area tree, the
scene upload's node layout, the sample table and the image writers, on a
seeded random mesh large enough for every threaded path (300k triangles: the
BVH build's chunked passes start at 2^18)."""
import os
import subprocess

import pytest

from fornos_b200 import build as fk_build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SOURCES = ["fk_mesh.cpp", "fk_bvh.cpp", "fk_tree.cpp", "fk_layout.cpp", "fk_image.cpp"]


@pytest.mark.parametrize("sanitizer,seed", [("address,undefined", 3), ("thread", 4)])
def test_host_code_under_sanitizers(tmp_path, sanitizer, seed):
    exe = str(tmp_path / "host_check")
    p = subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-pthread", "-fno-omit-frame-pointer",
                        "-fsanitize=" + sanitizer, "-I" + os.path.join(fk_build.CUDA, "include"),
                        os.path.join(ROOT, "tests", "host_check", "host_check.cpp")] +
                       [os.path.join(ROOT, "fornos_b200", "csrc", s) for s in SOURCES] + ["-lz", "-o", exe],
                       capture_output=True, text=True)
    if p.returncode != 0:
        pytest.skip("no %s build: %s" % (sanitizer, p.stderr.strip().splitlines()[-1:]))
    r = subprocess.run([exe, str(seed), "300000", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-1000:] + r.stderr[-2000:]
    assert "runtime error" not in r.stderr and "WARNING" not in r.stderr and "ERROR" not in r.stderr, \
        r.stderr[-3000:]
