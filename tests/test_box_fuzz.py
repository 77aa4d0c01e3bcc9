"""The traversal's box tests, fuzzed on the host: tests/box_fuzz/fuzz.cpp
compiles fornos_b200/csrc/fk_device.cuh itself with g++ (the stand-in
cuda_runtime.h maps each IEEE-rounded intrinsic to the same host operation,
no contraction) and checks, on random and adversarial rays and boxes at
scene scales from 1e-3 to 1e6 (origins on faces, flat boxes, direction
components zero, tiny or subnormal, thresholds from 0 to FLT_MAX), that

* box_near, the conservative inner-record test, accepts every box the
  reference's RayAABB (Shaders/ao_step1.comp:43-52) accepts against the same
  threshold, with an entry distance no larger than the reference's, and
* box_hit, the leaf-box test, takes exactly the reference's decision."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "box_fuzz", "fuzz.cpp")
OUT = os.path.join(ROOT, "tests", ".out")


@pytest.fixture(scope="module")
def fuzzer():
    os.makedirs(OUT, exist_ok=True)
    exe = os.path.join(OUT, "box_fuzz")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Werror",
                    "-I", os.path.join(ROOT, "tests", "box_fuzz"), SRC, "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_box_tests_against_the_reference(fuzzer, seed):
    p = subprocess.run([fuzzer, str(seed), "1000000"], capture_output=True, text=True)
    counts = dict(re.findall(r"(\w+) (\d+)", p.stdout.splitlines()[-1]))
    assert p.returncode == 0, p.stdout
    assert int(counts["near_violations"]) == 0 and int(counts["hit_mismatches"]) == 0
    assert int(counts["ref_accepts"]) > 100000  # the cases exercise acceptance, not only rejection
    # with every axis constrained, the margins add few boxes
    assert int(counts["regular_extra"]) < 0.01 * int(counts["regular"])
