"""The scene upload's host checks and layout (fornos_b200/csrc/fk_layout.cpp,
split over host threads) against a sequential restatement of them
(tests/layout_check/check.cpp): identical device arrays, inner records, leaf
list, depth and coordinate flags for every thread count, and on seeded
mutations of valid trees (skip pointers, corner ranges, box faces) the same
first defect and message.  The node arrays come from the reference's BVH
build (Src/bvh.cpp) restated by the library's host build."""
import os
import re
import subprocess

import numpy as np
import pytest

from tests import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OUT = os.path.join(ROOT, "tests", ".out")


@pytest.fixture(scope="module")
def checker():
    os.makedirs(OUT, exist_ok=True)
    exe = os.path.join(OUT, "layout_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-ffp-contract=off", "-Wall", "-Werror",
                    os.path.join(ROOT, "tests", "layout_check", "check.cpp"),
                    os.path.join(ROOT, "fornos_b200", "csrc", "fk_layout.cpp"), "-o", exe], check=True)
    return exe


def run(checker, nodes, corners, mutations, seed, tag):
    path = os.path.join(OUT, "layout_%s.bin" % tag)
    np.ascontiguousarray(nodes).tofile(path)
    p = subprocess.run([checker, path, str(corners), str(mutations), str(seed)], capture_output=True, text=True)
    counts = dict(re.findall(r"(\w+) (\d+)", p.stdout.splitlines()[-1]))
    assert p.returncode == 0, p.stdout
    assert int(counts["mismatches"]) == 0
    return counts


@pytest.mark.parametrize("name", ["sphere", "plane", "icosphere"])
def test_layout_matches_the_sequential_scan(checker, name):
    c = getattr(cases, name)()
    counts = run(checker, c.nodes, c.pos4.shape[0], 1500, 11, name)
    # the mutations exercise the defects, and leave some trees valid
    assert 500 < int(counts["rejected"]) < 1500


def test_layout_of_a_single_leaf_and_a_large_tree(checker):
    c = cases.plane(hi=384)
    assert c.nodes.shape[0] > 1 << 16  # past the size where the library goes to several threads
    run(checker, c.nodes, c.pos4.shape[0], 20, 5, "large")
    leaf = c.nodes[:1].copy()
    leaf["start"], leaf["end"], leaf["jump"] = 0, 3, 1
    run(checker, leaf, 3, 50, 6, "leaf")


@pytest.mark.parametrize("sanitizer,name,mutations", [("address,undefined", "icosphere", 400),
                                                      ("thread", "large", 10)])
def test_layout_under_sanitizers(checker, sanitizer, name, mutations):
    """The same comparison with the layout built under AddressSanitizer /
    UBSan (reads past the node array on malformed trees) and ThreadSanitizer
    (races between the ranges' threads)."""
    c = cases.icosphere() if name == "icosphere" else cases.plane(hi=384)
    exe = os.path.join(OUT, "layout_check_" + sanitizer.split(",")[0])
    p = subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-pthread", "-fno-omit-frame-pointer",
                        "-fsanitize=" + sanitizer, os.path.join(ROOT, "tests", "layout_check", "check.cpp"),
                        os.path.join(ROOT, "fornos_b200", "csrc", "fk_layout.cpp"), "-o", exe],
                       capture_output=True, text=True)
    if p.returncode != 0:
        pytest.skip("no %s runtime: %s" % (sanitizer, p.stderr.strip().splitlines()[-1:]))
    path = os.path.join(OUT, "layout_san_%s.bin" % name)
    np.ascontiguousarray(c.nodes).tofile(path)
    r = subprocess.run([exe, path, str(c.pos4.shape[0]), str(mutations), "9"], capture_output=True, text=True)
    assert r.returncode == 0 and "ERROR" not in r.stderr and "WARNING" not in r.stderr, r.stderr[-2000:]
    assert "mismatches 0" in r.stdout.splitlines()[-1]
