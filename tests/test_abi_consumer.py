"""include/fornos_gpu.h from a compiled program, as the reference's C++
solvers would bind it (Src/compute.h:37-87, Src/meshmapping.h:42-75 are the
interfaces it replaces).

tests/abi_consumer/consumer.c is compiled as C11 and as C++17 with warnings
as errors, against the header alone, with static assertions (generated here)
that every struct the ctypes binding (fornos_b200/_lib.py) mirrors has the
same size and field offsets; the program links the library and
* prints the layouts it sees (compared with ctypes);
* runs host calls through the header (mesh, vertex normals, BVH build and
  flatten, sample table) on a generated heightfield, whose arrays must equal
  the ctypes path's byte for byte;
* on the GPU, runs fk_bake through the header, whose every output must equal
  fk_bake through ctypes bit for bit.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from fornos_b200 import _lib as L
from fornos_b200 import api
from fornos_b200.workloads import MeshArrays
from tests import cases
from tests.cases import same_bits

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "abi_consumer", "consumer.c")
OUT = os.path.join(ROOT, "tests", ".out")

# header struct -> ctypes mirror
MIRRORS = {
    "fk_tuning": L.Tuning, "fk_mesh_desc": L.MeshDesc, "fk_scene_info": L.SceneInfo,
    "fk_sample_params": L.SampleParams, "fk_solver_params": L.SolverParams, "fk_batch_job": L.BatchJob,
    "fk_bake_sampler": L.BakeSampler, "fk_bake_desc": L.BakeDesc, "fk_bake_out": L.BakeOut,
    "fk_export_params": L.ExportParams, "fk_run_solver": L.RunSolver, "fk_run_params": L.RunParams,
    "fk_adam": L.Adam, "fk_denoise_params": L.DenoiseParams, "fk_denoise_stats": L.DenoiseStats,
}


def _asserts_header():
    lines = ["#include <stddef.h>", "#ifdef __cplusplus", "#define FK_ASSERT(c, m) static_assert(c, m)", "#else",
             "#define FK_ASSERT(c, m) _Static_assert(c, m)", "#endif"]
    for name, cls in MIRRORS.items():
        lines.append('FK_ASSERT(sizeof(%s) == %d, "%s size");' % (name, ctypes.sizeof(cls), name))
        for f, _ in cls._fields_:
            lines.append('FK_ASSERT(offsetof(%s, %s) == %d, "%s.%s offset");' % (name, f, getattr(cls, f).offset,
                                                                                  name, f))
    os.makedirs(OUT, exist_ok=True)
    path = os.path.join(OUT, "abi_layout_asserts.h")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return path


def _build(lang):
    asserts = _asserts_header()
    exe = os.path.join(OUT, "abi_consumer_" + lang)
    if lang == "c":
        cmd = ["gcc", "-std=c11", "-x", "c"]
    else:
        cmd = ["g++", "-std=c++17", "-x", "c++"]
    cmd += ["-Wall", "-Wextra", "-Werror", "-pedantic", "-O1", "-I", os.path.join(ROOT, "include"),
            '-DFK_LAYOUT_ASSERTS="%s"' % asserts, SRC, "-x", "none", L.LIB_PATH,
            "-Wl,-rpath," + os.path.dirname(L.LIB_PATH), "-o", exe]
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stdout + p.stderr
    return exe


@pytest.fixture(scope="module", params=["c", "cxx"])
def consumer(request, lib):
    return _build(request.param)


def test_header_layouts_match_the_ctypes_binding(consumer):
    p = subprocess.run([consumer, "layout"], capture_output=True, text=True, check=True)
    seen = {}
    for line in p.stdout.splitlines():
        name, *vals = line.split()
        seen[name] = [int(v) for v in vals]
    for name, cls in MIRRORS.items():
        want = [ctypes.sizeof(cls)] + [getattr(cls, f).offset for f, _ in cls._fields_]
        assert seen[name] == want, name


def _heightfield(q=24):
    j, i = np.meshgrid(np.arange(q + 1), np.arange(q + 1), indexing="ij")
    i, j = i.ravel(), j.ravel()
    pos = np.zeros((len(i), 3), np.float32)  # binary32 quotients, as the program computes them
    pos[:, 0] = np.float32(i) / np.float32(q)
    pos[:, 1] = np.float32(j) / np.float32(q)
    pos[:, 2] = np.float32((7 * i + 13 * j) % 11) / np.float32(100)
    v = np.arange(len(pos), dtype=np.uint32)
    vtx = np.stack([v, v, np.zeros_like(v)], -1)
    tri = []
    for jj in range(q):
        for ii in range(q):
            a = jj * (q + 1) + ii
            b, c = a + 1, a + q + 1
            tri += [(a, b, c + 1), (a, c + 1, c)]
    return MeshArrays(pos, pos[:, :2], np.array([[0, 0, 1]], np.float32), vtx, np.array(tri, np.uint32))


def test_host_calls_through_the_header(consumer):
    path = consumer + ".host.bin"
    subprocess.run([consumer, "host", path], check=True)
    raw = open(path, "rb").read()
    nn, nc = np.frombuffer(raw[:8], np.uint32)
    off = 8
    nodes = np.frombuffer(raw[off:off + 36 * nn], api.NODE_DTYPE)
    off += 36 * nn
    p4 = np.frombuffer(raw[off:off + 16 * nc], np.float32).reshape(-1, 4)
    off += 16 * nc
    n4 = np.frombuffer(raw[off:off + 16 * nc], np.float32).reshape(-1, 4)
    off += 16 * nc
    smp = np.frombuffer(raw[off:], np.float32).reshape(-1, 4)
    m = api.Mesh(_heightfield())
    m.compute_vertex_normals()
    e_nodes, e_p4, e_n4 = api.BVH.create_binary(m, 8, 8192).flatten(m)
    assert nodes.tobytes() == e_nodes.tobytes()
    assert same_bits(p4, e_p4) and same_bits(n4, e_n4)
    assert same_bits(smp, api.samples_cosine(32, 16, 5))


@pytest.mark.gpu
def test_fk_bake_through_the_header(consumer, ctx, oracle):
    c = cases.plane()
    ref = oracle.raster(c.lo, 64, 64, 0, c.dirs)
    pix8, pixt, idx = cases.pix8(ref), cases.pixt12(ref), ref["indices"]
    n = len(idx)
    src = consumer + ".bake_in.bin"
    with open(src, "wb") as fh:
        fh.write(np.array([len(c.nodes), len(c.pos4), 64, 64, n], np.uint32).tobytes())
        for a in (c.nodes, c.pos4, c.nrm4, pix8, pixt, idx):
            fh.write(np.ascontiguousarray(a).tobytes())
    dst = consumer + ".bake_out.bin"
    p = subprocess.run([consumer, "bake", src, dst], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    raw = np.frombuffer(open(dst, "rb").read(), np.uint8)
    widths = (("coords4", 16, np.float32, 4), ("tidx", 4, np.uint32, 1), ("height", 4, np.float32, 1),
              ("position3", 12, np.float32, 3), ("normals3", 12, np.float32, 3), ("ao", 4, np.float32, 1),
              ("bent_normals3", 12, np.float32, 3), ("thickness", 4, np.float32, 1))
    got, off = {}, 0
    for name, w, dt, k in widths:
        got[name] = raw[off:off + w * n].view(dt).reshape((n, k) if k > 1 else n)
        off += w * n
    want = {name: np.zeros((n, k) if k > 1 else n, dt) for name, w, dt, k in widths}
    smp = dict(sample_count=64, min_distance=0.001, max_distance=0.3, seed=7)
    api.bake(ctx, c.nodes, c.pos4, c.nrm4, 64, 64, pix8, pixt, idx, want, height_map=True, position_map=True,
             normals_map=True, ao=smp, bent_normals=dict(smp, tangent_space=True), thickness=smp)
    for name, _, _, _ in widths:
        assert same_bits(got[name], want[name]) if want[name].dtype == np.float32 else \
            np.array_equal(got[name], want[name]), name
    assert (want["tidx"] != api.MISS).mean() > 0.5
