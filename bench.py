"""Headline benchmark: plain bake throughput (Mrays/s) on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fornos|reference]
                    [--workload plane2048|sphere512|icosphere4096|plane250|batch|denoise]
                    [--traverse auto|ordered|skip|ordered4] [--schedule auto|static|dynamic]
                    [--tree sah|reference] [--no-denoise] [--no-batch] [--denoise-tex T] [--no-cpu-baseline]

One step = one full plain bake of the workload with every input resident in
HBM: mesh mapping (2 rays / texel), height, position and tangent-space normal
gathers, ambient occlusion + bent normals (one traversal, spp rays / texel,
counted as the reference's two sampling kernels) and thickness (spp rays /
texel).  value = rays of all ranks / max-over-ranks device time.  e2e = the
same bake through fk_bake from pinned host arrays (uploads and result copies
inside the timed region).  Multi-GPU: one process per GPU, each baking its
own seeded replica of the workload (weak scaling, no data-path collective).

The default line also carries fk_run's time from mesh files to image files
(`files_to_images`: the workload written as PLY, all six maps written as PNG /
EXR), the denoised-vs-plain comparison at 4096x4096 (`denoise`) and the
batched-bake comparison over the first 16 jobs of the batch workload
(`batch`); --workload batch measures all 64 batched jobs and --workload
denoise the comparison alone.  With the CPU baseline on, `parity` compares
the timed bake's outputs with the reference's at the CPU run's texels, and
the denoise and batch objects carry the same check of their plain and
batched paths.  --tree reference walks the reference's inner BVH nodes
instead of the surface-area tree built at upload.

--impl reference times the reference's own CPU implementation of the path
(the reference's shaders and host code compiled by oracle/build_ref.py, or
the oracle restatement when that build is absent) on the host cores, on a
strided texel sample of the same workload.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from fornos_b200 import workloads as W  # noqa: E402

WORKLOADS = {
    "plane2048": dict(
        desc="plain bake, all six bakers, 2048x2048: 64x64-quad plane low-poly, 1024x1024-quad heightfield "
             "high-poly (2,097,152 tris, 4-octave value noise + 200 bumps), AO / bent normals / thickness "
             "256 spp, min 0.001, max 0.3",
        gen=lambda seed: W.plane_pair(seed=seed, lo_quads=64, hi_quads=1024, bumps=200),
        tex=2048, spp=256, min_d=0.001, max_d=0.3, bakers=("height", "position", "normals", "ao", "bn", "thick")),
    "sphere512": dict(
        desc="plain bake, 512x512: 32x16 UV-sphere low-poly, 512x256 perturbed UV-sphere high-poly, mapping with "
             "maximum distance 0.1, height, tangent-space normals, AO 64 spp (min 0.001, max 0.5)",
        gen=lambda seed: W.sphere_pair(seed=seed),
        tex=512, spp=64, min_d=0.001, max_d=0.5, map_max=0.1, bakers=("height", "normals", "ao")),
    "icosphere4096": dict(
        desc="plain large bake, 4096x4096: subdivision-3 icosphere low-poly (cube-projection UVs), "
             "subdivision-9 icosphere high-poly (5,242,880 tris, 6-octave gradient noise), AO / bent normals / "
             "thickness 1024 spp, max 0.5",
        gen=lambda seed: W.icosphere_pair(seed=seed),
        tex=4096, spp=1024, min_d=0.001, max_d=0.5, bakers=("ao", "bn", "thick")),
    # profiling case: the plane workload's scene (381 MB, larger than L2) at 250x250 texels, 16 spp, so one
    # hemisphere launch lasts milliseconds under ncu
    "plane250": dict(
        desc="profiling case: the 1024x1024-quad heightfield scene of plane2048 at 250x250 texels, AO / bent "
             "normals / thickness 16 spp, min 0.001, max 0.3",
        gen=lambda seed: W.plane_pair(seed=seed, lo_quads=64, hi_quads=1024, bumps=200),
        tex=250, spp=16, min_d=0.001, max_d=0.3, bakers=("ao", "bn", "thick")),
}
TRAVERSE = {"auto": 0, "ordered": 1, "skip": 2, "ordered4": 3}
SCHEDULE = {"auto": 0, "static": 0x10, "dynamic": 0x20}
# DRAM bytes (read + write) per hemisphere-kernel launch from ncu captures, by workload: plane250, one AO+BN
# trace launch of 968,256 rays (profiles/hemi_trace_kernel_plane250.md); plane2048, the mean of two AO+BN
# chunk launches of 134,217,728 rays each, 4.46 and 2.94 GB (profiles/hemi_trace_traffic_plane2048.md).
NCU_TRAFFIC = {"plane250": 245.5e6, "plane2048": 3.700e9}


def rays_per_texel(wl):
    spp = wl["spp"]
    return 2 + spp * sum(k in wl["bakers"] for k in ("ao", "bn", "thick"))


def parse_tuning(text):
    """'refill=8,top_records=64' -> fk_tuning fields (fk_ctx_set_tuning)."""
    out = {}
    for item in filter(None, text.split(",")):
        k, v = item.split("=")
        out[k.strip()] = int(v)
    return out


def traversals_per_texel(wl):
    """Rays actually traced per texel: AO and bent normals share one traversal."""
    b = wl["bakers"]
    return 2 + wl["spp"] * ((("ao" in b) or ("bn" in b)) + ("thick" in b))


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    def __init__(self, device_index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        nv = self.nv
        names = {
            "hw_slowdown": getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8),
            "sw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
            "hw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
            "sw_power_cap": getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4),
        }
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for k, bit in names.items():
                    if r & bit:
                        self.reasons.add(k)
            except Exception:
                pass
            self._stop.wait(0.1)

    def __enter__(self):
        if self.nv:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self.nv:
            self.t.join()

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons)}


# ---------------------------------------------------------------- setup
class Prepared:
    """Host preprocessing of Src/fornos.cpp:53-157 with the product's host code."""

    def __init__(self, wl, seed):
        from fornos_b200 import api
        t0 = time.perf_counter()
        lo, hi = wl["gen"](seed)
        self.gen_s = time.perf_counter() - t0
        self.lo, self.hi = lo, hi
        t0 = time.perf_counter()
        self.hm = api.Mesh(hi)
        self.hm.compute_vertex_normals()
        self.lm = api.Mesh(lo)
        self.lm.compute_tangent_space()
        self.dm = self.lm.copy()
        self.dm.compute_vertex_normals_aggressive()
        self.prep_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        self.bvh = api.BVH.create_binary(self.hm, 8, 8192)
        self.bvh_s = time.perf_counter() - t0
        self.nodes, self.pos4, self.nrm4 = self.bvh.flatten(self.hm)
        self.triangles = hi.triangle_count


def device_preprocess(ctx, prep):
    """The host preprocessing of Prepared run by the device generators
    (fk_mesh_compute_normals_device / fk_mesh_compute_tangent_space_device)."""
    from fornos_b200 import api
    hm = api.Mesh(prep.hi)
    hm.compute_normals_device(ctx, api.NORMALS_VERTEX)
    lm = api.Mesh(prep.lo)
    lm.compute_tangent_space_device(ctx)
    dm = lm.copy()
    dm.compute_normals_device(ctx, api.NORMALS_WELDED)
    return hm, lm, dm


def write_ply(path, m):
    """A binary little-endian PLY of a MeshArrays mesh with one PLY vertex per
    mesh vertex (x y z nx ny nz s t as floats) and uint triangle lists: the
    layout the reference's PLY reader expects."""
    v = m.vertices.astype(np.int64)
    rec = np.zeros(len(v), dtype=[("p", "<f4", 3), ("n", "<f4", 3), ("t", "<f4", 2)])
    rec["p"] = m.positions[v[:, 0]]
    if len(m.normals):
        rec["n"] = m.normals[np.minimum(v[:, 2], len(m.normals) - 1)]
    if len(m.texcoords):
        rec["t"] = m.texcoords[np.minimum(v[:, 1], len(m.texcoords) - 1)]
    face = np.zeros(m.triangle_count, dtype=[("c", "u1"), ("i", "<u4", 3)])
    face["c"] = 3
    face["i"] = m.triangles
    head = ("ply\nformat binary_little_endian 1.0\nelement vertex %d\nproperty float x\nproperty float y\n"
            "property float z\nproperty float nx\nproperty float ny\nproperty float nz\nproperty float s\n"
            "property float t\nelement face %d\nproperty list uchar uint vertex_indices\nend_header\n"
            % (len(v), m.triangle_count))
    with open(path, "wb") as fh:
        fh.write(head.encode())
        fh.write(rec.tobytes())
        fh.write(face.tobytes())
    return os.path.getsize(path)


def files_to_images(ctx, prep, wl, seed):
    """fk_run (FornosRunner::start + run) on the workload written as PLY files:
    mesh files in, PNG / EXR maps out, every step on the device (load and the
    image encoding on the host).  Informational; one timed run after one
    warm-up run."""
    import tempfile

    from fornos_b200 import api
    with tempfile.TemporaryDirectory() as d:
        lo_p, hi_p = os.path.join(d, "lo.ply"), os.path.join(d, "hi.ply")
        size = write_ply(lo_p, prep.lo) + write_ply(hi_p, prep.hm.arrays())
        smp = dict(enabled=1, sample_count=wl["spp"], min_distance=wl["min_d"], max_distance=wl["max_d"])
        out = {"height": dict(enabled="height" in wl["bakers"], output_path=os.path.join(d, "height.png"),
                              max_distance=wl["max_d"]),
               "positions": dict(enabled="position" in wl["bakers"], output_path=os.path.join(d, "positions.exr")),
               "normals": dict(enabled="normals" in wl["bakers"], output_path=os.path.join(d, "normals.png")),
               "ao": dict(smp, enabled="ao" in wl["bakers"], output_path=os.path.join(d, "ao.png")),
               "bent_normals": dict(smp, enabled="bn" in wl["bakers"], output_path=os.path.join(d, "bn.png")),
               "thickness": dict(smp, enabled="thick" in wl["bakers"], output_path=os.path.join(d, "thick.png"))}
        kw = dict(lo_poly_mesh_path=lo_p, hi_poly_mesh_path=hi_p, hi_poly_mesh_normal=api.NORMAL_COMPUTE_PER_VERTEX,
                  tex_width=wl["tex"], tex_height=wl["tex"], seed=seed, **out)
        try:
            api.run(ctx, **kw)
            t0 = time.perf_counter()
            api.run(ctx, **kw)
            ms = (time.perf_counter() - t0) * 1e3
        except Exception as e:  # reported, never fatal to the bench line
            return {"error": str(e)[:200]}
        written = sorted(f for f in os.listdir(d) if not f.endswith(".ply"))
    return {"ms": round(ms, 1), "input_bytes": int(size), "outputs": written,
            "steps": "PLY load, hi vertex normals, lo tangents, welded copy, raster, BVH build, mapping, "
                     "six solvers, export with dilation 16, PNG / EXR writing"}


def reduce_over_ranks(ms, rays, world, device):
    """Max of the per-rank step times and sum of the per-rank rays (every
    rank takes this same collective step)."""
    if world == 1:
        return float(ms), float(rays)
    import torch
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    r = torch.tensor([float(rays)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(r)
    return float(t.item()), float(r.item())


def replica_seed(base, rank):
    """Each rank bakes its own seeded replica of the workload."""
    return base + rank


def pinned(shape, dtype):
    import torch
    t = torch.empty(int(np.prod(shape)) * np.dtype(dtype).itemsize, dtype=torch.uint8, pin_memory=True)
    return t.numpy().view(dtype).reshape(shape), t


# ---------------------------------------------------------------- GPU arm
def run_fornos(args, wl, rank, world):
    import torch

    from fornos_b200 import api

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream()
    ctx = api.Context(dev)
    ctx.set_stream(stream.cuda_stream)
    if args.tuning:
        ctx.set_tuning(**parse_tuning(args.tuning))
    trav = TRAVERSE[args.traverse] | SCHEDULE[args.schedule]
    prep = Prepared(wl, replica_seed(args.seed, rank))
    tex, spp, lo_d, hi_d = wl["tex"], wl["spp"], wl["min_d"], wl["max_d"]

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        tmap = api.TexelMap.from_meshes(ctx, prep.lm, prep.dm, tex, tex)
        e1.record(stream)
    stream.synchronize()
    raster_ms = e0.elapsed_time(e1)
    n = tmap.count
    # the same scene from the mesh, BVH built on the device (fk_scene_build; informational)
    api.Scene.build(ctx, prep.hm, 8, 8192).free()
    ctx.sync()
    t0 = time.perf_counter()
    api.Scene.build(ctx, prep.hm, 8, 8192).free()
    ctx.sync()
    scene_build_ms = (time.perf_counter() - t0) * 1e3
    # the same preprocessing on the device (informational; first call warms the pool)
    device_preprocess(ctx, prep)
    t0 = time.perf_counter()
    dprep = device_preprocess(ctx, prep)
    prep_device_ms = (time.perf_counter() - t0) * 1e3
    dh, hh = dprep[0].arrays(), prep.hm.arrays()
    if not (np.array_equal(dh.vertices, hh.vertices) and np.array_equal(dh.normals, hh.normals, equal_nan=True)):
        raise RuntimeError("device preprocessing differs from the host's")
    del dprep
    scene = api.Scene(ctx, prep.nodes, prep.pos4, prep.nrm4)
    if args.tree == "reference":
        scene.set_tree(api.TREE_REFERENCE)
    info = scene.info()
    samples = api.samples_cosine(spp, api.PERMS, args.seed)
    sbuf = ctx.upload(samples)
    B = {k: ctx.buffer(w * max(n, 1)) for k, w in (("coords", 16), ("tidx", 4), ("height", 4), ("position", 12),
                                                  ("normals", 12), ("ao", 4), ("bn", 12), ("thick", 4),
                                                  ("hits_ao", 4), ("hits_bn", 4), ("hits_thick", 4))}
    map_max = wl.get("map_max", api.FLT_MAX)
    bakers = wl["bakers"]
    hemi_events = []

    def step(record):
        api.meshmap(ctx, scene, tmap, True, B["coords"], B["tidx"], max_dist=map_max)
        if "height" in bakers:
            api.gather(ctx, scene, api.GATHER_HEIGHT, B["coords"], B["tidx"], B["height"], 0, n)
        if "position" in bakers:
            api.gather(ctx, scene, api.GATHER_POSITION, B["coords"], B["tidx"], B["position"], 0, n)
        if "normals" in bakers:
            api.gather(ctx, scene, api.GATHER_NORMAL, B["coords"], B["tidx"], B["normals"], 0, n)
            api.tangent_space(ctx, tmap, B["normals"])
        launches = []
        if "ao" in bakers or "bn" in bakers:
            kind = api.AO_BN if ("ao" in bakers and "bn" in bakers) else (api.AO if "ao" in bakers else api.BN)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            api.hemisphere(ctx, scene, B["coords"], B["tidx"], kind, spp, lo_d, hi_d, sbuf,
                           B["ao"] if kind != api.BN else B["bn"], B["bn"] if kind == api.AO_BN else None,
                           B["hits_ao"] if kind != api.BN else B["hits_bn"],
                           B["hits_bn"] if kind == api.AO_BN else None, 0, n, traverse=trav)
            b.record(stream)
            launches.append((a, b, kind))
            if "bn" in bakers:
                api.tangent_space(ctx, tmap, B["bn"])
        if "thick" in bakers:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            api.hemisphere(ctx, scene, B["coords"], B["tidx"], api.THICK, spp, lo_d, hi_d, sbuf, B["thick"],
                           None, B["hits_thick"], None, 0, n, traverse=trav)
            b.record(stream)
            launches.append((a, b, api.THICK))
        if record:
            hemi_events.append(launches)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step(False)
    stream.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launches
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        with torch.cuda.stream(stream):
            t0.record(stream)
            for _ in range(args.steps):
                step(True)
            t1.record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    gpu_launches = ctx.launches - launches0
    ms = t0.elapsed_time(t1) / args.steps
    hemi_ms = {}
    for launches in hemi_events:
        for a, b, kind in launches:
            hemi_ms.setdefault(kind, []).append(a.elapsed_time(b))
    rays = rays_per_texel(wl) * n
    ms_max, rays_all = reduce_over_ranks(ms, rays, world, "cuda")

    # ---- end to end through fk_bake from pinned host memory
    keep = []

    def pin(a):
        p, t = pinned(a.shape, a.dtype)
        p[...] = a
        keep.append(t)
        return p

    cm = tmap.download()
    pix8 = np.zeros((n, 8), np.float32)
    pix8[:, 0:3], pix8[:, 4:7] = cm["positions"], cm["directions"]
    pixt = np.zeros((n, 12), np.float32)
    pixt[:, 0:3], pixt[:, 4:7], pixt[:, 8:11] = cm["normals"], cm["tangents"], cm["bitangents"]
    h_nodes, h_pos, h_nrm = pin(prep.nodes), pin(prep.pos4), pin(prep.nrm4)
    h_pix, h_pixt, h_idx = pin(pix8), pin(pixt), pin(cm["indices"])
    outs = {k: pinned(shape, dt) for k, shape, dt in (
        ("height", (n,), np.float32), ("position3", (n, 3), np.float32), ("normals3", (n, 3), np.float32),
        ("ao", (n,), np.float32), ("bent_normals3", (n, 3), np.float32), ("thickness", (n,), np.float32))}
    out_arrays = {k: v[0] for k, v in outs.items()}
    sampler = dict(sample_count=spp, min_distance=lo_d, max_distance=hi_d, seed=args.seed)
    kw = dict(height_map="height" in bakers, position_map="position" in bakers, normals_map="normals" in bakers,
              ao=sampler if "ao" in bakers else None,
              bent_normals=dict(sampler, tangent_space=True) if "bn" in bakers else None,
              thickness=sampler if "thick" in bakers else None, traverse=trav,
              mapping_max_distance=wl.get("map_max", 0.0))

    def e2e_step():
        api.bake(ctx, h_nodes, h_pos, h_nrm, tex, tex, h_pix, h_pixt, h_idx, out_arrays, **kw)

    e2e_step()  # warm-up
    if world > 1:
        torch.distributed.barrier()
    w0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_ms = (time.perf_counter() - w0) * 1e3 / args.steps
    e2e_ms, _ = reduce_over_ranks(e2e_ms, 0, world, "cuda")
    h2d = sum(a.nbytes for a in (h_nodes, h_pos, h_nrm, h_pix, h_pixt, h_idx)) + samples.nbytes
    d2h = sum(a.nbytes for k, a in out_arrays.items()
              if (k == "height" and "height" in bakers) or (k == "position3" and "position" in bakers)
              or (k == "normals3" and "normals" in bakers) or (k == "ao" and "ao" in bakers)
              or (k == "bent_normals3" and "bn" in bakers) or (k == "thickness" and "thick" in bakers))

    # ---- roofline of the dominant kernel (hemisphere traversal)
    peak = api.fp32_peak(ctx)
    tests = {}
    for launches in hemi_events[:1]:
        for _, _, kind in launches:
            tests[kind] = api.traversal_counts(ctx, scene, B["coords"], B["tidx"], kind, spp, lo_d, hi_d, sbuf, 0, n,
                                               traverse=trav)
    flops = sum(24 * b + 104 * t for b, t in tests.values())
    kern_ms = sum(statistics.mean(v) for v in hemi_ms.values())
    achieved = flops / (kern_ms * 1e-3)
    mrays = rays_all / (ms_max * 1e-3) / 1e6
    result = {
        "metric": "Mrays/s (plain bake: mapping + AO + bent normals + thickness rays)",
        "value": round(mrays, 3), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_max, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded generated meshes; no public dataset)",
        "config": {"workload": args.workload, "desc": wl["desc"], "texels": n, "texture": tex, "spp": spp,
                   "high_poly_triangles": prep.triangles, "bvh_nodes": info["node_count"],
                   "bvh_depth": info["depth"], "traverse": args.traverse, "schedule": args.schedule, "tree": args.tree,
                   "tuning": ctx.get_tuning(),
                   "rays_per_texel": rays_per_texel(wl), "traversals_per_texel": traversals_per_texel(wl),
                   "rays_counted": "2 mapping + spp each for AO, bent normals, thickness, as the reference traces "
                                   "them; AO and bent normals share one traversal here, so the rays traced are "
                                   "traversals_per_texel per texel (value x traversals_per_texel / rays_per_texel "
                                   "Mrays/s)",
                   "l2": "inputs larger than L2 (scene %.0f MB resident)" % (info["device_bytes"] / 1e6),
                   "bvh_build_s": round(prep.bvh_s, 3), "scene_build_device_ms": round(scene_build_ms, 1),
                   "preprocess_host_ms": round(prep.prep_s * 1e3, 1), "preprocess_device_ms": round(prep_device_ms, 1),
                   "raster_ms": round(raster_ms, 3),
                   "parallelism": "replicas" if world > 1 else "single"},
        "e2e": {"value": round(rays_all / (e2e_ms * 1e-3) / 1e6, 3), "unit": "Mrays/s",
                "ms_per_step": round(e2e_ms, 3), "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(gpu_launches),
        "roofline": {"bound": "fp32", "kernel": "hemi_trace_kernel", "achieved": round(achieved / 1e12, 3),
                     "peak": round(peak / 1e12, 3), "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
                     "traffic": NCU_TRAFFIC.get(args.workload),
                     "peak_source": "measured in-run: fk_diag_fp32_peak (add/mul/min chains, 1 op per instruction)",
                     "flops_per_step": int(flops), "kernel_ms_per_step": round(kern_ms, 3),
                     "box_tests": {str(k): v[0] for k, v in tests.items()},
                     "tri_tests": {str(k): v[1] for k, v in tests.items()},
                     "flop_model": "24 per ray-box test + 104 per ray-triangle test, tests counted on the GPU"},
        "clocks": clk.summary(),
    }
    return result, (prep, tmap, B, n, ctx, stream, scene)


# ---------------------------------------------------------------- denoised vs plain AO + BN
def run_denoise_bench(args):
    """The denoised-vs-plain comparison alone, on the plane workload's scene."""
    import torch

    from fornos_b200 import api
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    ctx = api.Context(0)
    ctx.set_stream(stream.cuda_stream)
    prep = Prepared(WORKLOADS["plane2048"], args.seed)
    scene = api.Scene(ctx, prep.nodes, prep.pos4, prep.nrm4)
    r = denoise_compare(ctx, stream, prep, scene, args.denoiser, args.seed, args.denoise_tex)
    if "unavailable" in r:
        return dict(r, metric="AO + bent-normal texels/s, 16 spp + denoiser vs 1024 spp")
    return {"metric": "AO + bent-normal texels/s at %dx%d: 16 spp + denoiser (verified) vs plain 1024 spp" % (
                args.denoise_tex, args.denoise_tex),
            "value": r["denoised"]["texels_per_s"], "unit": "texels/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32 traversal, bf16 network", "data": "synthetic (seeded generated meshes)",
            "config": {"workload": "denoise%d" % args.denoise_tex, "scene": WORKLOADS["plane2048"]["desc"],
                       "seed": args.seed},
            "denoise": r}



DENOISE = dict(tex=4096, low=16, full=1024, label=4096, min_d=0.001, max_d=0.3, tile=64, cells=4, max_err=0.02,
               mae_texels=65536)


def denoise_compare(ctx, stream, prep, scene, weights, seed, tex=4096, check=None):
    """AO + bent normals of the plane workload's scene at tex x tex texels
    (4096 for the reported comparison; smaller sizes serve as profiling cases):
    the plain 1024-sample bake against the verified 16-sample + network bake
    (spot checks and per-tile fallback included), each timed with CUDA events
    over one whole pass, and each scored by mean absolute error against
    4096-sample values on 65,536 random texels with a mapping hit.  check:
    called with the plain bake's texel map and buffers (the CPU-baseline
    leg's parity check of the plain path)."""
    import torch

    from fornos_b200 import api
    if not os.path.exists(weights):
        return {"unavailable": "no trained denoiser weights at %s" % os.path.relpath(weights, ROOT)}
    d = dict(DENOISE, tex=tex)
    tm = api.TexelMap.from_meshes(ctx, prep.lm, prep.dm, tex, tex)
    n = tm.count
    coords, tidx = ctx.buffer(16 * n), ctx.buffer(4 * n)
    api.meshmap(ctx, scene, tm, True, coords, tidx)
    hit = np.nonzero(tidx.download(np.uint32, n) != api.MISS)[0]
    low = ctx.upload(api.samples_cosine(d["low"], api.PERMS, seed + 11))
    full = ctx.upload(api.samples_cosine(d["full"], api.PERMS, seed + 12))
    label = ctx.upload(api.samples_cosine(d["label"], api.PERMS, seed + 13))
    dn = api.Denoiser(ctx, np.load(weights)["params"])
    args = (d["min_d"], d["max_d"])

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(0) as clk, torch.cuda.stream(stream):
            stream.synchronize()
            a.record(stream)
            out = fn()
            b.record(stream)
            stream.synchronize()
        return a.elapsed_time(b), out, clk.summary()

    pao, pbn = ctx.buffer(4 * n), ctx.buffer(12 * n)
    plain = lambda off, cnt: api.hemisphere(ctx, scene, coords, tidx, api.AO_BN, d["full"], *args, full, pao, pbn,
                                            None, None, off, cnt)
    plain(0, max(1, n // 100))  # warm-up on 1 % of the texels
    t_plain, _, clk_plain = timed(lambda: plain(0, n))
    plain_parity = check(tm, coords, tidx, pao, pbn, d, seed + 12) if check else None
    dao, dbn = ctx.buffer(4 * n), ctx.buffer(12 * n)
    bake = lambda: dn.bake(scene, tm, coords, tidx, low, full, dao, dbn, low_samples=d["low"],
                           full_samples=d["full"], min_distance=d["min_d"], max_distance=d["max_d"], tile=d["tile"],
                           verify_cells=d["cells"], max_tile_error=d["max_err"])
    bake()  # warm-up
    runs = [timed(bake) for _ in range(3)]
    t_dn, stats, clk_dn = sorted(runs, key=lambda r: r[0])[1]
    ctx.check()
    # the network alone on each engine, over the 16-sample bake's feature image
    ao16, bn16 = ctx.buffer(4 * n), ctx.buffer(12 * n)
    api.hemisphere(ctx, scene, coords, tidx, api.AO_BN, d["low"], *args, low, ao16, bn16, None, None, 0, n)
    pos, nrm = ctx.buffer(12 * n), ctx.buffer(12 * n)
    api.gather(ctx, scene, api.GATHER_POSITION, coords, tidx, pos, 0, n)
    api.gather(ctx, scene, api.GATHER_NORMAL, coords, tidx, nrm, 0, n)
    image = api.denoise_features(ctx, tm, coords, tidx, ao16, bn16, pos, nrm, d["max_d"])
    oa, ob = ctx.buffer(4 * n), ctx.buffer(12 * n)
    net = {}
    flop = 2 * (250 * 64 + 64 * 64 + 64 * 4)  # per texel, without the padding
    peak = None
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"]
    except (OSError, KeyError, ValueError):
        pass
    for name, eng in (("tcgen05", api.DN_ENGINE_TCGEN05), ("mma_sync", api.DN_ENGINE_MMA_SYNC)):
        dn.set_engine(eng)
        dn.apply(tm, image, tidx, ao16, bn16, oa, ob)  # warm-up
        ms = sorted(timed(lambda: dn.apply(tm, image, tidx, ao16, bn16, oa, ob))[0] for _ in range(5))[2]
        tf = flop * n / (ms * 1e-3) / 1e12
        net[name] = dict(ms=round(ms, 3), tflops=round(tf, 2),
                         frac_of_bf16_peak=round(tf / peak, 4) if peak else None)
    dn.set_engine(api.DN_ENGINE_TCGEN05)
    ctx.check()
    net["flop_per_texel"] = flop
    net["peak"] = "%s TFLOP/s bf16 (MEASURED_PEAKS.json, burst)" % peak if peak else "MEASURED_PEAKS.json absent"
    for b in (ao16, bn16, pos, nrm, image, oa, ob):
        b.free()
    # accuracy against 4096-sample values on random texels with a mapping hit
    ids = np.sort(np.random.default_rng(seed).choice(hit, min(d["mae_texels"], len(hit)), replace=False))
    ids = ids.astype(np.uint32)
    lao, lbn = ctx.buffer(4 * n), ctx.buffer(12 * n)
    api.hemisphere_texels(ctx, scene, coords, tidx, n, api.AO_BN, d["label"], *args, label, ctx.upload(ids), lao,
                          lbn)
    pick = lambda b, w: (b.download(np.float32, n) if w == 1 else b.download(np.float32, (n, 3)))[ids]
    clean = lambda v: np.where(np.isfinite(v).all(1, keepdims=True), v, 0)
    la, lb = pick(lao, 1), clean(pick(lbn, 3))

    def score(ao_b, bn_b):
        return {"mae_ao": round(float(np.abs(pick(ao_b, 1) - la).mean()), 5),
                "mae_bn": round(float(np.abs(clean(pick(bn_b, 3)) - lb).mean()), 5)}

    covered = len(hit)
    res = {
        "texture": tex, "texels_with_hit": covered, "train_meta": json.loads(str(np.load(weights)["meta"])).get(
            "eval_mae"),
        "plain": dict(samples=d["full"], ms=round(t_plain, 2), texels_per_s=round(covered / (t_plain * 1e-3), 1),
                      clocks=clk_plain, **score(pao, pbn)),
        "denoised": dict(samples=d["low"], ms=round(t_dn, 2), texels_per_s=round(covered / (t_dn * 1e-3), 1),
                         clocks=clk_dn, stats=stats, **score(dao, dbn)),
        "mae_reference": "%d-sample AO + bent normals on %d random texels with a mapping hit" % (
            d["label"], len(ids)),
        "fallback_rule": "tile %d x %d, %d spot checks at %d samples, re-bake if error > %.2f" % (
            d["tile"], d["tile"], d["cells"] ** 2, d["full"], d["max_err"]),
        "network_kernel": net,
    }
    res["speedup"] = round(t_plain / t_dn, 2)
    if plain_parity is not None:
        res["plain_parity"] = plain_parity
    for b in (tm, coords, tidx, low, full, label, pao, pbn, dao, dbn, lao, lbn):
        b.free()
    dn.free()
    return res


# ---------------------------------------------------------------- CPU arm
class CpuBaseline:
    """The reference's CPU implementation of the path, timed on the host
    cores (all OpenMP threads) over a strided sample of the workload's
    compressed texels: the reference's shaders and host code compiled by
    oracle/build_ref.py, or the oracle restatement where that build is absent."""

    def __init__(self, wl, seed, prep=None, cmap=None, prefer_ref=True):
        from oracle import pyoracle
        self.oracle = pyoracle.Oracle()
        ref = None
        if prefer_ref:
            try:
                ref = pyoracle.Reference()
            except OSError:
                ref = None
        self.impl = ref if ref is not None else self.oracle
        self.kind = "reference" if ref is not None else "port"
        self.cores = self.oracle.threads()
        self.wl, self.spp = wl, wl["spp"]
        tex = wl["tex"]
        if prep is None:
            impl = self.impl
            lo, hi = wl["gen"](seed)
            v, nrm = impl.normals(hi, "vertex")
            hi.vertices, hi.normals = v, nrm
            lo.tangents, lo.bitangents = impl.tangent_space(lo)
            cmap = impl.raster(lo, tex, tex, 0, impl.normals(lo, "welded"))
            self.nodes, self.pos4, self.nrm4 = impl.scene(hi)
        else:
            self.nodes, self.pos4, self.nrm4 = prep.nodes, prep.pos4, prep.nrm4
        self.n = n = len(cmap["indices"])
        self.pix8 = np.zeros((n, 8), np.float32)
        self.pix8[:, 0:3], self.pix8[:, 4:7] = cmap["positions"], cmap["directions"]
        self.kinds = [k for k, b in ((0, "ao"), (1, "bn"), (2, "thick")) if b in wl["bakers"]]
        self.samples = self.impl.samples(self.spp, 4096, seed)
        self.stride = max(1, n // 64)

    def run(self, stride=None):
        """One timed pass over every stride-th texel: the reference's mapping,
        then its sampling shaders.  The reference's mapping has no distance
        limit; a workload's limit m is applied to its result (hits at t >= m
        become misses), which is what walks started at m return (grazing hits
        on box faces aside).  The outputs are kept in self.last for the
        parity check."""
        stride = stride or self.stride
        n, impl = self.n, self.impl
        sel = np.arange(0, n, stride, dtype=np.uint32)
        t0 = time.perf_counter()
        c_sel, t_sel = impl.meshmap(self.nodes, self.pos4, self.pix8[sel], True)
        if self.wl.get("map_max") is not None:
            far = (t_sel != 0xFFFFFFFF) & ~(c_sel[:, 0] < np.float32(self.wl["map_max"]))
            t_sel[far] = 0xFFFFFFFF
            c_sel[far] = (np.finfo(np.float32).max, 0.0, 0.0, 0.0)
        coords = np.zeros((n, 4), np.float32)
        tidx = np.full(n, 0xFFFFFFFF, np.uint32)
        coords[sel], tidx[sel] = c_sel, t_sel
        outs = {}
        for k in self.kinds:
            r = impl.hemisphere(k, self.nodes, self.pos4, self.nrm4, coords, tidx, self.samples, self.spp,
                                self.wl["min_d"], self.wl["max_d"], texels=sel)
            outs[k] = r[0] if isinstance(r, tuple) else r
        dt = time.perf_counter() - t0
        self.last = dict(sel=sel, coords=c_sel, tidx=t_sel, outs=outs)
        rays = len(sel) * (2 + self.spp * len(self.kinds))
        return rays / dt / 1e6, rays, dt, len(sel)

    def parity(self, B, n, cmap):
        """The GPU bake's buffers (B, n texels) at the texels of the last run
        against the reference's outputs there (oracle/parity.py)."""
        from oracle import parity
        L = self.last
        sel, hit = L["sel"], L["tidx"] != parity.MISS
        take = lambda name, w, dt=np.float32: B[name].download(dt, n if w == 1 else (n, w))[sel]
        rep = {"texels": int(len(sel)),
               "mapping": parity.mapping(L["coords"], L["tidx"], take("coords", 4), take("tidx", 1, np.uint32))}
        if self.wl.get("map_max") is not None:
            rep["mapping"]["note"] = ("the reference's mapping has no distance limit: its hits at t >= %g are "
                                      "dropped before comparing" % self.wl["map_max"])
        if 0 in L["outs"]:
            rep["ao"] = parity.sampled(L["outs"][0], take("ao", 1), hit, self.spp,
                                       gpu_hits=take("hits_ao", 1, np.uint32))
        if 1 in L["outs"]:
            bn = L["outs"][1]
            if "bn" in self.wl["bakers"]:  # the bench bake stores bent normals in tangent space
                bn = self.impl.tangent_transform(cmap["normals"][sel], cmap["tangents"][sel],
                                                 cmap["bitangents"][sel], bn)
            rep["bn"] = parity.sampled(bn, take("bn", 3), hit)
        if 2 in L["outs"]:
            rep["thick"] = parity.sampled(L["outs"][2], take("thick", 1), hit)
        rep["meets_bar"] = parity.meets_bar(rep)
        rep["bar"] = ("texel map, hit indices, barycentrics bit-exact; sampled outputs bit-exact on all but "
                      "<= 0.01% of texels, occluder counts within one sample")
        rep["compared_with"] = "%s (%s)" % ("oracle/_ref: the reference's shaders compiled on the host"
                                             if self.kind == "reference" else "the oracle restatement", self.kind)
        return rep

    def calibrate(self, budget_s):
        """Chooses the texel stride so one run takes about budget_s seconds."""
        stride = max(1, self.n // 64)
        _, _, dt, _ = self.run(stride)
        while dt < 0.25 and stride > 1:
            stride = max(1, stride // 8)
            _, _, dt, _ = self.run(stride)
        self.stride = max(1, int(stride * dt / budget_s)) if dt < budget_s else stride
        return self.stride

    def describe(self, rays, m):
        return "every %d-th of %d compressed texels (%d texels, %d rays): mapping + %s at %d spp" % (
            self.stride, self.n, m, rays, " + ".join({0: "AO", 1: "BN", 2: "thickness"}[k] for k in self.kinds),
            self.spp)


def plain_path_check(cpu, prep, texels=1024):
    """Parity check of the denoise comparison's plain 1024-sample AO + bent
    normal bake: the reference's mapping and sampling shaders (cpu.impl) on
    `texels` random texels with a mapping hit, against the GPU buffers."""
    from oracle import parity

    def check(tm, coords, tidx, pao, pbn, d, sample_seed):
        n = tm.count
        g_t = tidx.download(np.uint32, n)
        rng = np.random.default_rng(sample_seed)
        sel = np.sort(rng.choice(np.nonzero(g_t != parity.MISS)[0], min(texels, n), replace=False)).astype(np.uint32)
        cm = tm.download()
        pix8 = np.zeros((len(sel), 8), np.float32)
        pix8[:, 0:3], pix8[:, 4:7] = cm["positions"][sel], cm["directions"][sel]
        impl = cpu.impl
        c_sel, t_sel = impl.meshmap(prep.nodes, prep.pos4, pix8, True)
        rep = {"texels": int(len(sel)), "samples": d["full"],
               "mapping": parity.mapping(c_sel, t_sel, coords.download(np.float32, (n, 4))[sel], g_t[sel])}
        full_c = np.zeros((n, 4), np.float32)
        full_t = np.full(n, parity.MISS, np.uint32)
        full_c[sel], full_t[sel] = c_sel, t_sel
        table = impl.samples(d["full"], 4096, sample_seed)
        hit = t_sel != parity.MISS
        for k, name, buf, w in ((0, "ao", pao, 1), (1, "bn", pbn, 3)):
            r = impl.hemisphere(k, prep.nodes, prep.pos4, prep.nrm4, full_c, full_t, table, d["full"], d["min_d"],
                                d["max_d"], texels=sel)
            r = r[0] if isinstance(r, tuple) else r
            g = buf.download(np.float32, n if w == 1 else (n, 3))[sel]
            rep[name] = parity.sampled(r, g, hit, d["full"] if k == 0 else None)
        rep["meets_bar"] = parity.meets_bar(rep)
        rep["compared_with"] = cpu.kind
        return rep

    return check


def run_reference_arm(args, wl):
    cpu = CpuBaseline(wl, args.seed)
    cpu.calibrate(args.cpu_seconds)
    vals = []
    rays = m = 0
    for i in range(args.warmup + args.steps):
        mr, rays, dt, m = cpu.run()
        if i >= args.warmup:
            vals.append(mr)
    value = statistics.median(vals)
    return {
        "metric": "Mrays/s (plain bake: mapping + AO + bent normals + thickness rays)", "impl": "reference",
        "value": round(value, 4), "unit": "Mrays/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generated meshes; no public dataset)",
        "config": {"workload": args.workload, "desc": wl["desc"]},
        "cpu_baseline": {"value": round(value, 4), "unit": "Mrays/s", "cores": cpu.cores, "kind": cpu.kind,
                         "sample": cpu.describe(rays, m)},
        "e2e": {"value": round(value, 4), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def batch_jobs(seed, count):
    """The batched-bake workload: `count` jobs, each a sphere-style or
    plane-style pair from its own seed, high-poly triangle count log-uniform in
    10k..2M, texture from {256, 512, 1024, 2048}, AO spp from {32, 128, 512}."""
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(count):
        tris = float(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
        tex = int(rng.choice([256, 512, 1024, 2048]))
        spp = int(rng.choice([32, 128, 512]))
        if i % 2 == 0:
            hq = max(8, int(round((tris / 2) ** 0.5)))
            gen = (lambda s, hq=hq: W.plane_pair(seed=s, lo_quads=64, hi_quads=hq, bumps=200))
            lo_d, hi_d = 0.001, 0.3
        else:
            u = max(16, int(round(tris ** 0.5)))
            gen = (lambda s, u=u: W.sphere_pair(seed=s, hi_seg=(u, max(8, u // 2))))
            lo_d, hi_d = 0.001, 0.5
        jobs.append(dict(gen=gen, seed=seed * 1000 + i, tex=tex, spp=spp, min_d=lo_d, max_d=hi_d))
    return jobs


def batch_compare(ctx, stream, seed, njobs, check=None):
    """The batched-bake comparison over `njobs` jobs of batch_jobs(seed):
    per-job fk_hemisphere launches (context defaults, then the tuned
    schedule) against one batched persistent launch (default schedule,
    autotuned, autotuned in a CUDA graph).  AO only.  Scenes are built on the
    device (fk_scene_build); check(job, outputs) is the CPU-baseline leg's
    oracle comparison of one job."""
    import torch

    from fornos_b200 import api
    specs = batch_jobs(seed, njobs)
    jobs, keep = [], []
    tables = {}
    t_prep = time.perf_counter()
    for s in specs:
        lo, hi = s["gen"](s["seed"])
        hm = api.Mesh(hi)
        hm.compute_vertex_normals()
        lm = api.Mesh(lo)
        lm.compute_tangent_space()
        dm = lm.copy()
        dm.compute_vertex_normals_aggressive()
        tm = api.TexelMap.from_meshes(ctx, lm, dm, s["tex"], s["tex"])
        scene = api.Scene.build(ctx, hm, 8, 8192)
        n = tm.count
        coords, tidx = ctx.buffer(16 * n), ctx.buffer(4 * n)
        api.meshmap(ctx, scene, tm, True, coords, tidx)
        if s["spp"] not in tables:
            tables[s["spp"]] = ctx.upload(api.samples_cosine(s["spp"], api.PERMS, seed))
        jobs.append(dict(scene=scene, coords=coords, tidx=tidx, texel_count=n, spp=s["spp"], min_distance=s["min_d"],
                         max_distance=s["max_d"], samples=tables[s["spp"]], out0=ctx.buffer(4 * n),
                         hits0=ctx.buffer(4 * n), triangles=hi.triangle_count, tex=s["tex"], seed=s["seed"],
                         mesh=hm, tmap=tm))
        keep.append((tm, lm, dm))
    ctx.sync()
    prep_s = time.perf_counter() - t_prep
    rays = sum(j["texel_count"] * j["spp"] for j in jobs)
    clocks = {}

    def timed(fn, name):
        # one pass per call, every job's scene and texels already resident,
        # with the SM clock sampled during it
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(0) as clk, torch.cuda.stream(stream):
            stream.synchronize()
            a.record(stream)
            fn()
            b.record(stream)
            stream.synchronize()
        clocks.setdefault(name, []).append(clk.summary())
        return a.elapsed_time(b)

    def per_job(traverse=0):
        for j in jobs:
            api.hemisphere(ctx, j["scene"], j["coords"], j["tidx"], api.AO, j["spp"], j["min_distance"],
                           j["max_distance"], j["samples"], j["out0"], None, j["hits0"], None, 0, j["texel_count"],
                           traverse=traverse)

    outs = [dict(out0=ctx.buffer(4 * j["texel_count"]), hits0=ctx.buffer(4 * j["texel_count"])) for j in jobs]
    batch = api.Batch(ctx, [dict(j, **o) for j, o in zip(jobs, outs)], api.AO)
    default = ctx.get_tuning()
    # per-job and batched passes alternate, twice, so that neither arm runs on
    # a cooler GPU than the other; each arm keeps its faster pass
    t_jobs, t_batch = [], []
    for _ in range(2):
        t_jobs.append(timed(per_job, "per_job_launches"))
        t_batch.append(timed(lambda: batch.run(), "batch_default"))
    want = [(j["out0"].download(np.float32, j["texel_count"]), j["hits0"].download(np.uint32, j["texel_count"]))
            for j in jobs]
    tuned = batch.tune()
    # the same tuned schedule for per-job launches and the batch
    ctx.set_tuning(refill=tuned["refill"], leaf_batch=tuned["leaf_batch"], speculate=tuned["speculate"])
    t_jobs_tuned, t_tuned, t_graph = [], [], []
    batch.capture()
    for _ in range(2):
        t_jobs_tuned.append(timed(lambda: per_job(tuned["traverse"]), "per_job_tuned"))
        t_tuned.append(timed(lambda: batch.run(), "batch_tuned"))
        t_graph.append(timed(lambda: batch.replay(), "batch_tuned_graph"))
    ctx.set_tuning(**default)
    t_jobs, t_batch, t_jobs_tuned, t_tuned, t_graph = (min(v) for v in (t_jobs, t_batch, t_jobs_tuned, t_tuned,
                                                                        t_graph))
    identical = all(np.array_equal(o["out0"].download(np.float32, j["texel_count"]).view(np.uint32),
                                   w[0].view(np.uint32))
                    and np.array_equal(o["hits0"].download(np.uint32, j["texel_count"]), w[1])
                    for j, o, w in zip(jobs, outs, want))
    mr = lambda ms: round(rays / (ms * 1e-3) / 1e6, 2)
    res = {
        "jobs": len(jobs), "rays": rays, "texels": sum(j["texel_count"] for j in jobs),
        "triangles": [j["triangles"] for j in jobs], "textures": [j["tex"] for j in jobs],
        "spp": [j["spp"] for j in jobs], "prep_s": round(prep_s, 1),
        "per_job_launches": {"ms": round(t_jobs, 2), "mrays": mr(t_jobs), "tuning": default},
        "batch_default": {"ms": round(t_batch, 2), "mrays": mr(t_batch)},
        "per_job_tuned": {"ms": round(t_jobs_tuned, 2), "mrays": mr(t_jobs_tuned)},
        "batch_tuned": {"ms": round(t_tuned, 2), "mrays": mr(t_tuned), "tuning": tuned},
        "batch_tuned_graph": {"ms": round(t_graph, 2), "mrays": mr(t_graph), "info": batch.info()},
        "graph_vs_per_job_tuned": round(t_jobs_tuned / t_graph, 4),
        "batch_equals_per_job": bool(identical),
        "clocks": clocks,
    }
    if check is not None:
        k = int(np.argmin([j["triangles"] for j in jobs]))  # the smallest job: its reference run is quick
        res["oracle_check"] = check(jobs[k], outs[k], k)
    return res


def batch_check(cpu_kind="reference", texels=256):
    """Oracle comparison of one batched job (the CPU-baseline leg): the
    reference's AO shader (oracle/_ref, else the oracle) on `texels` random
    texels with a mapping hit, fed the job's own mapping and scene arrays,
    against the batch's outputs there."""
    from fornos_b200 import api
    from oracle import parity, pyoracle

    def check(job, out, k):
        impl = None
        if cpu_kind == "reference":
            try:
                impl = pyoracle.Reference()
            except OSError:
                impl = None
        kind = "reference" if impl is not None else "port"
        impl = impl or pyoracle.Oracle()
        n = job["texel_count"]
        ctx = job["scene"].ctx
        nodes, pos4, nrm4 = api.BVH.build_flat_device(ctx, job["mesh"], 8, 8192)
        coords, tidx = job["coords"].download(np.float32, (n, 4)), job["tidx"].download(np.uint32, n)
        hit = np.nonzero(tidx != parity.MISS)[0]
        sel = np.sort(np.random.default_rng(k).choice(hit, min(texels, len(hit)), replace=False)).astype(np.uint32)
        table = job["samples"].download(np.float32, (4096 * job["spp"], 4))
        r = impl.hemisphere(0, nodes, pos4, nrm4, coords, tidx, table, job["spp"], job["min_distance"],
                            job["max_distance"], texels=sel)
        r = r[0] if isinstance(r, tuple) else r
        got = out["out0"].download(np.float32, n)[sel]
        rep = parity.sampled(r, got, np.ones(len(sel), bool), job["spp"],
                             gpu_hits=out["hits0"].download(np.uint32, n)[sel])
        rep.update(job=k, triangles=job["triangles"], compared_with=kind, meets_bar=parity.meets_bar({"ao": rep}))
        return rep

    return check


def run_batch_bench(args):
    """C4 alone: the batched-bake comparison as its own JSON line."""
    import torch

    from fornos_b200 import api
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    ctx = api.Context(0)
    ctx.set_stream(stream.cuda_stream)
    r = batch_compare(ctx, stream, args.seed, args.batch_jobs, None if args.no_cpu_baseline else batch_check())
    return {
        "metric": "Mrays/s (batched AO bake of %d jobs)" % r["jobs"], "value": r["batch_tuned_graph"]["mrays"],
        "unit": "Mrays/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
        "data": "synthetic (seeded generated meshes)",
        "config": {"workload": "batch%d" % r["jobs"], "rays": r["rays"], "texels": r["texels"]},
        "batch": r,
    }


def side_workload(args, name, steps=2, warmup=1):
    """Another workload's plain bake, measured as the headline's is (device
    steps, e2e through fk_bake, the trace kernels' roofline) with fewer steps;
    with the CPU baseline on, its parity against the reference's outputs on a
    strided texel sample (about 4 s of CPU work)."""
    import copy
    wl = WORKLOADS[name]
    a = copy.copy(args)
    a.steps, a.warmup, a.workload = steps, warmup, name
    r, state = run_fornos(a, wl, 0, 1)
    out = {k: r[k] for k in ("value", "unit", "ms_per_step", "e2e", "clocks")}
    out["config"] = {k: r["config"][k] for k in ("desc", "texels", "texture", "spp", "high_poly_triangles",
                                                 "rays_per_texel", "traversals_per_texel")}
    out["roofline"] = {k: r["roofline"][k] for k in ("achieved", "peak", "unit", "frac", "kernel_ms_per_step")}
    if not args.no_cpu_baseline:
        prep, tmap = state[0], state[1]
        cmap = tmap.download()
        cpu = CpuBaseline(wl, args.seed, prep, cmap)
        cpu.calibrate(4.0)
        mr, rays, dt, m = cpu.run()
        out["cpu_baseline"] = {"value": round(mr, 4), "unit": "Mrays/s", "cores": cpu.cores, "kind": cpu.kind,
                               "sample": cpu.describe(rays, m)}
        out["parity"] = cpu.parity(state[2], state[3], cmap)
    for b in state[2].values():
        b.free()
    state[6].free()
    state[1].free()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fornos", choices=["fornos", "reference"])
    ap.add_argument("--workload", default="plane2048", choices=list(WORKLOADS) + ["batch", "denoise"])
    ap.add_argument("--batch-jobs", type=int, default=64)
    ap.add_argument("--traverse", default="auto", choices=list(TRAVERSE))
    ap.add_argument("--schedule", default="auto", choices=list(SCHEDULE))
    ap.add_argument("--tree", default="sah", choices=["reference", "sah"],
                    help="inner tree of the ordered traversals: rebuilt over the reference's leaves (sah) or the "
                         "reference's own")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-denoise", action="store_true", help="skip the denoised-vs-plain comparison")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-bake comparison of the default line")
    ap.add_argument("--tuning", default="",
                    help="fk_tuning knobs for the bake, e.g. refill=8,top_records=64 (default: the context's)")
    ap.add_argument("--side", default="sphere512",
                    help="other workloads measured in the default line (comma-separated; empty: none)")
    ap.add_argument("--line-batch-jobs", type=int, default=16,
                    help="jobs of the default line's batched-bake comparison (--workload batch: --batch-jobs)")
    ap.add_argument("--denoise-tex", type=int, default=4096,
                    help="texture size of the denoised-vs-plain comparison (4096 reported; smaller for profiling)")
    ap.add_argument("--denoiser", default=os.path.join(ROOT, "fornos_b200", "data", "denoiser_plane2048.npz"))
    args = ap.parse_args()
    if args.workload == "batch":
        print(json.dumps(run_batch_bench(args)))
        return 0
    if args.workload == "denoise":
        print(json.dumps(run_denoise_bench(args)))
        return 0
    wl = WORKLOADS[args.workload]
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))

    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference_arm(args, wl)))
        return 0

    import datetime

    import torch
    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                             device_id=torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0))))
    result, state = run_fornos(args, wl, rank, world)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        prep, tmap = state[0], state[1]
        cmap = tmap.download()
        cpu = CpuBaseline(wl, args.seed, prep, cmap)
        cpu.calibrate(args.cpu_seconds)
        mr, rays, dt, m = cpu.run()
        result["cpu_baseline"] = {"value": round(mr, 4), "unit": "Mrays/s", "cores": cpu.cores, "kind": cpu.kind,
                                  "sample": cpu.describe(rays, m)}
        # the timed bake's own outputs (last timed step) at the CPU run's texels
        result["parity"] = cpu.parity(state[2], state[3], cmap)
    if rank == 0 and world == 1:
        result["files_to_images"] = files_to_images(state[4], state[0], wl, args.seed)
    if rank == 0 and world == 1 and args.workload == "plane2048" and not args.no_denoise:
        prep, _, _, _, ctx, stream, scene = state
        check = plain_path_check(cpu, prep) if not args.no_cpu_baseline else None
        result["denoise"] = denoise_compare(ctx, stream, prep, scene, args.denoiser, args.seed, args.denoise_tex,
                                            check)
    if rank == 0 and world == 1 and args.workload == "plane2048" and args.side:
        result["side_workloads"] = {}
        for name in args.side.split(","):
            result["side_workloads"][name] = side_workload(args, name)
    if rank == 0 and world == 1 and args.workload == "plane2048" and not args.no_batch:
        ctx, stream = state[4], state[5]
        result["batch"] = batch_compare(ctx, stream, args.seed, args.line_batch_jobs,
                                        None if args.no_cpu_baseline else batch_check())
    if rank == 0:
        print(json.dumps(result))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
