"""Trains the learned AO + bent-normal denoiser on bakes the method itself
generates from seeded meshes, with the project's own CUDA training kernels.

    python -m fornos_b200.denoise_train [--train-seeds 200] [--eval-seeds 20]
        [--out fornos_b200/data/denoiser_plane2048.npz]

Data: the 64 x 64-quad plane / 1024 x 1024-quad heightfield generator
(4-octave value noise + 200 bumps) at 2048 x 2048 texels, AO / bent normals
with min distance 0.001 and max distance 0.3.  Per seed, every texel is baked
at 16 samples (the network's input); a random subset of texels with a mapping
hit is baked at 4096 samples through the texel-list pass, and those texels
become training rows (their 5 x 5 feature neighbourhood) with residual
targets (AO_4096 - AO_16, BN_4096 - BN_16).  Held-out seeds give the reported
mean absolute errors of the raw 16-sample values, the denoised values and the
plain 1024-sample bake against the 4096-sample labels.

Scene preparation (mesh generation, BVH build) runs in a process pool started
before any GPU work; everything on the GPU runs through the public API.
"""
import argparse
import collections
import itertools
import json
import math
import multiprocessing as mp
import os
import time

import numpy as np

LOW, LABEL, PLAIN = 16, 4096, 1024
MIN_D, MAX_D = 0.001, 0.3
TEX = 2048
DEFAULT_OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "denoiser_plane2048.npz")


def prepare(seed):
    """CPU half of a bake job (pool worker): meshes, BVH, flattened arrays."""
    from . import api
    from . import workloads as W
    lo, hi = W.plane_pair(seed=seed, lo_quads=64, hi_quads=1024, bumps=200)
    hm = api.Mesh(hi)
    hm.compute_vertex_normals()
    bvh = api.BVH.create_binary(hm, 8, 8192)
    nodes, pos4, nrm4 = bvh.flatten(hm)
    return seed, lo, nodes, pos4, nrm4


def prepared_in_order(pool, seeds, window):
    """prepare(seed) for every seed, in order, with at most `window` results
    in flight (each holds a few hundred MB of scene arrays)."""
    pending, it = collections.deque(), iter(seeds)
    for s in itertools.islice(it, window):
        pending.append(pool.apply_async(prepare, (s,)))
    while pending:
        r = pending.popleft().get()
        nxt = next(it, None)
        if nxt is not None:
            pending.append(pool.apply_async(prepare, (nxt,)))
        yield r


def init_params(seed):
    """He-style initial weights (W1's pad columns zero)."""
    from .api import DN_PARAMS, DN_LAYOUT
    rng = np.random.default_rng(seed)
    p = np.zeros(DN_PARAMS, np.float32)
    view = {k: p[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in DN_LAYOUT.items()}
    view["w1"][:, :250] = rng.normal(0, math.sqrt(2.0 / 250), (64, 250))
    view["w2"][:] = rng.normal(0, math.sqrt(2.0 / 64), (64, 64))
    view["w3"][:] = rng.normal(0, 0.1 * math.sqrt(1.0 / 64), (4, 64))
    return p


class SeedBake:
    """GPU half: scene, texel map, mapping, 16-sample bake and feature image."""

    def __init__(self, ctx, prepared, tex=TEX, low_table=None):
        from . import api
        seed, lo, nodes, pos4, nrm4 = prepared
        self.ctx, self.seed = ctx, seed
        lm = api.Mesh(lo)
        lm.compute_tangent_space()
        dm = lm.copy()
        dm.compute_vertex_normals_aggressive()
        self.scene = api.Scene(ctx, nodes, pos4, nrm4)
        self.tm = api.TexelMap.from_meshes(ctx, lm, dm, tex, tex)
        n = self.n = self.tm.count
        self.coords, self.tidx = ctx.buffer(16 * n), ctx.buffer(4 * n)
        api.meshmap(ctx, self.scene, self.tm, True, self.coords, self.tidx)
        self.low = low_table if low_table is not None else ctx.upload(api.samples_cosine(LOW, api.PERMS, seed))
        self.ao, self.bn = ctx.buffer(4 * n), ctx.buffer(12 * n)
        api.hemisphere(ctx, self.scene, self.coords, self.tidx, api.AO_BN, LOW, MIN_D, MAX_D, self.low, self.ao,
                       self.bn, None, None, 0, n)
        pos, nrm = ctx.buffer(12 * n), ctx.buffer(12 * n)
        api.gather(ctx, self.scene, api.GATHER_POSITION, self.coords, self.tidx, pos, 0, n)
        api.gather(ctx, self.scene, api.GATHER_NORMAL, self.coords, self.tidx, nrm, 0, n)
        self.image = api.denoise_features(ctx, self.tm, self.coords, self.tidx, self.ao, self.bn, pos, nrm, MAX_D)
        pos.free()
        nrm.free()
        self.tidx_host = self.tidx.download(np.uint32, n)
        self.indices = self.tm.download()["indices"]

    def texels(self, m, seed):
        hit = np.nonzero(self.tidx_host != 0xFFFFFFFF)[0]
        rng = np.random.default_rng(seed)
        return np.sort(rng.choice(hit, min(m, len(hit)), replace=False)).astype(np.uint32)

    def bake_texels(self, ids_buf, m, spp, table):
        """AO + BN at `spp` for the listed texels (full-size outputs)."""
        from . import api
        ao, bn = self.ctx.buffer(4 * self.n), self.ctx.buffer(12 * self.n)
        api.hemisphere_texels(self.ctx, self.scene, self.coords, self.tidx, self.n, api.AO_BN, spp, MIN_D, MAX_D,
                              table, ids_buf, ao, bn, count=m)
        return ao, bn

    def free(self):
        for b in (self.scene, self.tm, self.coords, self.tidx, self.ao, self.bn, self.image):
            b.free()


def clean_bn(b):
    b = np.array(b, np.float32)
    b[~np.isfinite(b).all(1)] = 0
    return b


def denoised_values(ao16, bn16, y):
    """The apply kernel's output rule on host arrays (for evaluation)."""
    ao = np.clip(ao16 + y[:, 0], 0, 1)
    v = clean_bn(bn16) + y[:, 1:4]
    d = np.sqrt((v * v).sum(1))
    bn = np.where(d[:, None] > 0, v / np.maximum(d, 1e-30)[:, None], 0)
    return ao, bn


def mae(ao, bn, lao, lbn):
    return float(np.abs(ao - lao).mean()), float(np.abs(bn - clean_bn(lbn)).mean())


def collect(ctx, sb, m, label_table, plain_table=None):
    """Rows, targets and the values needed to score them for m texels of a seed."""
    from . import api
    ids = sb.texels(m, sb.seed + 7919)
    m = len(ids)
    ids_buf = ctx.upload(ids)
    lao_b, lbn_b = sb.bake_texels(ids_buf, m, LABEL, label_table)
    rows = api.denoise_rows(ctx, sb.image, sb.tm.width, sb.tm.height, ctx.upload(sb.indices[ids]), m)
    ao16 = sb.ao.download(np.float32, sb.n)[ids]
    bn16 = sb.bn.download(np.float32, (sb.n, 3))[ids]
    lao = lao_b.download(np.float32, sb.n)[ids]
    lbn = clean_bn(lbn_b.download(np.float32, (sb.n, 3))[ids])
    out = dict(rows=rows.download(np.uint8, (m, 512)), ao16=ao16, bn16=bn16, lao=lao, lbn=lbn,
               target=np.concatenate([(lao - ao16)[:, None], lbn - clean_bn(bn16)], 1).astype(np.float32))
    if plain_table is not None:
        pao, pbn = sb.bake_texels(ids_buf, m, PLAIN, plain_table)
        out["pao"] = pao.download(np.float32, sb.n)[ids]
        out["pbn"] = pbn.download(np.float32, (sb.n, 3))[ids]
        pao.free()
        pbn.free()
    for b in (ids_buf, lao_b, lbn_b, rows):
        b.free()
    return out


def evaluate(ctx, dn, ev):
    """MAEs of raw 16-sample, denoised and plain 1024-sample values."""
    rows = ctx.upload(np.ascontiguousarray(ev["rows"]))
    m = len(ev["ao16"])
    y = dn.forward(rows, m).download(np.float32, (m, 4))
    ao, bn = denoised_values(ev["ao16"], ev["bn16"], y)
    r = {"raw16": mae(ev["ao16"], clean_bn(ev["bn16"]), ev["lao"], ev["lbn"]),
         "denoised16": mae(ao, bn, ev["lao"], ev["lbn"])}
    if "pao" in ev:
        r["plain1024"] = mae(ev["pao"], clean_bn(ev["pbn"]), ev["lao"], ev["lbn"])
    return r


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-seeds", type=int, default=200)
    ap.add_argument("--eval-seeds", type=int, default=20)
    ap.add_argument("--texels-per-seed", type=int, default=16384)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--workers", type=int, default=min(16, os.cpu_count() or 1))
    ap.add_argument("--out", default=DEFAULT_OUT)
    args = ap.parse_args()
    train_seeds = list(range(100, 100 + args.train_seeds))
    eval_seeds = list(range(1000, 1000 + args.eval_seeds))
    pool = mp.get_context("spawn").Pool(args.workers)  # before any GPU use
    from . import api
    ctx = api.Context(0)
    label_table = ctx.upload(api.samples_cosine(LABEL, api.PERMS, 4242))
    plain_table = ctx.upload(api.samples_cosine(PLAIN, api.PERMS, 1717))
    t0 = time.time()
    train, evals = [], []
    seeds = train_seeds + eval_seeds
    for k, prepared in enumerate(prepared_in_order(pool, seeds, args.workers + 2)):
        sb = SeedBake(ctx, prepared)
        is_eval = prepared[0] in eval_seeds
        rec = collect(ctx, sb, args.texels_per_seed, label_table, plain_table if is_eval else None)
        (evals if is_eval else train).append(rec)
        sb.free()
        if k % 20 == 0:
            print("seed %d (%d/%d) %.0fs" % (prepared[0], k + 1, len(seeds), time.time() - t0), flush=True)
    pool.close()
    data_s = time.time() - t0
    x = np.concatenate([r["rows"] for r in train])
    t = np.concatenate([r["target"] for r in train])
    args.batch = min(args.batch, len(x) // 128 * 128)  # a multiple of the kernels' 128-row tile
    if args.batch == 0:
        raise SystemExit("fewer than 128 training rows")
    n_rows = len(x) // args.batch * args.batch
    rows, targets = ctx.upload(x), ctx.upload(t)
    ev = {k: np.concatenate([r[k] for r in evals]) for k in evals[0]}
    dn = api.Denoiser(ctx, init_params(1))
    steps_per_epoch = n_rows // args.batch
    total = steps_per_epoch * args.epochs
    rng = np.random.default_rng(2)
    history = []
    t1 = time.time()
    step = 0
    for epoch in range(args.epochs):
        perm = ctx.upload(rng.permutation(len(x))[:n_rows].astype(np.uint32))
        for s in range(steps_per_epoch):
            lr = args.lr * 0.5 * (1 + math.cos(math.pi * step / total)) + 1e-5
            dn.train_step(rows, targets, len(x), args.batch, row_ids=perm, offset=s * args.batch, lr=lr)
            step += 1
        loss = dn.last_loss()
        history.append(loss)
        if epoch % 10 == 0 or epoch == args.epochs - 1:
            print("epoch %d loss %.6f eval %s" % (epoch, loss, json.dumps(evaluate(ctx, dn, ev))), flush=True)
    ctx.check()
    train_s = time.time() - t1
    result = evaluate(ctx, dn, ev)
    meta = dict(train_seeds=train_seeds, eval_seeds=eval_seeds, texels_per_seed=args.texels_per_seed,
                rows=int(len(x)), epochs=args.epochs, batch=args.batch, lr=args.lr, low_samples=LOW,
                label_samples=LABEL, plain_samples=PLAIN, texture=TEX, min_distance=MIN_D, max_distance=MAX_D,
                data_seconds=round(data_s, 1), train_seconds=round(train_s, 1), steps=step, eval_mae=result)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    np.savez(args.out, params=dn.get_params(), loss=np.array(history, np.float64), meta=json.dumps(meta))
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
