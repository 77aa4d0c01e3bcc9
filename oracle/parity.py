"""Parity figures of a GPU bake against the reference's own outputs on the
same texels.

Test infrastructure only: used by tests/ and by bench.py's CPU-baseline leg,
which compare the GPU buffers of a bake with the outputs of the reference's
mapping and sampling shaders (oracle/_ref, or the oracle restatement) for a
set of texels, fed the same texel map, scene and sample table.

The bar (the ordered traversal's): texel map, hit indices and barycentrics
bit-exact; sampled outputs bit-exact except on at most 0.01 % of texels
(grazing hits on leaf-box faces), each occluder count within one sample.
"""
import numpy as np

MISS = 0xFFFFFFFF


def bits(a):
    """Bit patterns with every NaN mapped to one value (x86 and CUDA produce
    different NaN payloads for the same invalid operation)."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).copy()
    u[np.isnan(a)] = 0x7FC00000
    return u


def rows_differ(a, b):
    """Per row: any float of the row differs in its bits."""
    d = bits(a) != bits(b)
    return d.reshape(len(d), -1).any(axis=1)


def occluders_from_ao(ao, spp):
    """Occluder count of an AO value 1 - occ / spp (Shaders/ao_step2.comp):
    exact when spp is a power of two, since occ / spp and 1 - occ / spp are
    then exact in binary32."""
    if spp & (spp - 1):
        return None
    return np.rint((1.0 - np.asarray(ao, np.float64)) * spp).astype(np.int64)


def mapping(ref_coords, ref_tidx, gpu_coords, gpu_tidx):
    """Mapping figures over the compared texels."""
    t_diff = ref_tidx != gpu_tidx
    return {"texels": int(len(ref_tidx)), "hit_texels": int((ref_tidx != MISS).sum()),
            "tidx_diff_frac": float(t_diff.mean()) if len(t_diff) else 0.0,
            "coords_bits_diff_frac": float(rows_differ(ref_coords, gpu_coords).mean()) if len(t_diff) else 0.0}


def sampled(ref_out, gpu_out, hit, spp=None, ref_hits=None, gpu_hits=None):
    """Figures of one sampled output over the texels in `hit` (mapping hit,
    same hit index on both sides): fraction of texels whose output differs in
    any bit, and, where counts are known on both sides, the fraction whose
    count differs and the largest difference."""
    r = {"texels": int(hit.sum())}
    if not hit.any():
        return dict(r, out_diff_frac=0.0)
    r["out_diff_frac"] = float(rows_differ(ref_out[hit], gpu_out[hit]).mean())
    if ref_hits is None and spp is not None and np.ndim(ref_out) == 1:
        ref_hits = occluders_from_ao(ref_out, spp)
    if ref_hits is not None and gpu_hits is not None:
        d = np.abs(np.asarray(ref_hits, np.int64)[hit] - np.asarray(gpu_hits, np.int64)[hit])
        r["hits_diff_frac"] = float((d != 0).mean())
        r["max_hits_delta"] = int(d.max())
    return r


def meets_bar(report):
    """True when every figure of a parity report meets the bar."""
    m = report.get("mapping", {})
    if m.get("tidx_diff_frac", 0.0) != 0.0 or m.get("coords_bits_diff_frac", 0.0) != 0.0:
        return False
    for k, v in report.items():
        if k == "mapping" or not isinstance(v, dict):
            continue
        if v.get("out_diff_frac", 0.0) > 1e-4 or v.get("hits_diff_frac", 0.0) > 1e-4:
            return False
        if v.get("max_hits_delta", 0) > 1:
            return False
    return True
