"""Seeded synthetic meshes for the bake workloads.

No sample meshes ship with Fornos, so every workload is generated here from an
explicit seed (numpy, float32 output).  Meshes use the reference's indexed form
(Src/mesh.h:35-63): per-vertex (position, texcoord, normal) indices and
per-triangle vertex indices, so seams can share positions while keeping
separate texcoords.

Workloads (sizes as named in the bake configurations):
  sphere_pair      512x512 bake: unit UV sphere 32x16 low-poly, 512x256 UV
                   sphere high-poly with r = 1 + 0.03 * sum_k sin(f_k*theta +
                   g_k*phi + p_k), k = 1..8.
  plane_pair       2048x2048 bake: 64x64-quad plane low-poly, 1024x1024-quad
                   heightfield (4-octave value noise + 200 hemispherical bumps).
  icosphere_pair   4096x4096 bake: subdivision-3 icosphere low-poly with
                   cube-projection UVs, subdivision-9 icosphere high-poly with
                   6-octave gradient-noise displacement.

High-poly normals are left for the caller to compute with the host's
Mesh::computeVertexNormals equivalent (Src/mesh.cpp:650-678), as the
reference runner does for NormalImport::ComputePerVertex.
"""
import numpy as np


class MeshArrays:
    """Indexed triangle mesh (float32 / uint32 numpy arrays)."""

    def __init__(self, positions, texcoords, normals, vertices, triangles, tangents=None, bitangents=None):
        self.positions = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
        self.texcoords = np.ascontiguousarray(texcoords, dtype=np.float32).reshape(-1, 2)
        self.normals = np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3)
        self.vertices = np.ascontiguousarray(vertices, dtype=np.uint32).reshape(-1, 3)
        self.triangles = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
        self.tangents = None if tangents is None else np.ascontiguousarray(tangents, dtype=np.float32).reshape(-1, 3)
        self.bitangents = None if bitangents is None else np.ascontiguousarray(bitangents, dtype=np.float32).reshape(-1, 3)

    @property
    def triangle_count(self):
        return int(self.triangles.shape[0])

    def copy(self):
        return MeshArrays(self.positions.copy(), self.texcoords.copy(), self.normals.copy(), self.vertices.copy(),
                          self.triangles.copy(),
                          None if self.tangents is None else self.tangents.copy(),
                          None if self.bitangents is None else self.bitangents.copy())


def _grid_vertices(nu, nv):
    """Vertex table for a (nu+1) x (nv+1) lattice where vertex (i, j) uses
    texcoord (i, j); position / normal indices are filled by the caller."""
    j, i = np.meshgrid(np.arange(nv + 1), np.arange(nu + 1), indexing="ij")
    return i.ravel(), j.ravel()


def uv_sphere(seg_u, seg_v, radius_fn=None):
    """UV sphere with equirectangular texcoords u = i / seg_u, v = j / seg_v.

    Rings j = 1 .. seg_v - 1 carry seg_u positions each (the seam shares
    positions, texcoords are duplicated); the poles are single positions.
    Triangles: 2 * seg_u * (seg_v - 1) (fans at both poles).
    radius_fn(theta, phi) -> radius, theta = polar angle, phi = azimuth.
    Normals: the radial direction (exact for the unit sphere)."""
    th = np.arange(1, seg_v, dtype=np.float64) * (np.pi / seg_v)
    ph = np.arange(seg_u, dtype=np.float64) * (2.0 * np.pi / seg_u)
    T, P = np.meshgrid(th, ph, indexing="ij")
    r = np.ones_like(T) if radius_fn is None else radius_fn(T, P)
    ring = np.stack([r * np.sin(T) * np.cos(P), r * np.sin(T) * np.sin(P), r * np.cos(T)], -1).reshape(-1, 3)
    r_n = 1.0 if radius_fn is None else float(radius_fn(np.array(0.0), np.array(0.0)))
    r_s = 1.0 if radius_fn is None else float(radius_fn(np.array(np.pi), np.array(0.0)))
    north = np.array([[0.0, 0.0, r_n]])
    south = np.array([[0.0, 0.0, -r_s]])
    pos = np.concatenate([ring, north, south]).astype(np.float32)
    n_ring = ring.shape[0]
    pn, ps = n_ring, n_ring + 1
    nrm = pos / np.linalg.norm(pos.astype(np.float64), axis=1, keepdims=True)

    ii, jj = _grid_vertices(seg_u, seg_v)
    uv = np.stack([ii / seg_u, jj / seg_v], -1)
    vid = lambda i, j: j * (seg_u + 1) + i
    pidx = np.empty(ii.shape, dtype=np.int64)
    inner = (jj > 0) & (jj < seg_v)
    pidx[inner] = (jj[inner] - 1) * seg_u + (ii[inner] % seg_u)
    pidx[jj == 0] = pn
    pidx[jj == seg_v] = ps
    verts = np.stack([pidx, np.arange(ii.size), pidx], -1)

    tris = []
    i = np.arange(seg_u)
    tris.append(np.stack([vid(i, 0), vid(i, 1), vid(i + 1, 1)], -1))
    for j in range(1, seg_v - 1):
        a, b, c, d = vid(i, j), vid(i + 1, j), vid(i, j + 1), vid(i + 1, j + 1)
        tris.append(np.stack([a, c, d], -1))
        tris.append(np.stack([a, d, b], -1))
    j = seg_v - 1
    tris.append(np.stack([vid(i, j), vid(i, j + 1), vid(i + 1, j)], -1))
    tris = np.concatenate(tris)
    return MeshArrays(pos, uv, nrm, verts, tris)


def grid_plane(nq, size=1.0, heights=None):
    """nq x nq-quad plane over [0, size]^2 in z = 0 (or z = heights[(nq+1)^2]),
    texcoords (x, y) / size, normal +z.  Positions are shared per lattice
    point; 2 * nq^2 triangles."""
    ii, jj = _grid_vertices(nq, nq)
    x = ii.astype(np.float64) * (size / nq)
    y = jj.astype(np.float64) * (size / nq)
    z = np.zeros_like(x) if heights is None else np.asarray(heights, dtype=np.float64).ravel()
    pos = np.stack([x, y, z], -1).astype(np.float32)
    uv = np.stack([ii / nq, jj / nq], -1)
    nrm = np.array([[0.0, 0.0, 1.0]], dtype=np.float32)
    n = ii.size
    verts = np.stack([np.arange(n), np.arange(n), np.zeros(n, dtype=np.int64)], -1)
    i, j = np.meshgrid(np.arange(nq), np.arange(nq), indexing="xy")
    a = (j * (nq + 1) + i).ravel()
    b, c, d = a + 1, a + nq + 1, a + nq + 2
    tris = np.concatenate([np.stack([a, b, d], -1), np.stack([a, d, c], -1)])
    order = np.stack([np.arange(a.size), np.arange(a.size) + a.size], -1).ravel()
    return MeshArrays(pos, uv, nrm, verts, tris[order])


# ------------------------------------------------------------------ noise
def value_noise_2d(x, y, octaves, freq0, lacunarity, gain, rng):
    """Sum of octaves of lattice value noise with smoothstep interpolation;
    lattice values uniform in [-1, 1) drawn from `rng` per octave."""
    out = np.zeros_like(x)
    amp, freq = 1.0, freq0
    for _ in range(octaves):
        n = int(np.ceil(freq)) + 2
        lat = rng.uniform(-1.0, 1.0, size=(n, n))
        fx, fy = x * freq, y * freq
        ix, iy = np.floor(fx).astype(np.int64), np.floor(fy).astype(np.int64)
        tx, ty = fx - ix, fy - iy
        sx, sy = tx * tx * (3 - 2 * tx), ty * ty * (3 - 2 * ty)
        ix, iy = np.clip(ix, 0, n - 2), np.clip(iy, 0, n - 2)
        v00, v10 = lat[iy, ix], lat[iy, ix + 1]
        v01, v11 = lat[iy + 1, ix], lat[iy + 1, ix + 1]
        out += amp * ((v00 * (1 - sx) + v10 * sx) * (1 - sy) + (v01 * (1 - sx) + v11 * sx) * sy)
        amp *= gain
        freq *= lacunarity
    return out


def gradient_noise_3d(p, octaves, freq0, rng, lacunarity=2.0, gain=0.5):
    """Perlin-style gradient noise, `octaves` octaves; gradient table of 256
    random unit vectors and a random permutation per octave."""
    out = np.zeros(p.shape[0])
    amp, freq = 1.0, freq0
    for _ in range(octaves):
        g = rng.normal(size=(256, 3))
        g /= np.linalg.norm(g, axis=1, keepdims=True)
        perm = rng.permutation(256)
        q = p * freq
        i0 = np.floor(q).astype(np.int64)
        f = q - i0
        w = f * f * f * (f * (f * 6 - 15) + 10)
        acc = np.zeros(p.shape[0])
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    h = perm[(perm[(perm[(i0[:, 0] + dx) & 255] + i0[:, 1] + dy) & 255] + i0[:, 2] + dz) & 255]
                    dv = f - np.array([dx, dy, dz], dtype=np.float64)
                    val = np.einsum("ij,ij->i", g[h], dv)
                    wx = w[:, 0] if dx else 1 - w[:, 0]
                    wy = w[:, 1] if dy else 1 - w[:, 1]
                    wz = w[:, 2] if dz else 1 - w[:, 2]
                    acc += wx * wy * wz * val
        out += amp * acc
        amp *= gain
        freq *= lacunarity
    return out


# ------------------------------------------------------------------ icosphere
def icosphere(subdiv):
    """Unit icosphere: 20 * 4^subdiv triangles, shared positions (float64)."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    for _ in range(subdiv):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (v.shape[0] + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // (v.shape[0] + 1), uniq % (v.shape[0] + 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = v.shape[0] + inv.reshape(3, -1).T  # (nf, 3): mids of edges 01, 12, 20
        v = np.concatenate([v, mid])
        f = np.concatenate([np.stack([f[:, 0], m[:, 0], m[:, 2]], -1), np.stack([f[:, 1], m[:, 1], m[:, 0]], -1),
                            np.stack([f[:, 2], m[:, 2], m[:, 1]], -1), m])
    return v, f


def cube_projection_uvs(pos, tris, margin=0.02):
    """Per-triangle cube projection into a 3 x 2 atlas: each triangle is
    assigned to the cube face of its centroid's dominant axis and its corners
    are projected onto that face.  Returns (texcoords[3 * nf, 2], per-corner
    texcoord index [nf, 3])."""
    c = pos[tris].mean(axis=1)
    ax = np.argmax(np.abs(c), axis=1)
    sgn = np.sign(c[np.arange(len(c)), ax])
    face = ax * 2 + (sgn < 0)
    p = pos[tris]  # nf, 3, 3
    u_ax = np.array([1, 2, 0])[ax]
    v_ax = np.array([2, 0, 1])[ax]
    den = np.abs(p[np.arange(len(c)), :, ax])
    uu = p[np.arange(len(c))[:, None], np.arange(3)[None, :], u_ax[:, None]] / den
    vv = p[np.arange(len(c))[:, None], np.arange(3)[None, :], v_ax[:, None]] / den
    tile_u, tile_v = (face % 3).astype(np.float64), (face // 3).astype(np.float64)
    s = (1.0 - 2 * margin)
    u = (tile_u[:, None] + margin + s * (np.clip(uu, -1, 1) * 0.5 + 0.5)) / 3.0
    v = (tile_v[:, None] + margin + s * (np.clip(vv, -1, 1) * 0.5 + 0.5)) / 2.0
    uv = np.stack([u, v], -1).reshape(-1, 2)
    return uv, np.arange(3 * len(c)).reshape(-1, 3)


# ------------------------------------------------------------------ workloads
def sphere_pair(seed=1, lo_seg=(32, 16), hi_seg=(512, 256)):
    rng = np.random.default_rng(seed)
    f = rng.integers(2, 17, size=8)
    g = rng.integers(2, 17, size=8)
    p = rng.uniform(0.0, 2 * np.pi, size=8)

    def radius(theta, phi):
        acc = np.zeros(np.shape(theta))
        for k in range(8):
            acc = acc + np.sin(f[k] * theta + g[k] * phi + p[k])
        return 1.0 + 0.03 * acc

    lo = uv_sphere(*lo_seg)
    hi = uv_sphere(*hi_seg, radius_fn=radius)
    return lo, hi


def plane_pair(seed=1, lo_quads=64, hi_quads=1024, bumps=200):
    rng = np.random.default_rng(seed)
    lo = grid_plane(lo_quads)
    n = hi_quads + 1
    ii, jj = _grid_vertices(hi_quads, hi_quads)
    x, y = ii / hi_quads, jj / hi_quads
    z = 0.05 * value_noise_2d(x, y, 4, 4.0, 2.0, 0.5, rng)
    cx, cy = rng.uniform(0, 1, bumps), rng.uniform(0, 1, bumps)
    rad = rng.uniform(0.01, 0.05, bumps)
    for k in range(bumps):
        d2 = (x - cx[k]) ** 2 + (y - cy[k]) ** 2
        z = z + np.sqrt(np.maximum(rad[k] ** 2 - d2, 0.0))
    hi = grid_plane(hi_quads, heights=z.reshape(n, n))
    return lo, hi


def icosphere_pair(seed=1, lo_subdiv=3, hi_subdiv=9):
    rng = np.random.default_rng(seed)
    v, f = icosphere(hi_subdiv)
    disp = 0.04 * gradient_noise_3d(v, 6, 2.0, rng)
    hv = (v * (1.0 + disp)[:, None]).astype(np.float32)
    nv = hv.shape[0]
    hi = MeshArrays(hv, np.zeros((1, 2)), v.astype(np.float32),
                    np.stack([np.arange(nv), np.zeros(nv, dtype=np.int64), np.arange(nv)], -1), f)
    lv, lf = icosphere(lo_subdiv)
    uv, uvidx = cube_projection_uvs(lv, lf)
    corners = np.stack([lf.ravel(), uvidx.ravel(), lf.ravel()], -1)
    lo = MeshArrays(lv.astype(np.float32), uv, lv.astype(np.float32), corners,
                    np.arange(corners.shape[0]).reshape(-1, 3))
    return lo, hi
