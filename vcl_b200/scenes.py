"""Seeded synthetic scenes for the fit workloads (no asset files).

Meshes, attributes, textures, spherical-Gaussian lobes and cameras are built
here in NumPy with float64 math and handed to the device as float32, the way
the reference's host code prepares its inputs (camera and rotation matrices
are computed on the host in matrix.cu:43-58 and :175-222, then copied).

Conventions shared with the kernels:
* matrices are column-major float32[16] (element (row r, col c) at c*4+r),
  clip = MVP @ [x, y, z, 1];
* the projection is the reference's Camera::forward (matrix.cu:209-219) with
  ``size = znear * tan(fov/2)``, i.e. a standard GL perspective;
* ``pvinv`` is inverse(mat3(P) @ mat3(V)) column-major (material.cu:111).
"""
from __future__ import annotations

import functools
from dataclasses import dataclass, field

import numpy as np

ZNEAR = 0.1
ZFAR = 10.0


# ----------------------------------------------------------------- meshes
def icosphere(subdiv: int):
    """Unit icosphere: 10*4^s + 2 vertices, 20*4^s triangles."""
    v, f = _icosphere(subdiv)
    return v.copy(), f.copy()


@functools.lru_cache(maxsize=None)
def _icosphere(subdiv: int):
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
             (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = np.array(verts, dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(faces, dtype=np.int64)
    for _ in range(subdiv):
        nv = v.shape[0]
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], axis=0)
        e.sort(axis=1)
        key = e[:, 0] * (nv + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a = uniq // (nv + 1)
        b = uniq % (nv + 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        v = np.concatenate([v, mid], axis=0)
        nf = f.shape[0]
        m01 = nv + inv[:nf]
        m12 = nv + inv[nf:2 * nf]
        m20 = nv + inv[2 * nf:]
        f = np.concatenate([
            np.stack([f[:, 0], m01, m20], 1),
            np.stack([f[:, 1], m12, m01], 1),
            np.stack([f[:, 2], m20, m12], 1),
            np.stack([m01, m12, m20], 1)], axis=0)
    return v, f


def uv_sphere(nu: int, nv: int):
    """UV sphere with nu segments around and nv rings; pole quads become one
    triangle each: 2*nu*(nv-1) triangles."""
    lat = np.linspace(-np.pi / 2, np.pi / 2, nv + 1)
    lon = np.linspace(0.0, 2 * np.pi, nu, endpoint=False)
    la, lo = np.meshgrid(lat, lon, indexing="ij")
    v = np.stack([np.cos(la) * np.cos(lo), np.sin(la), np.cos(la) * np.sin(lo)], -1).reshape(-1, 3)
    idx = np.arange((nv + 1) * nu).reshape(nv + 1, nu)
    i0 = idx[:-1, :]
    i1 = np.roll(idx[:-1, :], -1, axis=1)
    i2 = idx[1:, :]
    i3 = np.roll(idx[1:, :], -1, axis=1)
    t1 = np.stack([i0, i2, i1], -1)[1:, :].reshape(-1, 3)      # skip south pole degenerate
    t2 = np.stack([i1, i2, i3], -1)[:-1, :].reshape(-1, 3)     # skip north pole degenerate
    return v, np.concatenate([t1, t2], 0)


def spherical_uv(pos):
    p = pos / np.linalg.norm(pos, axis=1, keepdims=True)
    u = np.arctan2(p[:, 2], p[:, 0]) / (2 * np.pi) + 0.5
    v = np.arcsin(np.clip(p[:, 1], -1, 1)) / np.pi + 0.5
    return np.stack([u, v], 1)


# ---------------------------------------------------------------- cameras
def random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
        [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
        [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def look_at(eye, center=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0)):
    eye = np.asarray(eye, np.float64)
    f = eye - np.asarray(center, np.float64)
    f /= np.linalg.norm(f)
    up = np.asarray(up, np.float64)
    if abs(np.dot(up, f)) > 0.99:
        up = np.array([1.0, 0.0, 0.0])
    s = np.cross(up, f)
    s /= np.linalg.norm(s)
    u = np.cross(f, s)
    m = np.eye(4)
    m[0, :3], m[1, :3], m[2, :3] = s, u, f
    m[:3, 3] = -m[:3, :3] @ eye
    return m


def perspective(fov_deg=45.0, znear=ZNEAR, zfar=ZFAR, aspect=1.0):
    size = znear * np.tan(np.radians(fov_deg) / 2)
    sy = znear / size
    sx = sy / aspect
    fn = zfar - znear
    p = np.zeros((4, 4))
    p[0, 0], p[1, 1] = sx, sy
    p[2, 2] = -(zfar + znear) / fn
    p[2, 3] = -2 * zfar * znear / fn
    p[3, 2] = -1.0
    return p


def colmajor(m):
    return np.ascontiguousarray(np.asarray(m, np.float64).T.reshape(-1)).astype(np.float32)


def random_dir(rng):
    d = rng.normal(size=3)
    return d / np.linalg.norm(d)


# ------------------------------------------------------------------ scene
@dataclass
class Scene:
    """All host-side arrays of one fit job (float32/uint32, C-contiguous)."""
    name: str
    W: int
    H: int
    views: int
    pos: np.ndarray          # (Nv,3) starting positions (what is optimized)
    pos_target: np.ndarray   # (Nv,3) positions of the target render
    tri: np.ndarray          # (T,3) uint32
    uv: np.ndarray           # (Nv,2)
    normal: np.ndarray       # (Nv,3) constant shading normals
    tex_w: int
    tex_h: int
    C: int
    levels: int
    tex_target: np.ndarray   # level-0 texels (th,tw,C)
    tex_init: np.ndarray     # level-0 texels the fit starts from
    K: int
    lobe_axis: np.ndarray    # (K,3)
    lobe_sharp: np.ndarray   # (K,)
    lobe_amp: np.ndarray     # (K,C)
    lobe_axis_init: np.ndarray
    lobe_sharp_init: np.ndarray
    lobe_amp_init: np.ndarray
    mvp: np.ndarray          # (views,16)
    pvinv: np.ndarray        # (views,9)
    rot: np.ndarray          # (16,) object rotation (NormalAxis)
    roughness: float = 0.5
    ior: float = 1.45
    noise: float = 0.05
    iters: int = 100
    lr: float = 1e-2
    lr_pos: float = 0.0        # Adam step on vertex positions (0: same as lr)
    seed: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def nv(self):
        return int(self.pos.shape[0])

    @property
    def nt(self):
        return int(self.tri.shape[0])


def tex_levels(tw, th, requested=16):
    """Texture::init's level count (buffer.cu:379-386): LSB(w|h)+1, <= 16."""
    v = tw | th
    lsb = (v & -v).bit_length() - 1
    return max(1, min(requested, min(16, lsb + 1)))


def make_scene(name, *, mesh, W, H, views, tex, K, dist=(3.0, 3.0), disp=0.0, seed=0,
               C=4, iters=100, fov=45.0, fixed_front_view=False, lr_pos=0.0):
    rng = np.random.default_rng(seed)
    if mesh[0] == "ico":
        v, f = icosphere(mesh[1])
    else:
        v, f = uv_sphere(mesh[1], mesh[2])
    normal = v / np.linalg.norm(v, axis=1, keepdims=True)
    uv = spherical_uv(v)
    pos_target = v + normal * rng.normal(0.0, disp, size=(v.shape[0], 1)) if disp > 0 else v.copy()
    R = random_rotation(rng)
    P = perspective(fov)
    R4 = np.eye(4)
    R4[:3, :3] = R
    mvps, pvinvs = [], []
    for i in range(views):
        d = rng.uniform(dist[0], dist[1])
        eye = np.array([0.0, 0.0, d]) if (fixed_front_view and i == 0) else random_dir(rng) * d
        V = look_at(eye)
        mvps.append(colmajor(P @ V @ R4))
        pvinvs.append(np.ascontiguousarray(np.linalg.inv(P[:3, :3] @ V[:3, :3]).T.reshape(-1)).astype(np.float32))
    levels = tex_levels(tex, tex)
    tex_target = rng.random((tex, tex, C), dtype=np.float64).astype(np.float32)
    tex_init = np.full((tex, tex, C), 0.5, np.float32)
    axis = np.stack([random_dir(rng) for _ in range(K)])
    sharp = rng.uniform(2.0, 20.0, size=K)
    amp = rng.uniform(0.0, 1.0, size=(K, C))
    axis_init = axis + rng.normal(0, 0.05, size=axis.shape)
    axis_init /= np.linalg.norm(axis_init, axis=1, keepdims=True)
    sharp_init = sharp * rng.uniform(0.9, 1.1, size=K)
    amp_init = np.clip(amp + rng.normal(0, 0.05, size=amp.shape), 0, 1)
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    return Scene(
        name=name, W=W, H=H, views=views,
        pos=f32(v), pos_target=f32(pos_target), tri=np.ascontiguousarray(f, dtype=np.uint32),
        uv=f32(uv), normal=f32(normal), tex_w=tex, tex_h=tex, C=C, levels=levels,
        tex_target=tex_target, tex_init=tex_init, K=K,
        lobe_axis=f32(axis), lobe_sharp=f32(sharp), lobe_amp=f32(amp),
        lobe_axis_init=f32(axis_init), lobe_sharp_init=f32(sharp_init), lobe_amp_init=f32(amp_init),
        mvp=np.stack(mvps).astype(np.float32), pvinv=np.stack(pvinvs).astype(np.float32),
        rot=colmajor(R4), iters=iters, seed=seed, lr_pos=lr_pos)


def vertex_normals(pos, tri):
    """Area-weighted vertex normals (for meshes whose file has none)."""
    p = np.asarray(pos, np.float64)
    f = np.asarray(tri, np.int64)
    n = np.cross(p[f[:, 1]] - p[f[:, 0]], p[f[:, 2]] - p[f[:, 0]])
    out = np.zeros_like(p)
    for k in range(3):
        np.add.at(out, f[:, k], n)
    ln = np.linalg.norm(out, axis=1, keepdims=True)
    return out / np.where(ln > 0, ln, 1.0)


def scene_from_assets(name, mesh, texture, lobes, *, W, H, views, dist=(2.5, 4.0), seed=0, C=4, iters=100,
                      fov=45.0, lr_pos=0.0, tex_init=0.5):
    """A fit job from loaded assets (vcl_b200.capi.load_obj / load_bmp /
    load_sg): the welded mesh (normals computed when the file has none),
    the image as the target texture (channels padded with 1 up to C; the
    fit starts from a constant texture), the lobes as the target lighting
    (amplitude channels padded with 0; the fit starts from the same lobes),
    seeded cameras around the mesh's bounding sphere."""
    rng = np.random.default_rng(seed)
    pos = np.asarray(mesh["w_pos"], np.float64)
    tri = np.ascontiguousarray(mesh["w_tri"], dtype=np.uint32)
    ctr = 0.5 * (pos.min(0) + pos.max(0))
    rad = max(float(np.linalg.norm(pos - ctr, axis=1).max()), 1e-6)
    v = (pos - ctr) / rad                       # unit bounding sphere at the origin
    nrm = np.asarray(mesh["w_normal"], np.float64)
    if not np.any(nrm):
        nrm = vertex_normals(v, tri)
    uv = np.asarray(mesh["w_uv"], np.float64)
    img = np.asarray(texture, np.float32)
    if img.ndim == 2:
        img = img[..., None]
    th, tw = img.shape[:2]
    if img.shape[2] < C:
        img = np.concatenate([img, np.ones((th, tw, C - img.shape[2]), np.float32)], axis=2)
    img = np.ascontiguousarray(img[..., :C])
    axis, sharp, amp = (np.asarray(x, np.float64) for x in lobes)
    K = axis.shape[0]
    if amp.shape[1] < C:
        amp = np.concatenate([amp, np.zeros((K, C - amp.shape[1]))], axis=1)
    amp = amp[:, :C]
    R = random_rotation(rng)
    P = perspective(fov)
    R4 = np.eye(4)
    R4[:3, :3] = R
    mvps, pvinvs = [], []
    for _ in range(views):
        V = look_at(random_dir(rng) * rng.uniform(dist[0], dist[1]))
        mvps.append(colmajor(P @ V @ R4))
        pvinvs.append(np.ascontiguousarray(np.linalg.inv(P[:3, :3] @ V[:3, :3]).T.reshape(-1)).astype(np.float32))
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    return Scene(
        name=name, W=W, H=H, views=views, pos=f32(v), pos_target=f32(v), tri=tri, uv=f32(uv), normal=f32(nrm),
        tex_w=tw, tex_h=th, C=C, levels=tex_levels(tw, th), tex_target=img,
        tex_init=np.full((th, tw, C), tex_init, np.float32), K=K,
        lobe_axis=f32(axis), lobe_sharp=f32(sharp), lobe_amp=f32(amp),
        lobe_axis_init=f32(axis), lobe_sharp_init=f32(sharp), lobe_amp_init=f32(amp),
        mvp=np.stack(mvps).astype(np.float32), pvinv=np.stack(pvinvs).astype(np.float32),
        rot=colmajor(R4), iters=iters, seed=seed, lr_pos=lr_pos)


# The five workloads (sizes as the fit configurations state them).  Adam
# runs at 1e-2 on texture and lobes; on vertex positions of the larger meshes
# at 1e-3 (each parameter group has its own Adam, as in the reference's
# preset): at 1e-2 a 65k-triangle sphere crumples within tens of iterations
# into large overlapping triangles.
LR_POS = 1e-3
def config1(seed=0):
    """Plain pipeline, small: icosphere s3, 256^2 x 1 view, 512^2 texture, 16 lobes."""
    return make_scene("ico3-256x1-tex512-K16", mesh=("ico", 3), W=256, H=256, views=1, tex=512, K=16,
                      dist=(3.0, 3.0), seed=seed, iters=100, fixed_front_view=True)


def config2(seed=0, views=8):
    """Plain pipeline at scale: UV sphere 256x128 (~65k tris) displaced N(0,0.02),
    8 views at 1024^2, 2048^2 texture (12 levels), 32 lobes."""
    return make_scene(f"uvs256x128-1024x{views}-tex2048-K32", mesh=("uv", 256, 128), W=1024, H=1024,
                      views=views, tex=2048, K=32, dist=(2.5, 4.0), disp=0.02, seed=seed, iters=200,
                      lr_pos=LR_POS)


CONFIG3_RES = (128, 256, 512, 1024)
CONFIG3_TEX = (256, 512, 1024, 2048)


def config3_scene(seed, index):
    """One scene of the uneven batched mix: icosphere whose triangle count is
    drawn log-uniform in [1k, 200k] (subdivision 3..6 nearest in log scale),
    N(0, 0.01) displacement, resolution from {128..1024}^2, 1-16 views,
    texture from {256..2048}^2 with a full mip chain, 8-32 lobes."""
    rng = np.random.default_rng([seed, index])
    T = float(np.exp(rng.uniform(np.log(1e3), np.log(2e5))))
    subdiv = int(np.clip(np.floor(np.log(T / 20.0) / np.log(4.0) + 0.5), 3, 6))
    res = int(rng.choice(CONFIG3_RES))
    views = int(rng.integers(1, 17))
    tex = int(rng.choice(CONFIG3_TEX))
    K = int(rng.integers(8, 33))
    sub_seed = int(rng.integers(0, 2 ** 31 - 1))
    return make_scene(f"mix{index}-ico{subdiv}-{res}x{views}-tex{tex}-K{K}", mesh=("ico", subdiv), W=res, H=res,
                      views=views, tex=tex, K=K, dist=(2.5, 4.0), disp=0.01, seed=sub_seed, iters=100,
                      lr_pos=LR_POS)


def config3(seed=0, n=64):
    """The batched uneven-scene workload: n scenes from config3_scene."""
    return [config3_scene(seed, i) for i in range(n)]


def config5(seed=0, views=4):
    """Dense stress: icosphere s8 (1.31M tris) displaced N(0,0.005), 4 views at
    2048^2, 4096^2 texture (13 levels), 64 lobes."""
    return make_scene(f"ico8-2048x{views}-tex4096-K64", mesh=("ico", 8), W=2048, H=2048, views=views, tex=4096,
                      K=64, dist=(2.5, 4.0), disp=0.005, seed=seed, iters=100, lr_pos=LR_POS)


def small(seed=0, W=32, H=24, views=2, subdiv=1, tex=16, K=3, C=4):
    """Tiny scene for oracle-speed parity checks."""
    return make_scene(f"tiny-{W}x{H}x{views}", mesh=("ico", subdiv), W=W, H=H, views=views, tex=tex,
                      K=K, C=C, dist=(2.2, 3.0), disp=0.02, seed=seed, iters=3)
