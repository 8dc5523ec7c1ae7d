"""Seeded procedural scenes for the benchmark and parity configurations.

All random choices come from SoL's PCG sampler (include/sol/samplers.h:20-65,
restated in `Pcg` below) with fixed seeds, so every scene is reproducible.

  cornell_box   : the Cornell box of the first configuration (10-triangle room,
                  2-triangle ceiling light, a glass box and a Phong box), and,
                  with `textured=True`, the adjoint configuration's variant with
                  256x256 value-noise albedo textures on the back wall and floor.
  sphere_field  : displaced spheres above a ground plane under four quad lights
                  (the large configurations).  No icosphere subdivision has
                  exactly 16,384 triangles (20*4^k), so each sphere is a UV sphere
                  of 65 latitude bands x 128 segments: two 128-triangle polar fans
                  plus 63 bands of 256 triangles = 16,384 triangles, which gives
                  the stated 1,048,576 (64 spheres) and 4,194,304 (256 spheres).
"""
from __future__ import annotations

import math

import numpy as np

from . import abi
from .scene import Bsdf, Camera, Config, Light, Scene, Texture

M32 = 0xFFFFFFFF
M64 = 0xFFFFFFFFFFFFFFFF


class Pcg:
    """SoL's PcgSampler: PCG-XSH-RR with its seeding, floats in [0, 1)."""

    def __init__(self, seed: int):
        self.state = 0
        self.next_u32()
        self.state = (self.state + seed) & M64
        self.next_u32()

    def next_u32(self) -> int:
        old = self.state
        self.state = (old * 6364136223846793005 + 1) & M64
        xs = (((old >> 18) ^ old) >> 27) & M32
        rot = old >> 59
        return ((xs >> rot) | (xs << ((-rot) & 31))) & M32

    def __call__(self) -> float:
        f = np.float32(self.next_u32()) * np.float32(2.0 ** -32)
        return float(min(f, np.float32(0.99999994)))

    def uniform(self, lo: float, hi: float) -> float:
        return lo + (hi - lo) * self()


# ---------------------------------------------------------------------------
# Value noise
# ---------------------------------------------------------------------------

def _hash(ix, iy, iz, seed):
    h = (ix.astype(np.uint32) * np.uint32(0x8DA6B343)) ^ (iy.astype(np.uint32) * np.uint32(0xD8163841)) \
        ^ (iz.astype(np.uint32) * np.uint32(0xCB1AB31F)) ^ np.uint32(seed * 0x9E3779B9 & M32)
    h ^= h >> np.uint32(16)
    h *= np.uint32(0x7FEB352D)
    h ^= h >> np.uint32(15)
    h *= np.uint32(0x846CA68B)
    h ^= h >> np.uint32(16)
    return h.astype(np.float64) / float(M32) * 2.0 - 1.0   # [-1, 1]


def value_noise(p: np.ndarray, seed: int) -> np.ndarray:
    """Lattice value noise in [-1, 1] with smoothstep interpolation; p is (N, 3) or (N, 2)."""
    if p.shape[1] == 2:
        p = np.concatenate([p, np.zeros((p.shape[0], 1))], axis=1)
    with np.errstate(over="ignore"):
        i = np.floor(p).astype(np.int64)
        f = p - i
        w = f * f * (3.0 - 2.0 * f)
        out = np.zeros(p.shape[0])
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    c = _hash(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
                    wx = w[:, 0] if dx else 1.0 - w[:, 0]
                    wy = w[:, 1] if dy else 1.0 - w[:, 1]
                    wz = w[:, 2] if dz else 1.0 - w[:, 2]
                    out += c * wx * wy * wz
    return out


def fractal_noise(p: np.ndarray, seed: int, octaves: int = 3) -> np.ndarray:
    """Sum of `octaves` value-noise octaves (frequency x2, amplitude /2), in [-1, 1]."""
    total = np.zeros(p.shape[0])
    amp, freq, norm = 1.0, 1.0, 0.0
    for o in range(octaves):
        total += amp * value_noise(p * freq, seed + 101 * o)
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def noise_texture(size: int, seed: int, lo: float = 0.1, hi: float = 0.9, cells: float = 8.0) -> np.ndarray:
    """(3, size, size) planar RGB texture of 3-octave value noise mapped to [lo, hi]."""
    ys, xs = np.meshgrid(np.arange(size), np.arange(size), indexing="ij")
    p = np.stack([xs.ravel(), ys.ravel()], axis=1).astype(np.float64) * (cells / size)
    chans = []
    for c in range(3):
        n = fractal_noise(p, seed * 7 + c)
        chans.append((lo + (hi - lo) * (0.5 + 0.5 * n)).reshape(size, size))
    return np.clip(np.stack(chans), lo, hi).astype(np.float32)


# ---------------------------------------------------------------------------
# Mesh helpers
# ---------------------------------------------------------------------------

class MeshBuilder:
    def __init__(self):
        self.v, self.n, self.t, self.i, self.b, self.l = [], [], [], [], [], []
        self.nv = 0

    def add(self, verts, normals, uvs, tris, bsdf: int, light_ids=None):
        verts = np.asarray(verts, np.float32)
        self.v.append(verts)
        self.n.append(np.asarray(normals, np.float32))
        self.t.append(np.asarray(uvs, np.float32))
        tris = np.asarray(tris, np.int64)
        self.i.append((tris + self.nv).astype(np.uint32))
        self.b.append(np.full(len(tris), bsdf, np.int32))
        self.l.append(np.full(len(tris), -1, np.int32) if light_ids is None else np.asarray(light_ids, np.int32))
        self.nv += len(verts)

    def quad(self, p0, p1, p2, p3, bsdf: int, uv=((0, 0), (1, 0), (1, 1), (0, 1)), light_ids=None):
        """Quad p0 p1 p2 p3 as triangles (p0, p1, p2) and (p0, p2, p3); flat normal (p1 - p0) x (p2 - p0)."""
        p = np.asarray([p0, p1, p2, p3], np.float64)
        nrm = np.cross(p[1] - p[0], p[2] - p[0])
        nrm /= np.linalg.norm(nrm)
        self.add(p, np.tile(nrm, (4, 1)), uv, [[0, 1, 2], [0, 2, 3]], bsdf, light_ids)

    def scene(self, **kw) -> Scene:
        return Scene(vertices=np.concatenate(self.v), normals=np.concatenate(self.n),
                     tex_coords=np.concatenate(self.t), indices=np.concatenate(self.i),
                     tri_bsdf=np.concatenate(self.b), tri_light=np.concatenate(self.l), **kw)


def _box(builder: MeshBuilder, center, size, angle: float, bsdf: int):
    """Closed box (12 triangles, outward normals) rotated by `angle` about +y."""
    cx, cy, cz = center
    sx, sy, sz = size
    ca, sa = math.cos(angle), math.sin(angle)

    def P(x, y, z):
        x, z = x * sx * 0.5, z * sz * 0.5
        return (cx + ca * x + sa * z, cy + y * sy * 0.5, cz - sa * x + ca * z)
    faces = [  # counter-clockwise seen from outside
        [(-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)],
        [(1, -1, -1), (-1, -1, -1), (-1, 1, -1), (1, 1, -1)],
        [(1, -1, 1), (1, -1, -1), (1, 1, -1), (1, 1, 1)],
        [(-1, -1, -1), (-1, -1, 1), (-1, 1, 1), (-1, 1, -1)],
        [(-1, 1, 1), (1, 1, 1), (1, 1, -1), (-1, 1, -1)],
        [(-1, -1, -1), (1, -1, -1), (1, -1, 1), (-1, -1, 1)],
    ]
    for f in faces:
        builder.quad(*[P(*c) for c in f], bsdf=bsdf)


# ---------------------------------------------------------------------------
# Configuration 0 / 3: Cornell box
# ---------------------------------------------------------------------------

def cornell_box(seed: int = 0, textured: bool = False, tex_size: int = 256, tex_seed: int = 3,
                textures_override=None) -> Scene:
    """Cornell box in the unit cube, open towards -z, camera at (0.5, 0.5, -1.4).

    Materials follow test/data/cornell_box.mtl of SoL: floor/ceiling/back 0.73
    grey, red (0.65, 0.05, 0.05) and green (0.12, 0.45, 0.15) side walls; a
    0.25 x 0.25 light 1e-4 below the ceiling emitting (17, 12, 4) downwards with
    a diffuse 0.78 surface.  A glass box (IOR 1.5, ks = kt = 1) and a Phong box
    (exponent 64, ks 0.5) stand on the floor at positions and y-rotations drawn
    from PcgSampler(seed).  With `textured`, the back wall and floor albedos are
    `tex_size`^2 RGB images (3-octave value noise in [0.1, 0.9]).
    """
    rng = Pcg(seed)
    tex = [
        Texture(abi.TEX_CONSTANT_COLOR, (0.73, 0.73, 0.73)),   # 0 white
        Texture(abi.TEX_CONSTANT_COLOR, (0.65, 0.05, 0.05)),   # 1 red
        Texture(abi.TEX_CONSTANT_COLOR, (0.12, 0.45, 0.15)),   # 2 green
        Texture(abi.TEX_CONSTANT_COLOR, (0.78, 0.78, 0.78)),   # 3 light surface
        Texture(abi.TEX_CONSTANT_COLOR, (17.0, 12.0, 4.0)),    # 4 emission
        Texture(abi.TEX_CONSTANT_COLOR, (1.0, 1.0, 1.0)),      # 5 glass ks / kt
        Texture(abi.TEX_CONSTANT, (1.0 / 1.5, 0.0, 0.0)),      # 6 glass eta (1 / IOR)
        Texture(abi.TEX_CONSTANT_COLOR, (0.5, 0.5, 0.5)),      # 7 phong ks
        Texture(abi.TEX_CONSTANT, (64.0, 0.0, 0.0)),           # 8 phong ns
    ]
    bsdfs = [
        Bsdf(abi.BSDF_DIFFUSE, (0, -1, -1)),    # 0 white
        Bsdf(abi.BSDF_DIFFUSE, (1, -1, -1)),    # 1 red
        Bsdf(abi.BSDF_DIFFUSE, (2, -1, -1)),    # 2 green
        Bsdf(abi.BSDF_DIFFUSE, (3, -1, -1)),    # 3 light surface
        Bsdf(abi.BSDF_GLASS, (5, 5, 6)),        # 4 glass
        Bsdf(abi.BSDF_PHONG, (7, 8, -1)),       # 5 phong
    ]
    images = []
    back_bsdf = floor_bsdf = 0
    if textured:
        if textures_override is not None:
            images = [np.asarray(t, np.float32) for t in textures_override]
        else:
            images = [noise_texture(tex_size, tex_seed), noise_texture(tex_size, tex_seed + 1)]
        tex += [Texture(abi.TEX_IMAGE, image=0, filter=abi.FILTER_BILINEAR, border=abi.BORDER_REPEAT),   # 9 back
                Texture(abi.TEX_IMAGE, image=1, filter=abi.FILTER_BILINEAR, border=abi.BORDER_REPEAT)]   # 10 floor
        bsdfs += [Bsdf(abi.BSDF_DIFFUSE, (9, -1, -1)), Bsdf(abi.BSDF_DIFFUSE, (10, -1, -1))]
        back_bsdf, floor_bsdf = 6, 7

    mb = MeshBuilder()
    # Room (normals towards the inside).  The camera's right vector is
    # normalize(dir x up) = -x (src/cameras.cpp:14), so x = 1 is on the image's left.
    mb.quad((0, 0, 0), (0, 0, 1), (1, 0, 1), (1, 0, 0), floor_bsdf, uv=((0, 0), (0, 1), (1, 1), (1, 0)))      # floor
    mb.quad((0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1), 0)                                                    # ceiling
    mb.quad((0, 0, 1), (0, 1, 1), (1, 1, 1), (1, 0, 1), back_bsdf, uv=((0, 0), (0, 1), (1, 1), (1, 0)))       # back
    mb.quad((1, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0), 1)                                                    # red (x = 1)
    mb.quad((0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1), 2)                                                    # green (x = 0)
    # Light quad, emitting towards -y; one UniformTriangleLight per triangle.
    y = 1.0 - 1e-4
    l0, l1, l2, l3 = (0.375, y, 0.375), (0.625, y, 0.375), (0.625, y, 0.625), (0.375, y, 0.625)
    mb.quad(l0, l1, l2, l3, 3, light_ids=[0, 1])
    lights = [Light(abi.LIGHT_TRIANGLE, l0, l1, l2, intensity_tex=4),
              Light(abi.LIGHT_TRIANGLE, l0, l2, l3, intensity_tex=4)]
    # Boxes: glass 0.3^3 on the image's right half, Phong 0.3 x 0.6 x 0.3 on the left.
    gx, gz, ga = rng.uniform(0.22, 0.42), rng.uniform(0.25, 0.45), rng.uniform(0.0, math.pi / 2)
    px, pz, pa = rng.uniform(0.58, 0.78), rng.uniform(0.55, 0.75), rng.uniform(0.0, math.pi / 2)
    _box(mb, (gx, 0.15 + 1e-3, gz), (0.3, 0.3, 0.3), ga, 4)
    _box(mb, (px, 0.30 + 1e-3, pz), (0.3, 0.6, 0.3), pa, 5)
    cam = Camera(eye=(0.5, 0.5, -1.4), dir=(0.0, 0.0, 1.0), up=(0.0, 1.0, 0.0), fov=40.0, aspect=1.0)
    return mb.scene(textures=tex, bsdfs=bsdfs, lights=lights, images=images, camera=cam)


# ---------------------------------------------------------------------------
# Displaced-sphere scenes
# ---------------------------------------------------------------------------

def uv_sphere(bands: int = 65, segments: int = 128):
    """Unit UV sphere: vertices (N, 3), triangles (M, 3), uv (N, 2); M = 2*segments*(bands-1)."""
    verts = [(0.0, 1.0, 0.0)]
    uvs = [(0.5, 0.0)]
    for b in range(1, bands):
        th = math.pi * b / bands
        for s in range(segments):
            ph = 2.0 * math.pi * s / segments
            verts.append((math.sin(th) * math.cos(ph), math.cos(th), math.sin(th) * math.sin(ph)))
            uvs.append((s / segments, b / bands))
    verts.append((0.0, -1.0, 0.0))
    uvs.append((0.5, 1.0))
    south = len(verts) - 1

    def ring(b, s):
        return 1 + (b - 1) * segments + (s % segments)
    tris = []
    for s in range(segments):
        tris.append((0, ring(1, s + 1), ring(1, s)))
    for b in range(1, bands - 1):
        for s in range(segments):
            a, c = ring(b, s), ring(b, s + 1)
            d, e = ring(b + 1, s), ring(b + 1, s + 1)
            tris.append((a, c, e))
            tris.append((a, e, d))
    for s in range(segments):
        tris.append((south, ring(bands - 1, s), ring(bands - 1, s + 1)))
    return np.asarray(verts, np.float64), np.asarray(tris, np.int64), np.asarray(uvs, np.float64)


def _smooth_normals(v: np.ndarray, t: np.ndarray) -> np.ndarray:
    fn = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
    n = np.zeros_like(v)
    for k in range(3):
        np.add.at(n, t[:, k], fn)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    return n


def sphere_field(num_spheres: int = 64, seed: int = 1, bands: int = 65, segments: int = 128,
                 box: float = 10.0, aspect: float = 16.0 / 9.0, textured: bool = False, tex_size: int = 128,
                 sphere_sizes=None) -> Scene:
    """Displaced spheres in a `box`^3 volume above a 2-triangle ground, 4 quad lights.

    Per sphere (in draw order from PcgSampler(seed)): position x, y, z uniform in
    the box (y kept above the sphere's radius), scale U[0.05, 0.3], material
    choice uniform over {Diffuse, Phong, Glass}, then its parameters: albedo
    U[0.1, 0.9]^3, or Phong exponent log-uniform in [1, 1000] and ks U[0, 0.5],
    or IOR U[1.3, 1.8].  The radius is 1 + 0.1 * (3-octave value noise) of the
    unit direction.  Lights: four 2 x 2 quads at y = box + 1 facing down with
    white emission U[5, 20].  `sphere_sizes` optionally gives per-sphere
    (bands, segments) to vary the triangle count.
    """
    rng = Pcg(seed)
    tex, bsdfs, lights, images = [], [], [], []
    mb = MeshBuilder()
    # Ground: diffuse 0.5.
    tex.append(Texture(abi.TEX_CONSTANT_COLOR, (0.5, 0.5, 0.5)))
    bsdfs.append(Bsdf(abi.BSDF_DIFFUSE, (0, -1, -1)))
    g0, g1 = -2.0 * box, 3.0 * box
    mb.quad((g0, 0, g0), (g0, 0, g1), (g1, 0, g1), (g1, 0, g0), 0, uv=((0, 0), (0, 1), (1, 1), (1, 0)))
    if textured:
        images.append(noise_texture(tex_size, seed + 17))
        tex.append(Texture(abi.TEX_IMAGE, image=0, filter=abi.FILTER_BILINEAR, border=abi.BORDER_REPEAT))
        bsdfs.append(Bsdf(abi.BSDF_DIFFUSE, (len(tex) - 1, -1, -1)))
    cache = {}
    for k in range(num_spheres):
        px, py, pz = rng.uniform(0, box), rng(), rng.uniform(0, box)
        scale = rng.uniform(0.05, 0.3)
        py = scale * 1.2 + py * (box - scale * 1.2)
        kind = min(int(rng() * 3), 2)
        if kind == 0:
            albedo = (rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9))
            if textured and k % 2 == 0:
                b = 1   # the image-textured diffuse BSDF
            else:
                tex.append(Texture(abi.TEX_CONSTANT_COLOR, albedo))
                bsdfs.append(Bsdf(abi.BSDF_DIFFUSE, (len(tex) - 1, -1, -1)))
                b = len(bsdfs) - 1
        elif kind == 1:
            ns = math.exp(rng.uniform(0.0, math.log(1000.0)))
            ks = rng.uniform(0.0, 0.5)
            tex.append(Texture(abi.TEX_CONSTANT_COLOR, (ks, ks, ks)))
            tex.append(Texture(abi.TEX_CONSTANT, (ns, 0.0, 0.0)))
            bsdfs.append(Bsdf(abi.BSDF_PHONG, (len(tex) - 2, len(tex) - 1, -1)))
            b = len(bsdfs) - 1
        else:
            ior = rng.uniform(1.3, 1.8)
            tex.append(Texture(abi.TEX_CONSTANT_COLOR, (1.0, 1.0, 1.0)))
            tex.append(Texture(abi.TEX_CONSTANT, (1.0 / ior, 0.0, 0.0)))
            bsdfs.append(Bsdf(abi.BSDF_GLASS, (len(tex) - 2, len(tex) - 2, len(tex) - 1)))
            b = len(bsdfs) - 1
        nb, ns_ = sphere_sizes[k] if sphere_sizes is not None else (bands, segments)
        if (nb, ns_) not in cache:
            cache[(nb, ns_)] = uv_sphere(nb, ns_)
        uv_v, uv_t, uv_uv = cache[(nb, ns_)]
        disp = 1.0 + 0.1 * fractal_noise(uv_v * 2.0 + 13.0 * k, seed * 1000 + k)
        v = uv_v * (disp * scale)[:, None] + np.array([px, py, pz])
        mb.add(v, _smooth_normals(v, uv_t), uv_uv, uv_t, b)
    tex.append(Texture(abi.TEX_CONSTANT_COLOR, (0.8, 0.8, 0.8)))
    light_surface = len(bsdfs)
    bsdfs.append(Bsdf(abi.BSDF_DIFFUSE, (len(tex) - 1, -1, -1)))
    y = box + 1.0
    for cx, cz in ((0.25, 0.25), (0.75, 0.25), (0.25, 0.75), (0.75, 0.75)):
        e = rng.uniform(5.0, 20.0)
        tex.append(Texture(abi.TEX_CONSTANT_COLOR, (e, e, e)))
        x0, x1 = cx * box - 1.0, cx * box + 1.0
        z0, z1 = cz * box - 1.0, cz * box + 1.0
        q = ((x0, y, z0), (x1, y, z0), (x1, y, z1), (x0, y, z1))   # faces -y
        base = len(lights)
        mb.quad(*q, light_surface, light_ids=[base, base + 1])
        lights.append(Light(abi.LIGHT_TRIANGLE, q[0], q[1], q[2], intensity_tex=len(tex) - 1))
        lights.append(Light(abi.LIGHT_TRIANGLE, q[0], q[2], q[3], intensity_tex=len(tex) - 1))
    cam = Camera(eye=(0.5 * box, 0.7 * box, -0.7 * box), dir=(0.0, -0.4 * box, 1.2 * box), up=(0.0, 1.0, 0.0),
                 fov=60.0, aspect=aspect)
    return mb.scene(textures=tex, bsdfs=bsdfs, lights=lights, images=images, camera=cam)


def view_set(num_views: int = 64, seed: int = 2, box: float = 10.0, min_side: int = 64, max_side: int = 1024,
             max_spp: int = 64):
    """Seeded cameras into a sphere field of extent `box`: (Camera, side, spp) per view.

    Per view, in draw order from Pcg(seed): square film side log-uniform in
    [min_side, max_side], spp uniform in {1..max_spp}, eye on a ring around the
    field (angle, radius 0.6-1.0 box, height 0.2-0.8 box), look-at point in the
    middle of the field, field of view U[40, 70] degrees.
    """
    rng = Pcg(seed)
    out = []
    for _ in range(num_views):
        side = int(round(math.exp(rng.uniform(math.log(min_side), math.log(max_side)))))
        spp = 1 + min(int(rng() * max_spp), max_spp - 1)
        ang = rng.uniform(0.0, 2.0 * math.pi)
        r = rng.uniform(0.6, 1.0) * box
        hgt = rng.uniform(0.2, 0.8) * box
        eye = (0.5 * box + r * math.cos(ang), hgt, 0.5 * box + r * math.sin(ang))
        at = (rng.uniform(0.3, 0.7) * box, rng.uniform(0.0, 0.3) * box, rng.uniform(0.3, 0.7) * box)
        fov = rng.uniform(40.0, 70.0)
        cam = Camera(eye=eye, dir=tuple(a - e for a, e in zip(at, eye)), up=(0.0, 1.0, 0.0), fov=fov, aspect=1.0)
        out.append((cam, side, spp))
    return out


def scene_set_plan(num_scenes: int = 32, seed: int = 4, min_tris: int = 10_000, max_tris: int = 2_000_000,
                   min_side: int = 128, max_side: int = 512):
    """The sizes scene_set draws: (spheres, segments, side) per scene.

    Per scene, in draw order from Pcg(seed): a triangle budget log-uniform in
    [min_tris, max_tris] and a square film side log-uniform in [min_side,
    max_side].  The budget is met with n = clamp(budget / 16384, 2, 128) spheres
    of seg^2 triangles each (seg segments, seg/2 + 1 bands), seg the even number
    nearest sqrt(budget / n)."""
    rng = Pcg(seed)
    out = []
    for _ in range(num_scenes):
        budget = math.exp(rng.uniform(math.log(min_tris), math.log(max_tris)))
        side = int(round(math.exp(rng.uniform(math.log(min_side), math.log(max_side)))))
        n = max(2, min(128, int(round(budget / 16384))))
        seg = max(6, 2 * int(round(math.sqrt(budget / n) / 2)))
        out.append((n, seg, side))
    return out


def scene_set(num_scenes: int = 32, seed: int = 4, min_tris: int = 10_000, max_tris: int = 2_000_000,
              min_side: int = 128, max_side: int = 512, tex_size: int = 128, only=None):
    """Independent textured sphere fields of uneven size (sizes from
    scene_set_plan): (Scene, side) per scene.  Every scene has its own
    tex_size^2 RGB albedo image (ground and half of the diffuse spheres) and
    its own light emission.  `only`: indices of the scenes to build (scene k is
    the same scene either way); they come back in index order.
    """
    out = []
    for k, (n, seg, side) in enumerate(scene_set_plan(num_scenes, seed, min_tris, max_tris, min_side, max_side)):
        if only is not None and k not in only:
            continue
        sizes = [(seg // 2 + 1, seg)] * n
        out.append((sphere_field(n, seed=100 + k, textured=True, tex_size=tex_size, sphere_sizes=sizes,
                                 aspect=1.0), side))
    return out


# ---------------------------------------------------------------------------
# Named frames
# ---------------------------------------------------------------------------

CORNELL_CONFIG = Config(max_path_len=16, min_rr_path_len=3, min_survival_prob=0.05, max_survival_prob=0.75,
                        ray_offset=1e-5)
SPHERES_CONFIG = Config(max_path_len=8, min_rr_path_len=3, min_survival_prob=0.05, max_survival_prob=0.75,
                        ray_offset=1e-4)


def cornell_frame():
    """Cornell box, 256^2, 16 spp, max path length 16, RR from bounce 3."""
    return cornell_box(0), CORNELL_CONFIG, 256, 256, 16


def sphere_field_frame():
    """1,048,576-triangle sphere field, 1920x1080, 64 spp, max path length 8."""
    return sphere_field(64, seed=1), SPHERES_CONFIG, 1920, 1080, 64
