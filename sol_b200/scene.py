"""Flat scene description on the host (the contents of one sol::Scene whose root
is a TriangleMesh) and its conversion to the C ABI's SolGpuSceneDesc.

A scene is a set of numpy arrays plus small tables of textures, BSDFs, lights
and images, exactly the data SoL's OBJ loader feeds to the TriangleMesh,
Bsdf, Light and Texture constructors (src/formats/obj.cpp:375-516).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi


@dataclass
class Texture:
    type: int
    value: tuple = (0.0, 0.0, 0.0)
    image: int = -1
    filter: int = abi.FILTER_BILINEAR
    border: int = abi.BORDER_REPEAT


@dataclass
class Bsdf:
    type: int
    tex: tuple = (-1, -1, -1)
    a: int = -1
    b: int = -1


@dataclass
class Light:
    type: int
    v0: tuple = (0.0, 0.0, 0.0)
    v1: tuple = (0.0, 0.0, 0.0)
    v2: tuple = (0.0, 0.0, 0.0)
    intensity_tex: int = -1
    intensity: tuple = (0.0, 0.0, 0.0)


@dataclass
class Camera:
    """sol::PerspectiveCamera arguments (src/cameras.cpp:5-21)."""
    eye: tuple
    dir: tuple
    up: tuple
    fov: float
    aspect: float

    def to_c(self) -> abi.SolGpuCamera:
        """The constructed camera (sol_gpu_camera_perspective)."""
        from . import capi   # loads the CUDA library's C ABI
        c = abi.SolGpuCamera()
        v3 = C.c_float * 3
        capi.check(capi.lib.sol_gpu_camera_perspective(v3(*self.eye), v3(*self.dir), v3(*self.up), self.fov,
                                                       self.aspect, C.byref(c)), "sol_gpu_camera_perspective")
        return c


@dataclass
class Config:
    """sol::PathTracer::Config (include/sol/algorithms/path_tracer.h:23-29)."""
    max_path_len: int = 64
    min_rr_path_len: int = 3
    min_survival_prob: float = 0.05
    max_survival_prob: float = 0.75
    ray_offset: float = 1e-5

    def to_c(self) -> abi.SolGpuConfig:
        c = abi.SolGpuConfig()
        c.max_path_len = self.max_path_len
        c.min_rr_path_len = self.min_rr_path_len
        c.min_survival_prob = self.min_survival_prob
        c.max_survival_prob = self.max_survival_prob
        c.ray_offset = self.ray_offset
        return c


@dataclass
class Scene:
    vertices: np.ndarray            # (nv, 3) float32
    normals: np.ndarray             # (nv, 3) float32
    tex_coords: np.ndarray          # (nv, 2) float32
    indices: np.ndarray             # (nt, 3) uint32
    tri_bsdf: np.ndarray            # (nt,) int32
    tri_light: np.ndarray           # (nt,) int32
    textures: list = field(default_factory=list)
    bsdfs: list = field(default_factory=list)
    lights: list = field(default_factory=list)
    images: list = field(default_factory=list)   # each (3, h, w) float32, planar RGB
    camera: Camera | None = None

    @property
    def num_triangles(self) -> int:
        return int(self.indices.shape[0])

    def desc(self, bvh=None) -> "SceneDesc":
        """C descriptor; `bvh` = (node array, node count, prim indices) from build_bvh() to pass a prebuilt BVH."""
        return SceneDesc(self, bvh)


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class SceneDesc:
    """Keeps the arrays alive for as long as the ctypes descriptor is used."""

    def __init__(self, s: Scene, bvh=None):
        self.v = np.ascontiguousarray(s.vertices, dtype=np.float32)
        self.n = np.ascontiguousarray(s.normals, dtype=np.float32)
        self.t = np.ascontiguousarray(s.tex_coords, dtype=np.float32)
        self.i = np.ascontiguousarray(s.indices, dtype=np.uint32)
        self.b = np.ascontiguousarray(s.tri_bsdf, dtype=np.int32)
        self.l = np.ascontiguousarray(s.tri_light, dtype=np.int32)
        self.imgs = [np.ascontiguousarray(im, dtype=np.float32) for im in s.images]
        d = abi.SolGpuSceneDesc()
        d.num_vertices = self.v.shape[0]
        d.num_triangles = self.i.shape[0]
        d.vertices = _ptr(self.v, C.c_float)
        d.normals = _ptr(self.n, C.c_float)
        d.tex_coords = _ptr(self.t, C.c_float)
        d.indices = _ptr(self.i, C.c_uint32)
        d.tri_bsdf = _ptr(self.b, C.c_int32)
        d.tri_light = _ptr(self.l, C.c_int32)
        self.tex_arr = (abi.SolGpuTexture * max(1, len(s.textures)))()
        for k, t in enumerate(s.textures):
            self.tex_arr[k].type = t.type
            self.tex_arr[k].filter = t.filter
            self.tex_arr[k].border = t.border
            self.tex_arr[k].image = t.image
            self.tex_arr[k].value[:] = tuple(float(x) for x in t.value)
        self.bsdf_arr = (abi.SolGpuBsdf * max(1, len(s.bsdfs)))()
        for k, b in enumerate(s.bsdfs):
            self.bsdf_arr[k].type = b.type
            self.bsdf_arr[k].tex[:] = b.tex
            self.bsdf_arr[k].a = b.a
            self.bsdf_arr[k].b = b.b
        self.light_arr = (abi.SolGpuLight * max(1, len(s.lights)))()
        for k, li in enumerate(s.lights):
            L = self.light_arr[k]
            L.type = li.type
            L.intensity_tex = li.intensity_tex
            L.intensity[:] = tuple(float(x) for x in li.intensity)
            L.v0[:] = tuple(float(x) for x in li.v0)
            L.v1[:] = tuple(float(x) for x in li.v1)
            L.v2[:] = tuple(float(x) for x in li.v2)
        self.img_arr = (abi.SolGpuImage * max(1, len(self.imgs)))()
        for k, im in enumerate(self.imgs):
            self.img_arr[k].height = im.shape[1]
            self.img_arr[k].width = im.shape[2]
            for c in range(3):
                self.img_arr[k].channels[c] = _ptr(im[c], C.c_float)
        d.num_textures = len(s.textures)
        d.textures = self.tex_arr
        d.num_bsdfs = len(s.bsdfs)
        d.bsdfs = self.bsdf_arr
        d.num_lights = len(s.lights)
        d.lights = self.light_arr
        d.num_images = len(self.imgs)
        d.images = self.img_arr
        if bvh is not None:
            self.bvh_nodes, count, prims = bvh
            self.bvh_prims = np.ascontiguousarray(prims, dtype=np.uint32)
            d.num_bvh_nodes = count
            d.bvh_nodes = self.bvh_nodes
            d.bvh_prim_indices = _ptr(self.bvh_prims, C.c_uint32)
        self.c = d

    @property
    def ptr(self):
        return C.byref(self.c)


def build_bvh(s: Scene):
    """Host BVH through the C ABI (sol_gpu_build_bvh): returns (ctypes node array, prim indices)."""
    v = np.ascontiguousarray(s.vertices, dtype=np.float32)
    i = np.ascontiguousarray(s.indices, dtype=np.uint32)
    nt = i.shape[0]
    count = C.c_uint32(max(1, 2 * nt))
    nodes = (abi.SolGpuBvhNode * max(1, 2 * nt))()
    prims = np.zeros(max(1, nt), dtype=np.uint32)
    from . import capi   # loads the CUDA library's C ABI
    capi.check(capi.lib.sol_gpu_build_bvh(_ptr(v, C.c_float), v.shape[0], _ptr(i, C.c_uint32), nt, nodes,
                                          C.byref(count), _ptr(prims, C.c_uint32)), "sol_gpu_build_bvh")
    return nodes, count.value, prims[:nt]
