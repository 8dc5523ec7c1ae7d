"""SoL scene files into a Scene: the TOML scene description and OBJ/MTL geometry.

The data-format side of the renderer: `load_scene("scene.toml")` returns the
Scene that SoL's `Scene::load` (src/scene_loader.cpp) builds from the same
file, ready for GpuScene / GpuPathTracer / BatchRenderer.

Followed step by step:
  * scene file (src/scene_loader.cpp:44-108): `[camera]` of type "perspective"
    with eye, dir, up, fov and aspect falling back to the defaults
    (include/sol/scene.h:23-29; the aspect ratio is the caller's, as
    test/driver.cpp:197-199 passes the image's); `[[objects]]` of type "import"
    with an `.obj` file relative to the scene file; `root` names the object
    that becomes the scene.
  * OBJ (src/formats/obj.cpp:165-253): v / vn / vt / f / g / o / usemtl /
    mtllib; face indices v, v/t, v//n, v/t/n, negative ones relative to the
    elements read so far; faces with fewer than 3 indices or an index out of
    range are dropped; index 0 of each element list is a dummy (zero) entry.
  * MTL (obj.cpp:263-338): Ka Kd Ks Ke Tf (negative components clamped to 0),
    Ns Ni Tr d illum, map_*; a material missing from the libraries is the
    default (black) material.
  * material to BSDF (obj.cpp:370-418): illum 5 mirror(Ks); illum 7
    glass(Ks, Tf, 1/Ni); otherwise Phong(Ks, Ns) when Ks is not black,
    diffuse(Kd) when Kd is not black, and when both an interpolation with
    weight lum(Ks) / (lum(Kd) + lum(Ks)); neither: no BSDF (paths end there).
  * mesh (obj.cpp:431-516): one vertex per distinct (v, t, n) triple in order
    of first use, polygons fanned from their first vertex, emissive faces
    (Ke not black) become one triangle light each with Ke as intensity, and
    vertices without a normal get the normalized sum of the unit normals of
    the triangles using them.
  * textures, BSDFs and lights are shared when equal (SoL's hash-consing,
    src/scene_loader.h:60-112), in order of first use.

Numbers are read with the C library's strtof, as SoL reads them, so every
value is the same float.  Image maps (map_Kd, ...) would need image file
formats, which are outside this package: like SoL when an image cannot be
loaded, the constant value is used instead.
"""
from __future__ import annotations

import ctypes as C
import os
import tomllib

import numpy as np

from . import abi
from .scene import Bsdf, Camera, Light, Scene, Texture

_libc = C.CDLL(None)
_libc.strtof.restype = C.c_float
_libc.strtof.argtypes = [C.c_char_p, C.POINTER(C.c_char_p)]

_DEFAULT_EYE = (0.0, 0.0, 0.0)
_DEFAULT_DIR = (0.0, 0.0, 1.0)
_DEFAULT_UP = (0.0, 1.0, 0.0)
_DEFAULT_FOV = 60.0


class SceneFormatError(ValueError):
    """A scene file that cannot be loaded; the message names the file and line."""


def _strtof(token: str) -> float:
    return float(_libc.strtof(token.encode(), None))


def _floats(tokens, n: int) -> list:
    """Up to n numbers as consecutive strtof calls read them; missing ones are 0."""
    out = [_strtof(t) for t in tokens[:n]]
    return out + [0.0] * (n - len(out))


def _f32(x) -> np.float32:
    return np.float32(x)


class _Material:
    def __init__(self):
        self.kd = self.ks = self.ke = self.tf = self.ka = (0.0, 0.0, 0.0)
        self.ns = self.ni = self.tr = self.d = 0.0
        self.illum = 0
        self.map_kd = self.map_ks = self.map_ke = self.map_ns = ""


def _luminance(c) -> np.float32:
    # RgbColor::luminance (include/sol/color.h:58), in float
    r, g, b = (_f32(x) for x in c)
    return _f32(_f32(_f32(r * _f32(0.2126)) + _f32(g * _f32(0.7152))) + _f32(b * _f32(0.0722)))


def _is_black(c) -> bool:
    return all(x == 0.0 for x in c)


def _parse_index(tok: str):
    """obj.cpp:113-141: v[/t][/n] with optional parts; None when not an index."""
    if not tok or not (tok[0].isdigit() or tok[0] == '-'):
        return None
    parts = tok.split('/')
    try:
        v = int(parts[0])
        t = int(parts[1]) if len(parts) > 1 and parts[1] != '' else 0
        n = int(parts[2]) if len(parts) > 2 and parts[2] != '' else 0
    except ValueError:
        return None
    return v, t, n


def _parse_mtl(path: str, lib: dict) -> None:
    try:
        f = open(path, encoding="utf-8", errors="replace")
    except OSError:
        return   # SoL accepts missing material libraries when not strict
    mat = lib.setdefault("#dummy", _Material())
    with f:
        for line in f:
            tokens = line.split()
            if not tokens or tokens[0].startswith('#'):
                continue
            cmd, args = tokens[0], tokens[1:]
            if cmd == "newmtl" and args:
                mat = lib.setdefault(args[0], _Material())
            elif cmd in ("Ka", "Kd", "Ks", "Ke", "Tf"):
                col = tuple(max(x, 0.0) for x in _floats(args, 3))
                setattr(mat, cmd.lower(), col)
            elif cmd in ("Ns", "Ni", "Tr"):
                setattr(mat, cmd.lower(), _floats(args, 1)[0])
            elif cmd == "d":
                mat.d = _floats(args, 1)[0]
            elif cmd == "illum":
                mat.illum = int(_floats(args, 1)[0])
            elif cmd in ("map_Kd", "map_Ks", "map_Ke", "map_Ns"):
                setattr(mat, "map_" + cmd[4:].lower(), " ".join(args))


class _Builder:
    """Shared tables of the scene being built (SoL's hash-consing)."""

    def __init__(self):
        self.textures, self.bsdfs, self.lights = [], [], []
        self._tex, self._bsdf, self._light = {}, {}, {}

    def texture(self, kind: int, value) -> int:
        if kind == abi.TEX_CONSTANT:
            key = (kind, float(_f32(value)))
            val = (key[1], 0.0, 0.0)
        else:
            key = (kind,) + tuple(float(_f32(x)) for x in value)
            val = key[1:]
        if key not in self._tex:
            self._tex[key] = len(self.textures)
            self.textures.append(Texture(kind, val))
        return self._tex[key]

    def bsdf(self, kind: int, tex=(-1, -1, -1), a: int = -1, b: int = -1) -> int:
        key = (kind, tuple(tex), a, b)
        if key not in self._bsdf:
            self._bsdf[key] = len(self.bsdfs)
            self.bsdfs.append(Bsdf(kind, tuple(tex), a, b))
        return self._bsdf[key]

    def light(self, v0, v1, v2, tex: int) -> int:
        key = (tuple(map(float, v0)), tuple(map(float, v1)), tuple(map(float, v2)), tex)
        if key not in self._light:
            self._light[key] = len(self.lights)
            self.lights.append(Light(abi.LIGHT_TRIANGLE, key[0], key[1], key[2], intensity_tex=tex))
        return self._light[key]

    def material_bsdf(self, m: _Material) -> int:
        """convert_material (obj.cpp:370-418); -1 for no BSDF."""
        if m.illum == 5:
            return self.bsdf(abi.BSDF_MIRROR, (self.texture(abi.TEX_CONSTANT_COLOR, m.ks), -1, -1))
        if m.illum == 7:
            ks = self.texture(abi.TEX_CONSTANT_COLOR, m.ks)
            kt = self.texture(abi.TEX_CONSTANT_COLOR, m.tf)
            eta = self.texture(abi.TEX_CONSTANT, _f32(1.0) / _f32(m.ni) if m.ni != 0.0 else np.float32(np.inf))
            return self.bsdf(abi.BSDF_GLASS, (ks, kt, eta))
        diff = spec = -1
        diff_k = spec_k = _f32(0.0)
        if not _is_black(m.ks) or m.map_ks:
            ks = self.texture(abi.TEX_CONSTANT_COLOR, m.ks)
            ns = self.texture(abi.TEX_CONSTANT, m.ns)
            spec = self.bsdf(abi.BSDF_PHONG, (ks, ns, -1))
            spec_k = _f32(1.0) if m.map_ks else _luminance(m.ks)
        if not _is_black(m.kd) or m.map_kd:
            kd = self.texture(abi.TEX_CONSTANT_COLOR, m.kd)
            diff = self.bsdf(abi.BSDF_DIFFUSE, (kd, -1, -1))
            diff_k = _f32(1.0) if m.map_kd else _luminance(m.kd)
        if spec >= 0 and diff >= 0:
            k = self.texture(abi.TEX_CONSTANT, _f32(spec_k / _f32(diff_k + spec_k)))
            return self.bsdf(abi.BSDF_INTERP, (k, -1, -1), diff, spec)
        return diff if diff >= 0 else spec


def _normalize32(v: np.ndarray) -> np.ndarray:
    """normalize of core/math.h in float: v * (1 / sqrt(dot(v, v)))."""
    d = (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]
    inv = np.float32(1.0) / np.sqrt(d)
    return v * inv[:, None]


def _load_obj(path: str, b: _Builder):
    verts = [(0.0, 0.0, 0.0)]
    norms = [(0.0, 0.0, 0.0)]
    uvs = [(0.0, 0.0)]
    mat_names = ["#dummy"]
    mtl_files = []
    faces = []   # (indices, material index)
    material = 0
    try:
        f = open(path, encoding="utf-8", errors="replace")
    except OSError as e:
        raise SceneFormatError(f"Cannot open OBJ file '{path}'") from e
    with f:
        for line in f:
            tokens = line.split()
            if not tokens or tokens[0].startswith('#'):
                continue
            cmd = tokens[0]
            if cmd == "v":
                verts.append(tuple(_floats(tokens[1:], 3)))
            elif cmd == "vn":
                norms.append(tuple(_floats(tokens[1:], 3)))
            elif cmd == "vt":
                uvs.append(tuple(_floats(tokens[1:], 2)))
            elif cmd == "f":
                idx = []
                for tok in tokens[1:]:
                    p = _parse_index(tok)
                    if p is None:
                        break
                    idx.append(p)
                ok = len(idx) >= 3
                out = []
                for v, t, n in idx:
                    v = len(verts) + v if v < 0 else v
                    t = len(uvs) + t if t < 0 else t
                    n = len(norms) + n if n < 0 else n
                    ok &= v > 0 and t >= 0 and n >= 0 and v < len(verts) and t < len(uvs) and n < len(norms)
                    out.append((v, t, n))
                if ok:
                    faces.append((out, material))
            elif cmd == "usemtl" and len(tokens) > 1:
                name = tokens[1]
                if name in mat_names:
                    material = mat_names.index(name)
                else:
                    material = len(mat_names)
                    mat_names.append(name)
            elif cmd == "mtllib" and len(tokens) > 1:
                if tokens[1] not in mtl_files:
                    mtl_files.append(tokens[1])
    lib = {"#dummy": _Material()}
    base = os.path.dirname(os.path.abspath(path))
    for m in mtl_files:
        _parse_mtl(os.path.join(base, m), lib)
    mats = [lib.get(name, lib["#dummy"]) for name in mat_names]
    bsdf_of = {}

    vindex = {}
    V, N, T, fix = [], [], [], []
    tris, tri_bsdf, tri_light = [], [], []
    for idx, mi in faces:
        for key in idx:
            if key not in vindex:
                vindex[key] = len(V)
                v, t, n = key
                if n == 0:
                    fix.append(len(N))
                V.append(verts[v])
                N.append(norms[n])
                T.append(uvs[t])
        if mi not in bsdf_of:
            bsdf_of[mi] = b.material_bsdf(mats[mi])
        bsdf = bsdf_of[mi]
        m = mats[mi]
        emissive = not _is_black(m.ke) or bool(m.map_ke)
        first = vindex[idx[0]]
        cur = vindex[idx[1]]
        for i in range(1, len(idx) - 1):
            nxt = vindex[idx[i + 1]]
            light = -1
            if emissive:
                tex = b.texture(abi.TEX_CONSTANT_COLOR, m.ke)
                light = b.light(V[first], V[cur], V[nxt], tex)
            tris.append((first, cur, nxt))
            tri_bsdf.append(bsdf)
            tri_light.append(light)
            cur = nxt
    vertices = np.asarray(V, np.float32).reshape(-1, 3)
    normals = np.asarray(N, np.float32).reshape(-1, 3)
    tex_coords = np.asarray(T, np.float32).reshape(-1, 2)
    indices = np.asarray(tris, np.uint32).reshape(-1, 3)
    if fix:
        # obj.cpp:488-502: sum of the unit normals of the triangles using the vertex, normalized.
        p0, p1, p2 = vertices[indices[:, 0]], vertices[indices[:, 1]], vertices[indices[:, 2]]
        e1, e2 = p1 - p0, p2 - p0
        c = np.stack([e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1],
                      e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2],
                      e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]], axis=1).astype(np.float32)
        fn = _normalize32(c)
        smooth = np.zeros_like(normals)
        # Triangle by triangle, corner by corner (np.add.at adds in element order).
        np.add.at(smooth, indices.reshape(-1), np.repeat(fn, 3, axis=0))
        fix = np.asarray(fix)
        normals[fix] = _normalize32(smooth[fix])
    return vertices, normals, tex_coords, indices, np.asarray(tri_bsdf, np.int32), np.asarray(tri_light, np.int32)


def _vec3(v, default) -> tuple:
    if not isinstance(v, list):
        return default
    out = []
    for k in range(3):
        x = v[k] if k < len(v) else None
        out.append(float(_f32(x)) if isinstance(x, (int, float)) and not isinstance(x, bool) else default[k])
    return tuple(out)


def load_scene(path: str, aspect_ratio: float = 1.0) -> Scene:
    """The Scene SoL's Scene::load builds from the scene file at `path`; the
    camera's aspect ratio defaults to `aspect_ratio` (width / height)."""
    try:
        with open(path, "rb") as f:
            doc = tomllib.load(f)
    except OSError as e:
        raise SceneFormatError(f"Cannot open scene file '{path}'") from e
    except tomllib.TOMLDecodeError as e:
        raise SceneFormatError(f"{e} (in {path})") from e
    base = os.path.dirname(os.path.abspath(path))
    camera = None
    cam = doc.get("camera")
    if isinstance(cam, dict):
        kind = cam.get("type", "")
        if kind != "perspective":
            raise SceneFormatError(f"Unknown camera type '{kind}' (in {path})")
        fov = cam.get("fov", _DEFAULT_FOV)
        aspect = cam.get("aspect", aspect_ratio)
        camera = Camera(eye=_vec3(cam.get("eye"), _DEFAULT_EYE), dir=_vec3(cam.get("dir"), _DEFAULT_DIR),
                        up=_vec3(cam.get("up"), _DEFAULT_UP),
                        fov=float(_f32(fov)) if isinstance(fov, (int, float)) else _DEFAULT_FOV,
                        aspect=float(_f32(aspect)) if isinstance(aspect, (int, float)) else aspect_ratio)
    objects = {}
    for obj in doc.get("objects", []) if isinstance(doc.get("objects"), list) else []:
        if not isinstance(obj, dict):
            continue
        name, kind = obj.get("name", ""), obj.get("type", "")
        if kind != "import":
            raise SceneFormatError(f"Unknown node type '{kind}' (in {path})")
        file = obj.get("file", "")
        if not file.endswith(".obj"):
            raise SceneFormatError(f"Unknown file format for '{file}' (in {path})")
        if name in objects:
            raise SceneFormatError(f"Duplicate geometry found with name '{name}'")
        objects[name] = os.path.join(base, file)
    root = doc.get("root", "")
    # Every object is imported (its materials and lights join the scene's
    # tables, src/scene_loader.cpp:54-59); the root one becomes the geometry.
    b = _Builder()
    meshes = {name: _load_obj(file, b) for name, file in objects.items()}
    if root not in meshes:
        raise SceneFormatError(f"Root geometry named '{root}' cannot be found")
    v, n, t, i, tb, tl = meshes[root]
    return Scene(vertices=v, normals=n, tex_coords=t, indices=i, tri_bsdf=tb, tri_light=tl,
                 textures=b.textures, bsdfs=b.bsdfs, lights=b.lights, images=[], camera=camera)
