"""GPU megakernel against the CPU checkers, through the C ABI.

Tolerance: per-pixel agreement within 1e-4 relative (SoL's FP32 path tracer,
same seeds and draw order).  The kernels and the checker share arithmetic, so
almost every pixel is expected to be bit-identical; the exact fraction is
asserted as well."""
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle
from helpers import per_pixel_parity

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def gpu_render(scene, cfg, w, h, spp, index=0, film=None):
    from sol_b200.renderer import GpuPathTracer, Image
    img = Image(w, h)
    if film is not None:
        img.channels[...] = film
    GpuPathTracer(scene, cfg).render(img, index, spp)
    return img.channels


def test_cornell_64_matches_oracle(built):
    from sol_b200 import scenes
    scene, cfg, *_ = scenes.cornell_frame()
    g = gpu_render(scene, cfg, 64, 64, 4)
    o = oracle.render(scene, cfg, 64, 64, 4)
    exact, bad = per_pixel_parity(g, o)
    assert bad == 0
    assert exact >= 0.999


def test_cornell_full_config_matches_oracle(built):
    """The Cornell configuration at its full size: 256^2, 16 spp, depth 16."""
    from sol_b200 import scenes
    scene, cfg, w, h, spp = scenes.cornell_frame()
    g = gpu_render(scene, cfg, w, h, spp)
    o = oracle.render(scene, cfg, w, h, spp)
    exact, bad = per_pixel_parity(g, o)
    assert bad == 0
    assert exact >= 0.999


@pytest.mark.parametrize("path", sorted(GOLDEN.glob("render_*.npz")), ids=lambda p: p.stem)
def test_matches_sol_golden_films(built, path):
    sys.path.insert(0, str(GOLDEN))
    from make_golden import scene_for
    f = np.load(path)
    scene, cfg = scene_for(str(f["kind"]))
    g = gpu_render(scene, cfg, int(f["width"]), int(f["height"]), int(f["spp"]), int(f["sample_index"]))
    exact, bad = per_pixel_parity(g, f["film"])
    assert bad == 0
    assert exact >= 0.99


def test_sphere_field_matches_oracle(built):
    from sol_b200 import scenes
    scene = scenes.sphere_field(12, seed=5, bands=33, segments=64)
    g = gpu_render(scene, scenes.SPHERES_CONFIG, 160, 90, 4)
    o = oracle.render(scene, scenes.SPHERES_CONFIG, 160, 90, 4)
    exact, bad = per_pixel_parity(g, o)
    assert bad == 0
    assert exact >= 0.999


def test_textured_cornell_matches_oracle(built):
    from sol_b200 import scenes
    scene = scenes.cornell_box(0, textured=True, tex_size=256)
    g = gpu_render(scene, scenes.CORNELL_CONFIG, 64, 64, 4)
    o = oracle.render(scene, scenes.CORNELL_CONFIG, 64, 64, 4)
    exact, bad = per_pixel_parity(g, o)
    assert bad == 0 and exact >= 0.999


def test_accumulation_and_resume(built):
    """render(0,3) + render(3,5) adds into the film like SoL; equals render(0,8) up to rounding."""
    from sol_b200 import scenes
    scene, cfg, *_ = scenes.cornell_frame()
    g = gpu_render(scene, cfg, 32, 32, 3, 0)
    g = gpu_render(scene, cfg, 32, 32, 5, 3, film=g)
    o = oracle.render(scene, cfg, 32, 32, 3, 0)
    o = oracle.render(scene, cfg, 32, 32, 5, 3, film=o)
    exact, bad = per_pixel_parity(g, o)
    assert bad == 0 and exact >= 0.999
    whole = gpu_render(scene, cfg, 32, 32, 8, 0)
    assert np.allclose(g, whole, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("w,h", [(1, 1), (13, 7), (33, 5), (8, 4)])
def test_odd_image_sizes(built, w, h):
    from sol_b200 import scenes
    scene, cfg, *_ = scenes.cornell_frame()
    g = gpu_render(scene, cfg, w, h, 2)
    o = oracle.render(scene, cfg, w, h, 2)
    exact, bad = per_pixel_parity(g, o)
    assert bad == 0


def test_config_edge_cases(built):
    from sol_b200 import scenes
    from sol_b200.scene import Config
    scene = scenes.cornell_box(0)
    for cfg in (Config(max_path_len=0), Config(max_path_len=1), Config(max_path_len=4, min_rr_path_len=0),
                Config(max_path_len=64, min_survival_prob=0.5, max_survival_prob=0.5)):
        g = gpu_render(scene, cfg, 24, 24, 2)
        o = oracle.render(scene, cfg, 24, 24, 2)
        exact, bad = per_pixel_parity(g, o)
        assert bad == 0, cfg
    assert np.all(gpu_render(scene, Config(max_path_len=0), 8, 8, 2) == 0)


def test_empty_scene_renders_black(built):
    from sol_b200 import scenes
    from sol_b200.scene import Scene
    s = scenes.cornell_box(0)
    empty = Scene(vertices=np.zeros((0, 3), np.float32), normals=np.zeros((0, 3), np.float32),
                  tex_coords=np.zeros((0, 2), np.float32), indices=np.zeros((0, 3), np.uint32),
                  tri_bsdf=np.zeros(0, np.int32), tri_light=np.zeros(0, np.int32), textures=s.textures,
                  bsdfs=s.bsdfs, lights=s.lights, camera=s.camera)
    assert np.all(gpu_render(empty, scenes.CORNELL_CONFIG, 16, 16, 2) == 0)


def test_interp_mirror_point_and_sphere_lights(built):
    """BSDF and light kinds outside the benchmark scenes: Interp(Diffuse, Phong), Mirror,
    point and sphere lights, nearest/clamp/mirror texture modes."""
    from sol_b200 import capi, scenes
    from sol_b200.scene import Bsdf, Light, Texture
    s = scenes.cornell_box(0, textured=True, tex_size=32)
    s.textures.append(Texture(capi.TEX_CONSTANT, (0.3, 0, 0)))
    k = len(s.textures) - 1
    s.bsdfs.append(Bsdf(capi.BSDF_INTERP, (k, -1, -1), a=0, b=5))
    s.bsdfs.append(Bsdf(capi.BSDF_MIRROR, (5, -1, -1)))
    s.textures.append(Texture(capi.TEX_IMAGE, image=0, filter=capi.FILTER_NEAREST, border=capi.BORDER_CLAMP))
    s.textures.append(Texture(capi.TEX_IMAGE, image=1, filter=capi.FILTER_BILINEAR, border=capi.BORDER_MIRROR))
    s.bsdfs.append(Bsdf(capi.BSDF_DIFFUSE, (len(s.textures) - 2, -1, -1)))
    s.bsdfs.append(Bsdf(capi.BSDF_DIFFUSE, (len(s.textures) - 1, -1, -1)))
    nb = len(s.bsdfs)
    s.tri_bsdf[0:2] = nb - 4      # floor: interp
    s.tri_bsdf[6:8] = nb - 3      # red wall: mirror
    s.tri_bsdf[2:4] = nb - 2      # ceiling: nearest/clamp
    s.tri_bsdf[4:6] = nb - 1      # back: bilinear/mirror
    s.tex_coords = s.tex_coords * 3.0 - 1.0
    s.lights.append(Light(capi.LIGHT_POINT, (0.5, 0.8, 0.5), intensity=(0.5, 0.4, 0.3)))
    s.lights.append(Light(capi.LIGHT_SPHERE, (0.2, 0.8, 0.3), (0.05, 0, 0), intensity_tex=4))
    g = gpu_render(s, scenes.CORNELL_CONFIG, 48, 48, 4)
    o = oracle.render(s, scenes.CORNELL_CONFIG, 48, 48, 4)
    exact, bad = per_pixel_parity(g, o)
    assert bad == 0 and exact >= 0.999


@pytest.mark.skipif(not oracle.ref_available(), reason="SoL's sources are not built here")
def test_interp_and_lights_match_sol_pathtracer(built):
    from sol_b200 import capi, scenes
    from sol_b200.scene import Bsdf, Light, Texture
    s = scenes.cornell_box(0)
    s.textures.append(Texture(capi.TEX_CONSTANT, (0.3, 0, 0)))
    s.bsdfs.append(Bsdf(capi.BSDF_INTERP, (len(s.textures) - 1, -1, -1), a=0, b=5))
    s.bsdfs.append(Bsdf(capi.BSDF_MIRROR, (5, -1, -1)))
    s.tri_bsdf[0:2] = len(s.bsdfs) - 2
    s.tri_bsdf[6:8] = len(s.bsdfs) - 1
    s.lights.append(Light(capi.LIGHT_POINT, (0.5, 0.8, 0.5), intensity=(0.5, 0.4, 0.3)))
    s.lights.append(Light(capi.LIGHT_SPHERE, (0.2, 0.8, 0.3), (0.05, 0, 0), intensity_tex=4))
    g = gpu_render(s, scenes.CORNELL_CONFIG, 32, 32, 4)
    r, _ = oracle.RefScene(s).render(scenes.CORNELL_CONFIG, 32, 32, 4)
    exact, bad = per_pixel_parity(g, r)
    assert bad == 0 and exact >= 0.99


def test_device_film_entry_point(built):
    import torch
    from sol_b200 import scenes
    from sol_b200.renderer import GpuPathTracer
    scene, cfg, *_ = scenes.cornell_frame()
    film = torch.full((3, 32, 32), 0.25, dtype=torch.float32, device="cuda")
    pt = GpuPathTracer(scene, cfg)
    stream = torch.cuda.current_stream()
    pt.render_device(film.data_ptr(), 32, 32, 0, 4, stream.cuda_stream)
    stream.synchronize()
    o = oracle.render(scene, cfg, 32, 32, 4, film=np.full((3, 32, 32), 0.25, np.float32))
    exact, bad = per_pixel_parity(film.cpu().numpy(), o)
    assert bad == 0 and exact >= 0.999
    st = pt.stats()
    assert st.paths == 32 * 32 * 4
    assert st.rays >= st.paths and st.shadow_rays > 0 and st.kernel_ms > 0


@pytest.mark.parametrize("which", ["cornell", "spheres"])
def test_schedules_agree_bit_for_bit(built, which):
    """The per-pixel and the split schedule sum the same path colours in the same
    order, so their films are identical; AUTO picks one of them."""
    import torch
    from sol_b200 import capi, scenes
    from sol_b200.renderer import GpuPathTracer, GpuScene
    if which == "cornell":
        scene, cfg, w, h, spp = scenes.cornell_box(0, textured=True, tex_size=32), scenes.CORNELL_CONFIG, 96, 80, 7
    else:
        scene, cfg, w, h, spp = scenes.sphere_field(6, seed=3, bands=17, segments=32), scenes.SPHERES_CONFIG, 160, 90, 5
    gs = GpuScene(scene)
    pt = GpuPathTracer(gs, cfg)
    stream = torch.cuda.current_stream().cuda_stream
    films = {}
    for sched in (capi.SCHEDULE_PER_PIXEL, capi.SCHEDULE_SPLIT, capi.SCHEDULE_AUTO):
        gs.set_schedule(sched)
        f = torch.full((3, h, w), 0.5, device="cuda")
        pt.render_device(f.data_ptr(), w, h, 11, spp, stream)
        torch.cuda.synchronize()
        assert pt.stats().paths == w * h * spp
        films[sched] = f
    assert torch.equal(films[capi.SCHEDULE_PER_PIXEL], films[capi.SCHEDULE_SPLIT])
    assert torch.equal(films[capi.SCHEDULE_PER_PIXEL], films[capi.SCHEDULE_AUTO])
    o = oracle.render(scene, cfg, w, h, spp, sample_index=11, film=np.full((3, h, w), 0.5, np.float32))
    exact, bad = per_pixel_parity(films[capi.SCHEDULE_SPLIT].cpu().numpy(), o)
    assert bad == 0 and exact >= 0.999


@pytest.mark.parametrize("samples_per_chunk", [1, 2, 3])
def test_split_chunks_agree_bit_for_bit(built, samples_per_chunk):
    """A split render whose scratch limit holds fewer samples than it renders
    runs in chunks, carrying each pixel's running sum between them: the film is
    still the per-pixel schedule's, bit for bit."""
    import torch
    from sol_b200 import capi, scenes
    from sol_b200.renderer import GpuPathTracer, GpuScene
    scene, cfg, w, h, spp = scenes.sphere_field(6, seed=3, bands=17, segments=32), scenes.SPHERES_CONFIG, 100, 60, 7
    gs = GpuScene(scene)
    pt = GpuPathTracer(gs, cfg)
    stream = torch.cuda.current_stream().cuda_stream
    films = []
    for sched, limit in ((capi.SCHEDULE_PER_PIXEL, 0), (capi.SCHEDULE_SPLIT, samples_per_chunk * 12 * w * h)):
        gs.set_schedule(sched)
        gs.set_scratch_limit(limit)
        f = torch.full((3, h, w), 0.25, device="cuda")
        pt.render_device(f.data_ptr(), w, h, 3, spp, stream)
        torch.cuda.synchronize()
        assert pt.stats().paths == w * h * spp
        films.append(f)
    assert torch.equal(films[0], films[1])
    gs.set_scratch_limit(12 * w * h - 1)   # not even one sample fits
    with pytest.raises(capi.SolGpuError):
        pt.render_device(films[1].data_ptr(), w, h, 3, spp, stream)


@pytest.mark.parametrize("w,h,spp", [(160, 90, 5), (640, 360, 16)])
def test_basic_shading_build_matches_full(built, w, h, spp):
    """A scene without image textures and Interp BSDFs renders with the kernels
    built without those branches; the same scene carrying an image texture that
    no BSDF uses takes the full build.  Both films must agree bit for bit (the
    larger frame takes the full-occupancy kernels, the smaller the 12-block ones)."""
    import dataclasses
    import torch
    from sol_b200 import capi, scenes
    from sol_b200.scene import Texture
    from sol_b200.renderer import GpuPathTracer, GpuScene
    basic = scenes.sphere_field(6, seed=3, bands=17, segments=32)
    full = dataclasses.replace(basic, textures=list(basic.textures) + [Texture(capi.TEX_IMAGE, image=0)],
                               images=[scenes.noise_texture(8, 5)])
    stream = torch.cuda.current_stream().cuda_stream
    films = []
    for scene in (basic, full):
        f = torch.zeros((3, h, w), device="cuda")
        GpuPathTracer(GpuScene(scene), scenes.SPHERES_CONFIG).render_device(f.data_ptr(), w, h, 7, spp, stream)
        torch.cuda.synchronize()
        films.append(f)
    assert float(films[0].abs().sum()) > 0
    assert torch.equal(films[0], films[1])
