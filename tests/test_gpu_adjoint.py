"""Path-replay adjoint against central finite differences with common random
numbers, on the textured Cornell box of the adjoint configuration (two RGB
albedo images on the back wall and floor, constant albedos, Phong specular
colour and light emission).

The forward render and the adjoint are wrapped in a torch.autograd.Function;
the loss is L2 between the 16-spp render and a target rendered from other
textures.  Finite differences use eps = 1e-3 and the same sample indices, on
the GPU forward and, for a subset, on SoL's own CPU renderer.  Tolerance, per
parameter: |adjoint - FD| <= 2 % of max(|FD|, floor), the floor being 1 % of
the largest |FD| in the checked set (bench_workloads.grad_check); the step is
eps scaled by the parameter's value above 1 (bench_workloads.fd_step).
Russian roulette makes the estimate discontinuous in the parameters: a
survival decision that flips inside [x - eps, x + eps] adds its jump, and the
jump's square, to the difference of the quadratic loss, which no derivative
has.  With roulette off every checked parameter must pass; with it on, at most
one parameter in 32 may miss (each reported with its difference at eps / 2)."""
import bench_workloads as bw
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

W = H = 64
SPP = 8
EPS = 1e-3


def _setup(tex_size=64, seed=0):
    import torch
    from sol_b200 import scenes
    from sol_b200.renderer import GpuPathTracer, GpuScene
    truth = scenes.cornell_box(0, textured=True, tex_size=tex_size, tex_seed=3)
    start = scenes.cornell_box(0, textured=True, tex_size=tex_size, tex_seed=11)
    cfg = scenes.CORNELL_CONFIG
    gt = GpuScene(truth)
    target = torch.zeros((3, H, W), device="cuda")
    GpuPathTracer(gt, cfg).render_device(target.data_ptr(), W, H, 10_000, 64, torch.cuda.current_stream().cuda_stream)
    target /= 64
    gs = GpuScene(start)
    return start, gs, GpuPathTracer(gs, cfg), target


class Render:
    """torch.autograd.Function over sol_gpu_render_device / sol_gpu_adjoint."""

    @staticmethod
    def make(pt, scene, spp, index):
        import torch

        class Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, params):
                scene.set_params(params.detach().cpu().numpy())
                film = torch.zeros((3, H, W), device="cuda")
                pt.render_device(film.data_ptr(), W, H, index, spp, torch.cuda.current_stream().cuda_stream)
                ctx.n = params.numel()
                return film / spp

            @staticmethod
            def backward(ctx, grad_image):
                dl_dfilm = (grad_image / spp).contiguous()
                grad = torch.zeros(ctx.n, device="cuda")
                pt.adjoint(dl_dfilm.data_ptr(), grad.data_ptr(), W, H, index, spp, torch.cuda.current_stream().cuda_stream)
                return grad

        return Fn.apply


def _fd(loss_of, params0, idx, eps=EPS):
    """Central differences of loss_of(values) at `params0` for the indices
    `idx`, the step scaled by the value above 1 (bench_workloads.fd_step)."""
    out = []
    for i in idx:
        h = bw.fd_step(params0[i], eps)
        hi = params0.copy(); hi[i] += h
        lo = params0.copy(); lo[i] -= h
        out.append((loss_of(hi) - loss_of(lo)) / (2 * h))
    return np.array(out)


def _check_with_roulette(g, fd, loss_of, params0, idx, max_misses):
    """Per-parameter check with roulette on: misses allowed up to `max_misses`,
    reported with their central differences at eps / 2."""
    check = bw.grad_check(g, fd)
    print("per-parameter check:", check)
    if check["within_tol"] < check["params"]:
        misses = bw.roulette_misses(g, fd, _fd(loss_of, params0, idx, EPS / 2), check)
        print("misses:", misses)
        assert len(misses) <= max_misses


def _loss_np(img, target):
    d = img.astype(np.float64) - target.astype(np.float64)
    return float(np.sum(d * d))


def _choose(gs, n_texels, seed):
    count, tex_off, img_off = gs.param_layout()
    rng = np.random.default_rng(seed)
    consts = [tex_off[1] + 0, tex_off[2] + 1, tex_off[0] + 2, tex_off[4] + 0, tex_off[4] + 1, tex_off[7] + 2,
              tex_off[3] + 1]                     # red, green, white albedo; emission r, g; phong ks b; light surface
    texels = list(rng.choice(np.arange(img_off[0], count), size=n_texels, replace=False))
    return consts + [int(t) for t in texels]


def test_adjoint_matches_gpu_finite_differences(built):
    import torch
    scene, gs, pt, target = _setup()
    params0 = torch.from_numpy(gs.get_params()).cuda()
    fn = Render.make(pt, gs, SPP, 0)
    p = params0.clone().requires_grad_(True)
    loss = ((fn(p) - target) ** 2).sum()
    loss.backward()
    g_adj = p.grad.cpu().numpy()
    idx = _choose(gs, 57, seed=1)
    tgt = target.cpu().numpy()
    p0 = params0.cpu().numpy()

    def loss_of(values):
        return _loss_np(fn(torch.from_numpy(values).cuda()).cpu().numpy(), tgt)
    _check_with_roulette(g_adj[idx], _fd(loss_of, p0, idx), loss_of, p0, idx, max_misses=2)
    gs.set_params(p0)


def test_adjoint_matches_gpu_finite_differences_without_roulette(built):
    """The same check with Russian roulette off (min_rr_path_len =
    max_path_len): the estimator is smooth in the parameters and every
    parameter must match."""
    import torch
    from sol_b200 import scenes
    from sol_b200.renderer import GpuPathTracer
    from sol_b200.scene import Config
    scene, gs, _, target = _setup()
    c = scenes.CORNELL_CONFIG
    cfg = Config(max_path_len=c.max_path_len, min_rr_path_len=c.max_path_len, min_survival_prob=c.min_survival_prob,
                 max_survival_prob=c.max_survival_prob, ray_offset=c.ray_offset)
    pt = GpuPathTracer(gs, cfg)
    params0 = torch.from_numpy(gs.get_params()).cuda()
    fn = Render.make(pt, gs, SPP, 0)
    p = params0.clone().requires_grad_(True)
    ((fn(p) - target) ** 2).sum().backward()
    g_adj = p.grad.cpu().numpy()
    idx = _choose(gs, 57, seed=1)
    tgt = target.cpu().numpy()
    p0 = params0.cpu().numpy()

    def loss_of(values):
        return _loss_np(fn(torch.from_numpy(values).cuda()).cpu().numpy(), tgt)
    check = bw.grad_check(g_adj[idx], _fd(loss_of, p0, idx))
    print("adjoint vs GPU FD without roulette:", check)
    assert check["within_tol"] == check["params"]
    gs.set_params(p0)


@pytest.mark.skipif(not oracle.ref_available(), reason="SoL's sources are not built here")
def test_adjoint_matches_sol_cpu_finite_differences(built):
    """Finite differences of SoL's own PathTracer (CPU) on the constants and a few texels."""
    import torch
    from sol_b200 import scenes
    scene, gs, pt, target = _setup(tex_size=32)
    params0 = gs.get_params()
    fn = Render.make(pt, gs, SPP, 0)
    p = torch.from_numpy(params0).cuda().requires_grad_(True)
    ((fn(p) - target) ** 2).sum().backward()
    g_adj = p.grad.cpu().numpy()
    count, tex_off, img_off = gs.param_layout()
    tgt = target.cpu().numpy()

    def cpu_loss(values):
        s = scenes.cornell_box(0, textured=True, tex_size=32, tex_seed=11)
        for t, off in zip(s.textures, tex_off):
            if t.type == 1:
                t.value = tuple(float(x) for x in values[off:off + 3])
            elif t.type == 0:
                t.value = (float(values[off]), 0.0, 0.0)
        s.images = [values[o:o + 3 * 32 * 32].reshape(3, 32, 32).copy() for o in img_off]
        film, _ = oracle.RefScene(s).render(scenes.CORNELL_CONFIG, W, H, SPP, sample_index=0)
        return _loss_np(film / SPP, tgt)

    idx = _choose(gs, 5, seed=2)[:10]
    _check_with_roulette(g_adj[idx], _fd(cpu_loss, params0, idx), cpu_loss, params0, idx, max_misses=1)


def test_loss_kernel_matches_numpy(built):
    import torch
    from sol_b200.renderer import image_l2
    rng = np.random.default_rng(0)
    a = torch.from_numpy(rng.random((3, 50, 70), dtype=np.float32)).cuda()
    b = torch.from_numpy(rng.random((3, 50, 70), dtype=np.float32)).cuda()
    g = torch.zeros_like(a)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    image_l2(a.data_ptr(), b.data_ptr(), a.numel(), 0.5, g.data_ptr(), loss.data_ptr())
    torch.cuda.synchronize()
    d = 0.5 * a.cpu().numpy().astype(np.float64) - b.cpu().numpy()
    assert abs(loss.item() - np.sum(d * d)) <= 1e-9 * np.sum(d * d)
    assert np.allclose(g.cpu().numpy(), 2 * 0.5 * d, rtol=1e-5, atol=1e-6)


def test_params_roundtrip(built):
    from sol_b200 import scenes
    from sol_b200.renderer import GpuScene
    s = scenes.cornell_box(0, textured=True, tex_size=16)
    gs = GpuScene(s)
    v = gs.get_params()
    count, tex_off, img_off = gs.param_layout()
    assert v.size == count == 7 * 3 + 2 + 2 * 3 * 16 * 16   # 7 colours, 2 scalars, 2 images
    assert np.array_equal(v[img_off[0]:img_off[0] + 3 * 256].reshape(3, 16, 16), s.images[0])
    v2 = v.copy()
    v2[tex_off[0]:tex_off[0] + 3] = 0.5
    gs.set_params(v2)
    assert np.array_equal(gs.get_params(), v2)


def test_fused_batch_forward_adjoint_matches_separate_kernels(built):
    """One launch over views of two scenes: films equal the megakernel's bit for bit,
    losses and gradients equal the separate adjoint's (up to atomic summation order)."""
    import torch
    from sol_b200 import scenes
    from sol_b200.renderer import BatchRenderer, GpuPathTracer, GpuScene
    sa = scenes.cornell_box(0, textured=True, tex_size=32)
    sb = scenes.cornell_box(1, textured=True, tex_size=16, tex_seed=7)
    ga, gb = GpuScene(sa), GpuScene(sb)
    cfg = scenes.CORNELL_CONFIG
    stream = torch.cuda.current_stream().cuda_stream
    views = [(0, sa.camera, 40, 24, 3, 4), (1, sb.camera, 24, 32, 100, 2), (0, sa.camera, 16, 16, 9, 3)]
    targets = [torch.rand((3, h, w), device="cuda") * 0.5 for (_, _, w, h, _, _) in views]
    films = [torch.zeros((3, h, w), device="cuda") for (_, _, w, h, _, _) in views]
    grads = [torch.zeros(g.param_layout()[0], device="cuda") for g in (ga, gb)]
    losses = torch.zeros(len(views), dtype=torch.float64, device="cuda")
    br = BatchRenderer([ga, gb])
    br.forward_adjoint(cfg, [(si, cam, w, h, idx, spp, f.data_ptr(), t.data_ptr(), grads[si].data_ptr(),
                              losses[k:k + 1].data_ptr())
                             for k, ((si, cam, w, h, idx, spp), f, t) in enumerate(zip(views, films, targets))], stream)
    torch.cuda.synchronize()
    ref_grads = [torch.zeros_like(g) for g in grads]
    for k, ((si, cam, w, h, idx, spp), f, t) in enumerate(zip(views, films, targets)):
        pt = GpuPathTracer((ga, gb)[si], cfg, camera=cam)
        film = torch.zeros((3, h, w), device="cuda")
        pt.render_device(film.data_ptr(), w, h, idx, spp, stream)
        torch.cuda.synchronize()
        assert torch.equal(film, f)
        d = film / spp - t
        assert abs(losses[k].item() - float((d.double() ** 2).sum())) <= 1e-6 * max(1.0, losses[k].item())
        dl = (2 * d / spp).contiguous()
        pt.adjoint(dl.data_ptr(), ref_grads[si].data_ptr(), w, h, idx, spp, stream)
    torch.cuda.synchronize()
    for g, r in zip(grads, ref_grads):
        assert torch.allclose(g, r, rtol=1e-4, atol=1e-6)
        assert float(r.abs().sum()) > 0


def test_phong_exponent_gradient_direct_lighting(built):
    """The Phong exponent's gradient with max path length 1 (camera hit and light
    sample): the sampled light direction does not depend on the exponent, so the
    derivative with sampling detached is the per-sample derivative and matches
    central differences with common random numbers (GPU forward and, where
    built, SoL's CPU renderer) within 2%.  With longer paths the bounce
    direction moves with the exponent and the two agree only in expectation."""
    import torch
    from sol_b200 import capi, scenes
    from sol_b200.renderer import GpuPathTracer
    from sol_b200.scene import Config
    scene, gs, _, target = _setup(tex_size=32)
    cfg = Config(max_path_len=1, min_rr_path_len=3, min_survival_prob=0.05, max_survival_prob=0.75, ray_offset=1e-5)
    pt = GpuPathTracer(gs, cfg)
    count, tex_off, _ = gs.param_layout()
    phong = [b for b in scene.bsdfs if b.type == capi.BSDF_PHONG][0]
    j = tex_off[phong.tex[1]]
    params0 = gs.get_params()
    assert params0[j] == 64.0
    # A broad lobe: at exponent 64 the box's highlight toward the light is
    # below float range from this camera and the image does not depend on it.
    params0[j] = 4.0
    gs.set_params(params0)
    fn = Render.make(pt, gs, SPP, 0)
    p = torch.from_numpy(params0).cuda().requires_grad_(True)
    ((fn(p) - target) ** 2).sum().backward()
    g = float(p.grad[j])
    tgt = target.cpu().numpy()
    vals = []
    for sgn in (1.0, -1.0):
        q = torch.from_numpy(params0).cuda()
        q[j] += sgn * EPS
        vals.append(_loss_np(fn(q).cpu().numpy(), tgt))
    fd = (vals[0] - vals[1]) / (2 * EPS)
    gs.set_params(params0)
    print("exponent gradient", g, "GPU FD", fd)
    assert fd != 0.0 and abs(g - fd) <= 0.02 * abs(fd)
    if oracle.ref_available():
        cpu = []
        for sgn in (1.0, -1.0):
            s = scenes.cornell_box(0, textured=True, tex_size=32, tex_seed=11)
            t = s.textures[phong.tex[1]]
            t.value = (float(params0[j] + sgn * EPS), 0.0, 0.0)
            film, _ = oracle.RefScene(s).render(cfg, W, H, SPP, sample_index=0)
            cpu.append(_loss_np(film / SPP, tgt))
        fd_cpu = (cpu[0] - cpu[1]) / (2 * EPS)
        print("SoL CPU FD", fd_cpu)
        assert abs(g - fd_cpu) <= 0.02 * abs(fd_cpu)


def test_adjoint_full_configuration_per_parameter(built):
    """The adjoint configuration at full size: 128x128 at 16 spp, two 256x256
    albedo images (393,223 parameters), target at 1024 spp; 64 seeded
    parameters against central differences of the GPU forward, per parameter."""
    import torch
    from sol_b200 import scenes
    from sol_b200.renderer import GpuPathTracer, GpuScene, image_l2
    Wf = Hf = 128
    S = 16
    cfg = scenes.CORNELL_CONFIG
    truth = GpuScene(scenes.cornell_box(0, textured=True, tex_size=256, tex_seed=3))
    target = torch.zeros((3, Hf, Wf), device="cuda")
    GpuPathTracer(truth, cfg).render_device(target.data_ptr(), Wf, Hf, 1 << 24, 1024)
    target /= 1024
    gs = GpuScene(scenes.cornell_box(0, textured=True, tex_size=256, tex_seed=11))
    count, tex_off, img_off = gs.param_layout()
    # The configuration's 393,223 parameters (two 256x256 RGB images, Phong
    # exponent, Phong ks RGB, emission RGB) are all in the vector, which also
    # holds the other constant textures (wall albedos, glass).
    assert count - img_off[0] == 2 * 3 * 256 * 256 and count >= 393223
    pt = GpuPathTracer(gs, cfg)
    film = torch.zeros((3, Hf, Wf), device="cuda")
    pt.render_device(film.data_ptr(), Wf, Hf, 7 * S, S)
    dl = torch.zeros_like(film)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    image_l2(film.data_ptr(), target.data_ptr(), film.numel(), 1.0 / S, dl.data_ptr(), loss.data_ptr())
    grad = torch.zeros(gs.param_layout()[0], device="cuda")
    pt.adjoint(dl.data_ptr(), grad.data_ptr(), Wf, Hf, 7 * S, S)
    torch.cuda.synchronize()
    tgt = target.double()

    def render_loss():
        f = torch.zeros((3, Hf, Wf), device="cuda")
        pt.render_device(f.data_ptr(), Wf, Hf, 7 * S, S)
        torch.cuda.synchronize()
        return float(((f.double() / S - tgt) ** 2).sum())
    assert abs(render_loss() - float(loss.item())) <= 1e-5 * float(loss.item())
    idx = bw.choose_params(gs, 64, seed=5)
    fd = bw.fd_gradient(gs, render_loss, idx)
    check = bw.grad_check(grad.cpu().numpy()[idx], fd)
    print("full adjoint configuration:", check)
    if check["within_tol"] < check["params"]:
        # Any miss must be a roulette jump: its central difference changes when eps halves.
        fd_half = bw.fd_gradient(gs, render_loss, idx, eps=bw.EPS / 2)
        misses = bw.roulette_misses(grad.cpu().numpy()[idx], fd, fd_half, check)
        print("misses:", misses)
        assert len(misses) <= 2


def test_fd_outlier_is_a_russian_roulette_discontinuity(built):
    """Scene 29 of the 32-scene set with the bench's 16 checked parameters,
    where one parameter's central difference (34.2) missed the adjoint (31.6)
    with roulette on.  With roulette off (min_rr_path_len = max_path_len) the
    estimate is smooth in the parameters and every parameter must match; with
    it on, at most that one may miss."""
    import torch
    from sol_b200 import scenes
    from sol_b200.renderer import BatchRenderer, GpuPathTracer, GpuScene
    from sol_b200.scene import Config
    (scene, side), = scenes.scene_set(only=[29])
    S = 16
    gs = GpuScene(scene)
    base_cfg = scenes.SPHERES_CONFIG
    target = torch.zeros((3, side, side), device="cuda")
    GpuPathTracer(gs, base_cfg).render_device(target.data_ptr(), side, side, 1 << 22, 64)
    target *= 0.9 / 64
    tgt = target.double()
    idx = bw.choose_params(gs, 16, seed=100 + 29)
    no_rr = Config(max_path_len=base_cfg.max_path_len, min_rr_path_len=base_cfg.max_path_len,
                   min_survival_prob=base_cfg.min_survival_prob, max_survival_prob=base_cfg.max_survival_prob,
                   ray_offset=base_cfg.ray_offset)
    results = {}
    for name, cfg in (("rr", base_cfg), ("no_rr", no_rr)):
        pt = GpuPathTracer(gs, cfg)
        film = torch.zeros_like(target)
        grad = torch.zeros(gs.param_layout()[0], device="cuda")
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        BatchRenderer([gs]).forward_adjoint(cfg, [(0, scene.camera, side, side, 3 * S, S, film.data_ptr(),
                                                   target.data_ptr(), grad.data_ptr(), loss.data_ptr())])
        torch.cuda.synchronize()

        def render_loss(pt=pt):
            f = torch.zeros_like(target)
            pt.render_device(f.data_ptr(), side, side, 3 * S, S)
            torch.cuda.synchronize()
            return float(((f.double() / S - tgt) ** 2).sum())
        g = grad.cpu().numpy()[idx]
        fd = bw.fd_gradient(gs, render_loss, idx)
        fd_half = bw.fd_gradient(gs, render_loss, idx, eps=bw.EPS / 2)
        results[name] = (g, fd, fd_half, bw.grad_check(g, fd))
        print(name, results[name][3])
    g, fd, fd_half, check = results["no_rr"]
    assert check["within_tol"] == check["params"]
    g, fd, fd_half, check = results["rr"]
    misses = bw.roulette_misses(g, fd, fd_half, check)
    print("roulette on, misses:", misses)
    assert len(misses) <= 1
