"""sol_gpu_batch_forward_adjoint_noalloc against sol_gpu_batch_forward_adjoint.

The allocation-free entry point runs the same fused forward + adjoint kernel
with its tables and counters in a fixed array inside the library.  Two calls in
a row must each give the films (bit for bit), losses and gradients of the
batch entry point on the same views, and the second (after the first has set
the device up) must leave the device's free memory unchanged; oversized calls
must be refused.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _views(sa, sb):
    # (scene index, camera, width, height, sample index, sample count)
    return [(0, sa.camera, 40, 24, 3, 4), (1, sb.camera, 24, 32, 100, 2), (0, sa.camera, 16, 16, 9, 3)]


def _adjoint_views(capi, views, films, targets, grads, losses):
    from sol_b200.scene import Camera
    arr = (capi.SolGpuAdjointView * len(views))()
    for k, (si, cam, w, h, index, count) in enumerate(views):
        a = arr[k]
        a.view.scene = si
        a.view.camera = cam.to_c() if isinstance(cam, Camera) else cam
        a.view.width, a.view.height = w, h
        a.view.sample_index, a.view.sample_count = index, count
        a.view.film = films[k].data_ptr()
        a.target = targets[k].data_ptr()
        a.grad = grads[si].data_ptr()
        a.loss = losses[k:k + 1].data_ptr()
    return arr


def _buffers(torch, views, param_counts):
    films = [torch.zeros((3, h, w), device="cuda") for (_, _, w, h, _, _) in views]
    grads = [torch.zeros(n, device="cuda") for n in param_counts]
    losses = torch.zeros(len(views), dtype=torch.float64, device="cuda")
    return films, grads, losses


def test_noalloc_matches_batch_entry_point_twice(built):
    import torch
    from sol_b200 import capi, scenes
    from sol_b200.renderer import BatchRenderer, GpuScene
    sa = scenes.cornell_box(0, textured=True, tex_size=32)
    sb = scenes.cornell_box(1, textured=True, tex_size=16, tex_seed=7)
    ga, gb = GpuScene(sa), GpuScene(sb)
    cfg = scenes.CORNELL_CONFIG
    stream = torch.cuda.current_stream().cuda_stream
    views = _views(sa, sb)
    gen = torch.Generator(device="cuda").manual_seed(5)
    targets = [torch.rand((3, h, w), device="cuda", generator=gen) * 0.5 for (_, _, w, h, _, _) in views]
    counts = [ga.param_layout()[0], gb.param_layout()[0]]

    # The existing entry point (through a SolGpuBatch).
    films_ref, grads_ref, losses_ref = _buffers(torch, views, counts)
    br = BatchRenderer([ga, gb])
    br.forward_adjoint(cfg, [(si, cam, w, h, idx, spp, f.data_ptr(), t.data_ptr(), grads_ref[si].data_ptr(),
                              losses_ref[k:k + 1].data_ptr())
                             for k, ((si, cam, w, h, idx, spp), f, t) in enumerate(zip(views, films_ref, targets))],
                       stream)
    torch.cuda.synchronize()
    assert float(grads_ref[0].abs().sum()) > 0 and float(grads_ref[1].abs().sum()) > 0

    # Two calls in a row of the allocation-free entry point, each into fresh
    # buffers allocated (and zeroed) before the call.
    handles = (capi.ScenePtr * 2)(ga.handle, gb.handle)
    c_cfg = cfg.to_c()
    outs = [_buffers(torch, views, counts) for _ in range(2)]
    arrays = [_adjoint_views(capi, views, f, targets, g, l) for (f, g, l) in outs]
    torch.cuda.synchronize()
    free = []
    for arr in arrays:
        before = torch.cuda.mem_get_info()[0]
        capi.check(capi.lib.sol_gpu_batch_forward_adjoint_noalloc(handles, 2, C.byref(c_cfg), arr, len(views),
                                                                  stream),
                   "sol_gpu_batch_forward_adjoint_noalloc")
        torch.cuda.synchronize()
        free.append((before, torch.cuda.mem_get_info()[0]))
    # The first call may load the library's module on this device; the second
    # finds everything in place and takes no device memory.
    assert free[1][0] == free[1][1], free
    for films, grads, losses in outs:
        for f, r in zip(films, films_ref):
            assert torch.equal(f, r)
        # Losses and gradients are sums of atomics: equal up to summation order.
        assert torch.allclose(losses, losses_ref, rtol=1e-9, atol=0.0)
        for g, r in zip(grads, grads_ref):
            assert torch.allclose(g, r, rtol=1e-4, atol=1e-6)
    br.stats()  # reads the scenes' self-check words; raises if one fired


def test_noalloc_rejects_oversized_calls(built):
    import torch
    from sol_b200 import capi, scenes
    from sol_b200.renderer import GpuScene
    sa = scenes.cornell_box(0)
    ga = GpuScene(sa)
    c_cfg = scenes.CORNELL_CONFIG.to_c()
    film = torch.zeros((3, 4, 4), device="cuda")
    target = torch.zeros((3, 4, 4), device="cuda")
    grad = torch.zeros(max(1, ga.param_layout()[0]), device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    views = [(0, sa.camera, 4, 4, 0, 1)] * 513
    arr = _adjoint_views(capi, views, [film] * 513, [target] * 513, [grad], loss.expand(513))
    one = (capi.ScenePtr * 1)(ga.handle)
    rc = capi.lib.sol_gpu_batch_forward_adjoint_noalloc(one, 1, C.byref(c_cfg), arr, 513, 0)
    assert rc == capi.ERR_INVALID_ARG
    assert b"512 views" in capi.lib.sol_gpu_last_error()
    many = (capi.ScenePtr * 65)(*([ga.handle] * 65))
    rc = capi.lib.sol_gpu_batch_forward_adjoint_noalloc(many, 65, C.byref(c_cfg), arr, 1, 0)
    assert rc == capi.ERR_INVALID_ARG
    assert b"64 scenes" in capi.lib.sol_gpu_last_error()
    torch.cuda.synchronize()
    assert float(film.abs().sum()) == 0.0 and float(loss.abs().sum()) == 0.0
    assert np.isfinite(float(grad.sum()))
