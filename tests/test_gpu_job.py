"""GpuRenderJob (sol_gpu_job_*): sol::RenderJob's contract on the GPU.

The film after the job equals the frames SoL's RenderJob loop would render
(render_job.cpp:27-31: frame start i, count i + samples_per_frame, clipped to
sample_count - i), added one by one; the frame callback sees the image so far
and stops the job by returning False; cancel() and wait(timeout) behave as
RenderJob's."""
import time

import numpy as np
import pytest

import oracle
from helpers import per_pixel_parity

pytestmark = pytest.mark.gpu


def _frames(sample_count, spf):
    out, i = [], 0
    while sample_count == 0 or i < sample_count:
        j = i + spf
        if i + j > sample_count and sample_count != 0:
            j = sample_count - i
        out.append((i, j))
        i += spf
    return out


def test_job_film_matches_frame_by_frame_renders(built):
    from sol_b200 import scenes
    from sol_b200.renderer import GpuPathTracer, GpuRenderJob, Image
    scene, cfg = scenes.cornell_box(0), scenes.CORNELL_CONFIG
    pt = GpuPathTracer(scene, cfg)
    img = Image(40, 30)
    img.channels[...] = 0.25
    seen = []
    job = GpuRenderJob(pt, img)
    job.sample_count, job.samples_per_frame = 10, 3

    def frame_end(j):
        seen.append(float(j.output.channels.sum()))
        return True
    job.start(frame_end)
    assert job.wait()
    frames = _frames(10, 3)
    assert job.frames == len(frames) == len(seen)
    assert all(b > a for a, b in zip(seen, seen[1:]))   # the callback saw the image grow
    ref = Image(40, 30)
    ref.channels[...] = 0.25
    for i, n in frames:
        pt.render(ref, i, n)
    assert np.array_equal(img.channels, ref.channels)
    o = np.full((3, 30, 40), 0.25, np.float32)
    for i, n in frames:
        o = oracle.render(scene, cfg, 40, 30, n, sample_index=i, film=o)
    exact, bad = per_pixel_parity(img.channels, o)
    assert bad == 0
    job.close()


def test_job_stops_when_callback_returns_false(built):
    from sol_b200 import scenes
    from sol_b200.renderer import GpuPathTracer, GpuRenderJob, Image
    pt = GpuPathTracer(scenes.cornell_box(0), scenes.CORNELL_CONFIG)
    img = Image(16, 16)
    job = GpuRenderJob(pt, img)
    job.sample_count, job.samples_per_frame = 0, 2          # unlimited
    job.start(lambda j: j.frames < 2)
    assert job.wait()
    assert job.frames == 2
    ref = Image(16, 16)
    for i, n in ((0, 2), (2, 4)):      # unlimited job: counts are not clipped
        pt.render(ref, i, n)
    assert np.array_equal(img.channels, ref.channels)
    job.close()


def test_job_wait_timeout_and_cancel(built):
    from sol_b200 import scenes
    from sol_b200.renderer import GpuPathTracer, GpuRenderJob, Image
    pt = GpuPathTracer(scenes.cornell_box(0), scenes.CORNELL_CONFIG)
    img = Image(64, 64)
    job = GpuRenderJob(pt, img)
    job.sample_count, job.samples_per_frame = 0, 1
    job.start(lambda j: (time.sleep(0.01), True)[1])
    assert job.wait(50) is False          # still running
    job.cancel()
    assert job.wait()
    assert job.frames >= 1 and float(img.channels.sum()) > 0
    job.close()
