// Test infrastructure (oracle): SoL scenes rendered by the GPU drop-in,
// sol::GpuPathTracer (sol_b200/adapter), under SoL's own Renderer / RenderJob
// interfaces.  Built as libsol_dropin.so beside libsol_ref.so (whose SoL code
// and scene handles it uses) and linked against the product library; only the
// drop-in tests load it.
#include <cstring>
#include <exception>

#include "sol/algorithms/path_tracer.h"
#include "sol/image.h"
#include "sol/render_job.h"

#include "adapter/gpu_path_tracer.h"
#include "ref_harness.h"
#include "sol_gpu.h"

extern "C" {

/// The same scene rendered by the GPU drop-in, sol::GpuPathTracer, optionally
/// driven by sol::RenderJob (src/render_job.cpp:23-40) with `samples_per_frame`.
/// Films are added into like ref_scene_render.  Returns 0, or -1 with the
/// exception text in ref_last_error().
int ref_adapter_render(RefScene* rs, const SolGpuConfig* cfg, uint64_t sample_index, uint32_t sample_count,
                       uint32_t width, uint32_t height, float* r, float* g, float* b, int device,
                       int use_render_job, uint32_t samples_per_frame) {
    try {
        sol::PathTracer::Config c;
        c.max_path_len = cfg->max_path_len;
        c.min_rr_path_len = cfg->min_rr_path_len;
        c.min_survival_prob = cfg->min_survival_prob;
        c.max_survival_prob = cfg->max_survival_prob;
        c.ray_offset = cfg->ray_offset;
        sol::GpuPathTracer tracer(rs->scene, c, device);
        sol::Image image(width, height, 3);
        float* film[3] = {r, g, b};
        const size_t n = (size_t)width * height;
        for (int ch = 0; ch < 3; ++ch) std::memcpy(image.channel(ch).get(), film[ch], sizeof(float) * n);
        if (use_render_job) {
            sol::RenderJob job(tracer, image);
            job.sample_count = sample_count;
            job.samples_per_frame = samples_per_frame;
            job.start();
            job.wait();
        } else {
            tracer.render(image, sample_index, sample_count);
        }
        for (int ch = 0; ch < 3; ++ch) std::memcpy(film[ch], image.channel(ch).get(), sizeof(float) * n);
        return 0;
    } catch (const std::exception& e) {
        ref_set_error(e.what());
        return -1;
    }
}

}  // extern "C"
