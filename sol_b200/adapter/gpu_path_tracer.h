// sol::GpuPathTracer — drop-in replacement for sol::PathTracer
// (include/sol/algorithms/path_tracer.h:33-54) that renders on a CUDA device
// through the C ABI in sol_gpu.h.
//
// Same constructor shape (scene, config) and the same render() contract
// (include/sol/renderer.h:31-34): samples [sample_index, sample_index +
// sample_count) of every pixel are added into the image, deterministically in
// the sample index, with results equal to PathTracer's.  The scene is flattened
// and uploaded on first use (or by prepare()); the BVH that SoL's TriangleMesh
// built is reused as is.  render() throws std::runtime_error on failure, since
// Renderer::render has no error channel.  It may be called from any thread
// (RenderJob renders on its own std::thread), one call at a time.
#pragma once

#include <mutex>

#include "sol/algorithms/path_tracer.h"
#include "sol/renderer.h"
#include "sol_gpu.h"

namespace sol {

class GpuPathTracer final : public Renderer {
public:
    using Config = PathTracer::Config;

    GpuPathTracer(const Scene& scene, const Config& config = {}, int device = 0);
    ~GpuPathTracer() override;

    void render(Image& image, size_t sample_index, size_t sample_count = 1) const override;

    /// Flattens and uploads the scene now instead of at the first render.
    void prepare() const;

    /// The device-side scene handle (after prepare()).
    SolGpuScene* gpu_scene() const { return gpu_scene_; }

private:
    Config config_;
    int device_;
    mutable std::mutex mutex_;
    mutable SolGpuScene* gpu_scene_ = nullptr;
    mutable SolGpuCamera camera_{};
};

}  // namespace sol
