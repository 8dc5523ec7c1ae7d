// SolGpuJob: progressive rendering on a host thread, the GPU counterpart of
// sol::RenderJob (include/sol/render_job.h, src/render_job.cpp:23-59).
//
// The job keeps the film on the device: it starts as a copy of the caller's
// host film, every frame adds its samples into it (sol_gpu_render_device on
// the job's own stream), and after each frame the film is copied back into the
// caller's planes before the frame callback runs, so the callback sees the
// image SoL's frame_end callback would see.  The next frame starts only after
// the callback returns non-zero, as in SoL.  Frames cover the sample ranges
// SoL's loop gives them (render_job.cpp:27-31): frame start i advances by
// samples_per_frame, and the count passed is i + samples_per_frame, or
// sample_count - i when i + that count exceeds sample_count — so with the same
// renderer the film matches sol::RenderJob's bit for bit.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

#include "../../include/sol_gpu.h"
#include "host/handles.h"

using namespace sol_b200;

struct SolGpuJob {
    SolGpuScene* scene = nullptr;
    SolGpuCamera camera{};
    SolGpuConfig config{};
    uint32_t width = 0, height = 0;
    float* out[3] = {nullptr, nullptr, nullptr};
    uint64_t sample_count = 0;
    uint32_t samples_per_frame = 1;
    SolGpuFrameEnd frame_end = nullptr;
    void* user = nullptr;

    float* d_film = nullptr;
    float* h_film = nullptr;       // pinned staging for the copy back
    cudaStream_t stream = nullptr;
    std::thread thread;
    std::mutex mutex;
    std::condition_variable done_cond;
    bool done = true;
    std::atomic<bool> cancelled{false};
    std::atomic<uint64_t> frames{0};
    int status = SOL_GPU_OK;
    std::string error;
};

namespace {

void finish(SolGpuJob* j, int status, const std::string& error) {
    std::lock_guard<std::mutex> lock(j->mutex);
    j->status = status;
    j->error = error;
    j->done = true;
    j->done_cond.notify_all();
}

void run(SolGpuJob* j) {
    DeviceGuard guard(j->scene->device);
    if (guard.err != cudaSuccess) { finish(j, SOL_GPU_ERR_CUDA, "cudaSetDevice failed"); return; }
    const size_t plane = (size_t)j->width * j->height;
    const uint64_t n = j->sample_count;
    const uint64_t spf = j->samples_per_frame;
    for (uint64_t i = 0; n == 0 || i < n; i += spf) {
        uint64_t count = i + spf;                 // render_job.cpp:28-30
        if (i + count > n && n != 0) count = n - i;
        if (count > 0xffffffffull) { finish(j, SOL_GPU_ERR_INVALID_ARG, "frame sample count too large"); return; }
        int rc = sol_gpu_render_device(j->scene, &j->camera, &j->config, i, (uint32_t)count, j->width, j->height,
                                       j->d_film, j->stream);
        cudaError_t e = cudaSuccess;
        if (rc == SOL_GPU_OK) e = cudaMemcpyAsync(j->h_film, j->d_film, 3 * plane * sizeof(float), cudaMemcpyDeviceToHost,
                                                  j->stream);
        if (rc == SOL_GPU_OK && e == cudaSuccess) e = cudaStreamSynchronize(j->stream);
        if (rc == SOL_GPU_OK && e != cudaSuccess) rc = cuda_fail(e, "frame");
        if (rc == SOL_GPU_OK) {
            SolGpuRenderStats st;
            rc = sol_gpu_render_stats(j->scene, &st);   // reports kernel self-check failures
        }
        if (rc != SOL_GPU_OK) { finish(j, rc, last_error()); return; }
        for (int c = 0; c < 3; ++c) std::memcpy(j->out[c], j->h_film + c * plane, plane * sizeof(float));
        j->frames.fetch_add(1);
        if ((j->frame_end && !j->frame_end(j->user, j->frames.load())) || j->cancelled.load()) break;
    }
    finish(j, SOL_GPU_OK, "");
}

}  // namespace

extern "C" {

int sol_gpu_job_start(SolGpuScene* scene, const SolGpuCamera* camera, const SolGpuConfig* config, uint32_t width,
                      uint32_t height, float* film_r, float* film_g, float* film_b, uint64_t sample_count,
                      uint32_t samples_per_frame, SolGpuFrameEnd frame_end, void* user, SolGpuJob** out) {
    if (!scene || !camera || !config || !film_r || !film_g || !film_b || !out)
        return fail(SOL_GPU_ERR_INVALID_ARG, "scene, camera, config, film and out must not be NULL");
    if (width == 0 || height == 0) return fail(SOL_GPU_ERR_INVALID_ARG, "image size must be positive");
    if (samples_per_frame == 0) return fail(SOL_GPU_ERR_INVALID_ARG, "samples_per_frame must be positive");
    DeviceGuard guard(scene->device);
    if (guard.err != cudaSuccess) return cuda_fail(guard.err, "cudaSetDevice");
    auto* j = new SolGpuJob();
    j->scene = scene;
    j->camera = *camera;
    j->config = *config;
    j->width = width;
    j->height = height;
    j->out[0] = film_r;
    j->out[1] = film_g;
    j->out[2] = film_b;
    j->sample_count = sample_count;
    j->samples_per_frame = samples_per_frame;
    j->frame_end = frame_end;
    j->user = user;
    const size_t plane = (size_t)width * height;
    cudaError_t e = cudaStreamCreateWithFlags(&j->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&j->d_film), 3 * plane * sizeof(float));
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&j->h_film), 3 * plane * sizeof(float), 0);
    if (e == cudaSuccess) {
        // The device film starts as the caller's image (renders add into it).
        for (int c = 0; c < 3; ++c) std::memcpy(j->h_film + c * plane, j->out[c], plane * sizeof(float));
        e = cudaMemcpy(j->d_film, j->h_film, 3 * plane * sizeof(float), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        int rc = cuda_fail(e, "job set-up");
        sol_gpu_job_destroy(j);
        return rc;
    }
    j->done = false;
    j->thread = std::thread(run, j);
    *out = j;
    return SOL_GPU_OK;
}

int sol_gpu_job_wait(SolGpuJob* j, uint32_t timeout_ms, int* finished) {
    if (!j || !finished) return fail(SOL_GPU_ERR_INVALID_ARG, "job and finished must not be NULL");
    std::unique_lock<std::mutex> lock(j->mutex);
    if (timeout_ms != 0) {
        if (!j->done_cond.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] { return j->done; })) {
            *finished = 0;
            return SOL_GPU_OK;
        }
    } else {
        j->done_cond.wait(lock, [&] { return j->done; });
    }
    lock.unlock();
    if (j->thread.joinable()) j->thread.join();
    *finished = 1;
    if (j->status != SOL_GPU_OK) return fail(j->status, j->error);
    return SOL_GPU_OK;
}

int sol_gpu_job_cancel(SolGpuJob* j) {
    if (!j) return fail(SOL_GPU_ERR_INVALID_ARG, "job must not be NULL");
    j->cancelled.store(true);
    return SOL_GPU_OK;
}

int sol_gpu_job_frames(const SolGpuJob* j, uint64_t* frames) {
    if (!j || !frames) return fail(SOL_GPU_ERR_INVALID_ARG, "job and frames must not be NULL");
    *frames = j->frames.load();
    return SOL_GPU_OK;
}

int sol_gpu_job_destroy(SolGpuJob* j) {
    if (!j) return SOL_GPU_OK;
    j->cancelled.store(true);
    if (j->thread.joinable()) j->thread.join();
    DeviceGuard guard(j->scene->device);
    if (j->stream) cudaStreamDestroy(j->stream);
    cudaFree(j->d_film);
    if (j->h_film) cudaFreeHost(j->h_film);
    delete j;
    return SOL_GPU_OK;
}

}  // extern "C"
