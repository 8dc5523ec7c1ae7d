// Internal: the scene handle behind SolGpuScene and the status helpers shared
// by the C ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../../include/sol_gpu.h"
#include "../core/layout.h"
#include "../kernels/kernels.h"

struct SolGpuScene {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    sol_b200::DNode* nodes = nullptr;
    sol_b200::DTri* tris = nullptr;
    sol_b200::DTriShade* shade = nullptr;
    sol_b200::DBsdf* bsdfs = nullptr;
    sol_b200::DTexture* textures = nullptr;
    sol_b200::DImage* images = nullptr;
    float* texels = nullptr;
    sol_b200::DLight* lights = nullptr;
    sol_b200::DeviceCounters* counters = nullptr;
    unsigned int* fault = nullptr;   // kFault* bits set by the kernels' self-checks
    float* split_scratch = nullptr;  // per-sample colours of split-schedule renders
    sol_b200::L2Window l2;           // upper BVH levels kept in L2 by the render launches
    float4* adj_texels4 = nullptr;   // interleaved texel gradients of sol_gpu_adjoint
    uint64_t adj_texels4_count = 0;
    size_t split_floats = 0;
    float* film_tmp = nullptr;       // device film for host-film renders
    size_t film_tmp_floats = 0;
    float* film_host = nullptr;      // pinned staging for host-film renders
    size_t film_host_floats = 0;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    bool instrumented = false;
    int schedule = SOL_GPU_SCHEDULE_AUTO;
    bool basic_shading = false;      // no image textures and no Interp BSDFs: K1's basic-shading build applies
    uint64_t scratch_limit = 0;      // split-schedule colour scratch per render (0: kSplitScratchMaxBytes)
    uint32_t last_launches = 0;      // kernels of the last render
    uint32_t last_chunk = 0;         // its samples per split chunk (0: per pixel)
    bool rendered = false;
    sol_b200::SceneView view{};
    uint32_t default_max_steps = 0;  // traversal bound that no valid hierarchy reaches
    SolGpuSceneInfo info{};
    // Parameter vector (texture values), see sol_gpu_param_layout.
    std::vector<sol_b200::DTexture> host_textures;
    std::vector<sol_b200::DImage> host_images;
    std::vector<uint64_t> texture_offsets;     // per texture (image textures: their image's block)
    std::vector<uint64_t> image_offsets;       // per image
    uint64_t param_count = 0;
    uint64_t constants_count = 0;              // values before the first image block
    unsigned long long* param_offsets = nullptr;   // device copy of texture_offsets
    size_t texel_count = 0;
};

namespace sol_b200 {

/// Records `msg` as the calling thread's last error and returns `code`.
int fail(int code, const std::string& msg);
/// The calling thread's last error message.
const char* last_error();
/// Maps a CUDA error to a status code (out-of-memory is reported as such).
int cuda_fail(cudaError_t e, const char* what);

/// Makes `device` current for the scope of a call and restores the caller's device.
struct DeviceGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != device) err = cudaSetDevice(device);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

DConfig to_config(const SolGpuConfig& c);

/// Reads (and clears) the fault word of a scene after its work finished;
/// returns SOL_GPU_OK or an error describing the failed self-check.
int check_fault(SolGpuScene* s);
DCamera to_camera(const SolGpuCamera& c);

}  // namespace sol_b200
