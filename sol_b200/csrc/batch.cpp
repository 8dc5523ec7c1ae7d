// Batched wavefront rendering: SolGpuBatch and its C ABI entry points
// (include/sol_gpu.h), host side.  The stages are in kernels/wavefront.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/sol_gpu.h"
#include "host/handles.h"
#include "kernels/adjoint.h"
#include "kernels/kernels.h"
#include "kernels/wavefront.h"

using namespace sol_b200;

struct SolGpuBatch {
    int device = 0;
    int num_sms = 0;
    std::vector<SolGpuScene*> scenes;
    SolGpuBatchOptions opts{};
    uint32_t allocated = 0;           // pool capacity in memory
    void* pool = nullptr;
    WfParams host{};                  // host copy of the device parameters
    WfParams* d_params = nullptr;
    WfCounters* d_ctr = nullptr;
    SceneView* d_scenes = nullptr;
    std::vector<SceneView> h_scenes;   // the same views on the host (kernel-parameter scene tables)
    WfView* d_views = nullptr;
    size_t views_cap = 0;
    AdjView* d_adj_views = nullptr;
    size_t adj_views_cap = 0;
    DeviceCounters* d_dc = nullptr;   // counters of the megakernel-type launches
    float* scratch = nullptr;         // per-sample colours of split views (and the wavefront's running sums)
    uint64_t scratch_floats = 0;
    WfSceneTable wf_table{};          // the scenes as the wavefront stages take them (kernel parameter)
    float4* d_scene_box = nullptr;    // per scene: bounds of the hierarchy's root (reordering keys)
    uint32_t* d_sort_bins = nullptr;  // reordering histogram and offsets
    bool graph_sort = false;          // the captured graph reorders the queues
    bool graph_packed = false;        // the captured graph packs the shadow queue in extend order
    bool basic = false;               // every scene has basic shading
    unsigned long long max_iterations = 0;   // wavefront bounce-loop bound (0: the default)
    uint64_t scratch_limit = 0;       // wavefront scratch bytes per render (0: kWfScratchMaxBytes)
    WfLaunch launch{};
    int launch_block = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t capture = nullptr;
    WfCounters* h_ctr = nullptr;      // pinned, for the host-driven loop
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    bool rendered = false;
    bool last_dc = false;             // the last launch counted into d_dc (megakernel schedules)
    uint32_t last_passes = 0;         // wavefront launches (sample chunks) of the last render
};

namespace {

constexpr uint32_t kDefaultCapacity = 1u << 22;
constexpr uint32_t kMaxCapacity = 1u << 26;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t pool_bytes(uint32_t c) {
    size_t b = 0;
    b += 9 * align256(sizeof(float4) * (size_t)c);                    // thru color ray_o[2] ray_d[2] sh_o sh_d sh_c
    b += align256(sizeof(unsigned long long) * (size_t)c);            // rng
    b += align256(sizeof(uint2) * (size_t)c);                         // item
    b += align256(sizeof(float4) * (size_t)c);                        // hit
    b += (2 + kWfBins) * align256(sizeof(uint32_t) * (size_t)c);      // ended queues, bins
    b += 3 * align256(sizeof(float4) * (size_t)c);                    // reordering: spare arrays
    b += align256(sizeof(uint32_t) * (size_t)c);                      // reordering: keys
    return b;
}

void destroy_graph(SolGpuBatch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

int alloc_pool(SolGpuBatch* b, uint32_t capacity) {
    if (b->pool && b->allocated >= capacity) return SOL_GPU_OK;
    destroy_graph(b);
    cudaFree(b->pool);
    b->pool = nullptr;
    b->allocated = 0;
    cudaError_t e = cudaMalloc(&b->pool, pool_bytes(capacity));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc path pool");
    b->allocated = capacity;
    char* p = static_cast<char*>(b->pool);
    auto take = [&](size_t bytes) { char* r = p; p += align256(bytes); return r; };
    const size_t c = capacity;
    WfParams& h = b->host;
    h.thru = reinterpret_cast<float4*>(take(sizeof(float4) * c));
    h.color = reinterpret_cast<float4*>(take(sizeof(float4) * c));
    h.rng = reinterpret_cast<unsigned long long*>(take(sizeof(unsigned long long) * c));
    h.item = reinterpret_cast<uint2*>(take(sizeof(uint2) * c));
    for (int k = 0; k < 2; ++k) {
        h.ray_o[k] = reinterpret_cast<float4*>(take(sizeof(float4) * c));
        h.ray_d[k] = reinterpret_cast<float4*>(take(sizeof(float4) * c));
        h.q_ended[k] = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * c));
    }
    h.hit = reinterpret_cast<float4*>(take(sizeof(float4) * c));
    h.sh_o = reinterpret_cast<float4*>(take(sizeof(float4) * c));
    h.sh_d = reinterpret_cast<float4*>(take(sizeof(float4) * c));
    h.sh_c = reinterpret_cast<float4*>(take(sizeof(float4) * c));
    for (int k = 0; k < 3; ++k) h.alt[k] = reinterpret_cast<float4*>(take(sizeof(float4) * c));
    h.sort_key = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * c));
    h.q_bins = reinterpret_cast<uint32_t*>(p);
    return SOL_GPU_OK;
}

int configure_launch(SolGpuBatch* b) {
    int block = (int)(b->opts.block_size ? b->opts.block_size : 128);
    if (block != 64 && block != 128 && block != 256) return fail(SOL_GPU_ERR_INVALID_ARG, "block_size must be 64, 128 or 256");
    if (block == b->launch_block) return SOL_GPU_OK;
    for (int s = 0; s < 4; ++s) {
        int per_sm = wavefront_blocks_per_sm(s, block);
        if (per_sm <= 0) return fail(SOL_GPU_ERR_CUDA, "wavefront occupancy query failed");
        b->launch.grid[s] = per_sm * b->num_sms;
        b->launch.block[s] = block;
    }
    b->launch.sms = b->num_sms;
    b->launch_block = block;
    destroy_graph(b);
    return SOL_GPU_OK;
}

/// Graph = WHILE(condition) { generate, extend, shade, shadow, advance }.
int build_graph(SolGpuBatch* b) {
    if (b->exec) return SOL_GPU_OK;
    cudaError_t e = cudaGraphCreate(&b->graph, 0);
    cudaGraphConditionalHandle handle{};
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&handle, b->graph, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node{};
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, b->graph, nullptr, 0, &np);
    if (e != cudaSuccess) { destroy_graph(b); return cuda_fail(e, "graph conditional node"); }
    cudaGraph_t body = np.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(b->capture, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaError_t le = launch_wf_iteration(b->d_params, b->wf_table, b->basic, b->graph_sort, b->graph_packed,
                                             b->launch, handle, 1, b->capture);
        e = cudaStreamEndCapture(b->capture, &body);
        if (e == cudaSuccess) e = le;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) { destroy_graph(b); cudaGetLastError(); return cuda_fail(e, "graph capture"); }
    return SOL_GPU_OK;
}

/// Largest per-sample colour scratch the multi-view megakernel may use for
/// its split views; views beyond it run per pixel.
constexpr uint64_t kViewsScratchMaxBytes = uint64_t(4) << 30;

/// Builds and uploads the view table.  For the megakernel schedule, views of
/// more than one sample are split ((sample, pixel) work items, colours in
/// scratch), as sol_gpu_render_device's AUTO schedule splits them, in view
/// order while their scratch fits in kViewsScratchMaxBytes; `sum_floats`
/// receives the size of their sum pass.
int upload_views(SolGpuBatch* b, const SolGpuView* views, uint32_t n, uint32_t* total_items, uint64_t* pixels,
                 cudaStream_t stream, bool megakernel = false, uint64_t* sum_floats = nullptr) {
    std::vector<WfView> v(n);
    uint64_t items = 0, px = 0;
    std::vector<uint64_t> scratch_at(n, 0);
    uint64_t scratch_floats = 0, sum_at = 0;
    if (megakernel) {
        for (uint32_t i = 0; i < n; ++i) {
            const SolGpuView& s = views[i];
            const uint64_t plane = (uint64_t)s.width * s.height;
            const uint64_t need = 3 * plane * s.sample_count;
            if (s.sample_count > 1 && (scratch_floats + need) * sizeof(float) <= kViewsScratchMaxBytes) {
                scratch_at[i] = scratch_floats + 1;   // + 1: 0 marks "not split"
                scratch_floats += need;
            }
        }
        if (b->scratch_floats < scratch_floats) {
            cudaFree(b->scratch);
            b->scratch = nullptr;
            b->scratch_floats = 0;
            cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->scratch), scratch_floats * sizeof(float));
            if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc view scratch");
            b->scratch_floats = scratch_floats;
        }
    }
    for (uint32_t i = 0; i < n; ++i) {
        const SolGpuView& s = views[i];
        if (s.scene >= b->scenes.size()) return fail(SOL_GPU_ERR_INVALID_ARG, "view scene index out of range");
        if (s.width == 0 || s.height == 0) return fail(SOL_GPU_ERR_INVALID_ARG, "view size must be positive");
        if (!s.film) return fail(SOL_GPU_ERR_INVALID_ARG, "view film must not be NULL");
        WfView& w = v[i];
        std::memcpy(w.eye, s.camera.eye, sizeof(w.eye));
        std::memcpy(w.dir, s.camera.dir, sizeof(w.dir));
        std::memcpy(w.right, s.camera.right, sizeof(w.right));
        std::memcpy(w.up, s.camera.up, sizeof(w.up));
        w.scene = s.scene;
        w.width = s.width;
        w.height = s.height;
        w.sample_count = s.sample_count;
        w.sample_index = s.sample_index;
        w.film = s.film;
        w.tiles_x = (s.width + 7) / 8;
        w.item_begin = (uint32_t)items;
        w.split = scratch_at[i] != 0;
        w.scratch = w.split ? b->scratch + (scratch_at[i] - 1) : nullptr;
        w.sum_begin = sum_at;
        w.running = nullptr;
        w.first_chunk = 1;
        w.last_chunk = 1;
        if (w.split) sum_at += 3 * (uint64_t)s.width * s.height;
        items += (uint64_t)w.tiles_x * ((s.height + 3) / 4) * 32 * (w.split ? s.sample_count : 1u);
        px += (uint64_t)s.width * s.height;
        if (items > 0xffffffffull) return fail(SOL_GPU_ERR_INVALID_ARG, "batch too large (more than 2^32 work items)");
    }
    if (b->views_cap < n) {
        cudaFree(b->d_views);
        b->d_views = nullptr;
        b->views_cap = 0;
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->d_views), sizeof(WfView) * std::max<size_t>(n, 64));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc views");
        b->views_cap = std::max<size_t>(n, 64);
    }
    cudaError_t e = cudaMemcpyAsync(b->d_views, v.data(), sizeof(WfView) * n, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return cuda_fail(e, "views upload");
    *total_items = (uint32_t)items;
    *pixels = px;
    if (sum_floats) *sum_floats = sum_at;
    return SOL_GPU_OK;
}

/// Largest scratch (per-sample colours and running sums) the wavefront may
/// hold for one render; batches needing more run in chunks of samples.
#ifndef SOL_WF_SCRATCH_MAX_MB
#define SOL_WF_SCRATCH_MAX_MB 8192
#endif
constexpr uint64_t kWfScratchMaxBytes = uint64_t(SOL_WF_SCRATCH_MAX_MB) << 20;

/// Re-reads the scenes' device views (their traversal bound may have changed
/// since the batch was made) and refreshes the tables built from them.
int refresh_scenes(SolGpuBatch* b) {
    bool changed = false;
    for (size_t i = 0; i < b->scenes.size(); ++i)
        if (std::memcmp(&b->h_scenes[i], &b->scenes[i]->view, sizeof(SceneView)) != 0) {
            b->h_scenes[i] = b->scenes[i]->view;
            changed = true;
        }
    if (!changed) return SOL_GPU_OK;
    cudaError_t e = cudaMemcpy(b->d_scenes, b->h_scenes.data(), sizeof(SceneView) * b->h_scenes.size(),
                               cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "scene table upload");
    for (size_t i = 0; i < b->h_scenes.size() && i < kWfMaxScenes; ++i) b->wf_table.v[i] = b->h_scenes[i];
    destroy_graph(b);
    return SOL_GPU_OK;
}

int render_megakernel(SolGpuBatch* b, const SolGpuConfig* config, const SolGpuView* views, uint32_t n,
                      cudaStream_t stream) {
    uint32_t total_items = 0;
    uint64_t pixels = 0, sum_floats = 0;
    int rc = upload_views(b, views, n, &total_items, &pixels, stream, true, &sum_floats);
    if (rc != SOL_GPU_OK) return rc;
    {
        if (!b->d_dc) {
            cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->d_dc), sizeof(DeviceCounters));
            if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc counters");
        }
        uint32_t max_spp = 0;
        for (uint32_t i = 0; i < n; ++i) max_spp = std::max(max_spp, views[i].sample_count);
        const int per_sm = megakernel_views_blocks_per_sm();
        if (per_sm <= 0) return fail(SOL_GPU_ERR_CUDA, "megakernel occupancy query failed");
        cudaError_t e = cudaMemsetAsync(b->d_dc, 0, sizeof(DeviceCounters), stream);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
        cudaEventRecord(b->ev_start, stream);
        if (n > 0) {
            const bool basic = std::all_of(b->scenes.begin(), b->scenes.end(),
                                           [](const SolGpuScene* s) { return s->basic_shading; });
            e = launch_megakernel_views(b->d_views, n, total_items, max_spp, b->d_scenes, b->h_scenes.data(),
                                        (uint32_t)b->h_scenes.size(), basic, to_config(*config), b->d_dc,
                                        b->scenes[0]->fault, per_sm * b->num_sms, stream,
                                        b->scenes.size() == 1 ? b->scenes[0]->l2 : L2Window{});
            if (e == cudaSuccess) e = launch_sum_samples_views(b->d_views, n, sum_floats, stream);
            if (e != cudaSuccess) return cuda_fail(e, "megakernel launch");
        }
        cudaEventRecord(b->ev_stop, stream);
        b->rendered = true;
        b->last_dc = true;
        return SOL_GPU_OK;
    }
}

/// Work items of one sample of a view: its 8x4 pixel tiles, 32 items each.
uint64_t items_per_sample(const SolGpuView& v) {
    return (uint64_t)((v.width + 7) / 8) * ((v.height + 3) / 4) * 32;
}

/// One launch of the wavefront over a set of views (one chunk of samples).
struct WfPass {
    size_t first_view = 0;   // into the concatenated view tables
    uint32_t num_views = 0;
    uint32_t total_items = 0;
    uint64_t sum_pixels = 0;   // pixels of the pass's views (threads of its sum pass)
};

/// The wavefront: views are split into (sample, pixel) work items whose path
/// colours go to per-sample scratch planes, summed per pixel in sample order
/// afterwards.  When the scratch of every sample would exceed
/// kWfScratchMaxBytes, the samples run in chunks of K (the largest K that
/// fits): chunk j renders samples [jK, (j+1)K) of every view that has them,
/// carrying each pixel's sum from chunk to chunk.
int render_wavefront(SolGpuBatch* b, const SolGpuConfig* config, const SolGpuView* views, uint32_t n,
                     cudaStream_t stream) {
    if (b->scenes.size() > kWfMaxScenes)
        return fail(SOL_GPU_ERR_UNSUPPORTED, "the wavefront schedule takes at most 64 scenes per batch");
    uint32_t max_spp = 0;
    uint64_t all_floats = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const SolGpuView& s = views[i];
        if (s.scene >= b->scenes.size()) return fail(SOL_GPU_ERR_INVALID_ARG, "view scene index out of range");
        if (s.width == 0 || s.height == 0) return fail(SOL_GPU_ERR_INVALID_ARG, "view size must be positive");
        if (!s.film) return fail(SOL_GPU_ERR_INVALID_ARG, "view film must not be NULL");
        max_spp = std::max(max_spp, s.sample_count);
        all_floats += 4ull * items_per_sample(s) * s.sample_count;
    }
    const uint64_t limit = (b->scratch_limit ? b->scratch_limit : kWfScratchMaxBytes) / sizeof(float);
    // Scratch floats of chunks of k samples: one float4 per work item of the
    // first chunk (item order), plus 3 planes of running sums per view that
    // needs more than one chunk.
    auto need = [&](uint32_t k) {
        uint64_t f = 0;
        for (uint32_t i = 0; i < n; ++i) {
            f += 4ull * items_per_sample(views[i]) * std::min(k, views[i].sample_count);
            if (views[i].sample_count > k) f += 3ull * views[i].width * views[i].height;
        }
        return f;
    };
    uint32_t chunk = std::max(max_spp, 1u);
    if (all_floats > limit) {
        if (need(1) > limit) return fail(SOL_GPU_ERR_OUT_OF_MEMORY, "batch films too large for the wavefront's scratch");
        uint32_t lo = 1, hi = max_spp;   // largest k with need(k) <= limit
        while (hi - lo > 1) { const uint32_t mid = lo + (hi - lo) / 2; if (need(mid) <= limit) lo = mid; else hi = mid; }
        chunk = lo;
    }
    const uint64_t scratch_floats = std::max<uint64_t>(need(chunk), 1);
    if (b->scratch_floats < scratch_floats) {
        cudaFree(b->scratch);
        b->scratch = nullptr;
        b->scratch_floats = 0;
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->scratch), scratch_floats * sizeof(float));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc wavefront scratch");
        b->scratch_floats = scratch_floats;
    }
    // Running sums sit after the largest chunk's per-sample planes; each
    // chunked view keeps its place across chunks.
    std::vector<uint64_t> running_at(n, 0);
    {
        uint64_t at = 0;
        for (uint32_t i = 0; i < n; ++i) at += 4ull * items_per_sample(views[i]) * std::min(chunk, views[i].sample_count);
        for (uint32_t i = 0; i < n; ++i)
            if (views[i].sample_count > chunk) { running_at[i] = at; at += 3ull * views[i].width * views[i].height; }
    }
    std::vector<WfView> table;
    std::vector<WfPass> passes;
    uint64_t paths = 0;
    for (uint32_t c0 = 0; c0 < max_spp; c0 += chunk) {
        WfPass pass;
        pass.first_view = table.size();
        uint64_t items = 0, scratch_at = 0;
        for (uint32_t i = 0; i < n; ++i) {
            const SolGpuView& s = views[i];
            if (s.sample_count <= c0) continue;
            const uint32_t k = std::min(chunk, s.sample_count - c0);
            WfView w{};
            std::memcpy(w.eye, s.camera.eye, sizeof(w.eye));
            std::memcpy(w.dir, s.camera.dir, sizeof(w.dir));
            std::memcpy(w.right, s.camera.right, sizeof(w.right));
            std::memcpy(w.up, s.camera.up, sizeof(w.up));
            w.scene = s.scene;
            w.width = s.width;
            w.height = s.height;
            w.sample_count = k;
            w.sample_index = s.sample_index + c0;
            w.film = s.film;
            w.tiles_x = (s.width + 7) / 8;
            w.item_begin = (uint32_t)items;
            w.split = 1;
            w.scratch = b->scratch + scratch_at;
            w.sum_begin = pass.sum_pixels;
            w.running = s.sample_count > chunk ? b->scratch + running_at[i] : nullptr;
            w.first_chunk = c0 == 0;
            w.last_chunk = c0 + k >= s.sample_count;
            scratch_at += 4ull * items_per_sample(s) * k;
            pass.sum_pixels += (uint64_t)s.width * s.height;
            items += (uint64_t)w.tiles_x * ((s.height + 3) / 4) * 32 * k;
            paths += (uint64_t)s.width * s.height * k;
            if (items > 0xffffffffull) return fail(SOL_GPU_ERR_INVALID_ARG, "batch too large (more than 2^32 work items)");
            table.push_back(w);
        }
        pass.num_views = (uint32_t)(table.size() - pass.first_view);
        pass.total_items = (uint32_t)items;
        passes.push_back(pass);
    }
    if (b->views_cap < table.size()) {
        cudaFree(b->d_views);
        b->d_views = nullptr;
        b->views_cap = 0;
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->d_views), sizeof(WfView) * std::max<size_t>(table.size(), 64));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc views");
        b->views_cap = std::max<size_t>(table.size(), 64);
    }
    // Copies from pageable host memory are staged before cudaMemcpyAsync
    // returns (CUDA runtime API, "API synchronization behavior"), so the host
    // tables and parameters may change right after each call.
    cudaError_t e = cudaSuccess;
    if (!table.empty())
        e = cudaMemcpyAsync(b->d_views, table.data(), sizeof(WfView) * table.size(), cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return cuda_fail(e, "views upload");
    uint32_t want = b->opts.capacity ? b->opts.capacity : kDefaultCapacity;
    want = std::min<uint32_t>(std::max<uint32_t>(want, 32), kMaxCapacity);
    // No more slots than the largest chunk has work items.
    uint64_t most_items = 32;
    for (const WfPass& pass : passes) most_items = std::max<uint64_t>(most_items, pass.total_items);
    want = (uint32_t)std::min<uint64_t>(want, most_items);
    int rc = alloc_pool(b, want);
    if (rc != SOL_GPU_OK) return rc;
    rc = configure_launch(b);
    if (rc != SOL_GPU_OK) return rc;
    WfParams& h = b->host;
    const bool ray_sort = b->opts.ray_order == SOL_GPU_RAY_ORDER_SORTED;
    const bool packed = b->opts.ray_order == SOL_GPU_RAY_ORDER_PACKED_SHADOWS;
    if (ray_sort != b->graph_sort || packed != b->graph_packed) {
        destroy_graph(b);
        b->graph_sort = ray_sort;
        b->graph_packed = packed;
    }
    h.ray_sort = ray_sort ? 1u : 0u;
    h.shadow_packed = packed ? 1u : 0u;
    {
        uint32_t bits = 0;
        while ((1u << bits) < b->scenes.size()) ++bits;
        h.scene_bits = bits;
    }
    h.scene_box = b->d_scene_box;
    h.sort_bins = b->d_sort_bins;
    h.sort_threshold = b->opts.sort_threshold;
    h.refill_below = kWfRefillBelow;
    h.cfg = to_config(*config);
    h.ctr = b->d_ctr;
    cudaEventRecord(b->ev_start, stream);
    bool first_pass = true;
    for (const WfPass& pass : passes) {
        if (pass.num_views == 0) continue;
        h.keep_counts = first_pass ? 0u : 1u;   // counters add up over the chunks of samples
        first_pass = false;
        h.capacity = (uint32_t)std::min<uint64_t>(want, std::max<uint64_t>(pass.total_items, 32));
        h.num_views = pass.num_views;
        h.total_items = pass.total_items;
        h.views = b->d_views + pass.first_view;
        // Bound on bounce iterations: a path takes at most max_path_len + 1
        // of them (its start and each vertex) and a slot runs its paths one
        // after the other, so no render of these items needs more than
        // items x (max_path_len + 2).
        h.max_iterations = b->max_iterations ? b->max_iterations
                                             : (unsigned long long)pass.total_items * (config->max_path_len + 2ull) + 16ull;
        e = cudaMemcpyAsync(b->d_params, &h, sizeof(WfParams), cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return cuda_fail(e, "params upload");
        e = launch_wf_init(b->d_params, h.capacity, stream);
        if (e != cudaSuccess) return cuda_fail(e, "wavefront init");
        if (!b->opts.host_loop && build_graph(b) == SOL_GPU_OK) {
            e = cudaGraphLaunch(b->exec, stream);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
        } else {
            // Host-driven loop: the same stages, one iteration per round trip.
            cudaGraphConditionalHandle none{};
            for (uint64_t it = 0;; ++it) {
                e = launch_wf_iteration(b->d_params, b->wf_table, b->basic, ray_sort, packed, b->launch, none, 0,
                                        stream);
                if (e == cudaSuccess) e = cudaMemcpyAsync(b->h_ctr, b->d_ctr, sizeof(WfCounters), cudaMemcpyDeviceToHost, stream);
                if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
                if (e != cudaSuccess) return cuda_fail(e, "wavefront iteration");
                if (!b->h_ctr->more) break;
                if (it > h.max_iterations) return fail(SOL_GPU_ERR_TIMEOUT, "bounce loop exceeded its bound");
            }
        }
        e = launch_sum_items_views(h.views, pass.num_views, pass.sum_pixels, stream);
        if (e != cudaSuccess) return cuda_fail(e, "sum pass");
    }
    cudaEventRecord(b->ev_stop, stream);
    b->rendered = true;
    b->last_dc = false;
    b->last_passes = (uint32_t)passes.size();
    (void)paths;
    return SOL_GPU_OK;
}

int render_batch(SolGpuBatch* b, const SolGpuConfig* config, const SolGpuView* views, uint32_t n, cudaStream_t stream) {
    int rc = refresh_scenes(b);
    if (rc != SOL_GPU_OK) return rc;
    if (b->opts.schedule == SOL_GPU_BATCH_MEGAKERNEL) return render_megakernel(b, config, views, n, stream);
    return render_wavefront(b, config, views, n, stream);
}

std::string device_name(int device) {
    cudaDeviceProp p{};
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return "unknown";
    return p.name;
}

std::string tune_key(SolGpuBatch* b, const SolGpuView* views, uint32_t n) {
    uint64_t px = 0, tris = 0;
    for (uint32_t i = 0; i < n; ++i) px += (uint64_t)views[i].width * views[i].height;
    for (auto* s : b->scenes) tris += s->info.num_triangles;
    std::ostringstream k;
    k << device_name(b->device) << "|views=" << n << "|px2=" << (int)std::lround(std::log2((double)std::max<uint64_t>(px, 1)))
      << "|tri2=" << (int)std::lround(std::log2((double)std::max<uint64_t>(tris, 1)));
    return k.str();
}

bool read_cache(const char* path, const std::string& key, SolGpuBatchOptions* o) {
    std::ifstream f(path);
    std::string line;
    bool found = false;
    while (std::getline(f, line)) {
        std::istringstream in(line);
        std::string k;
        SolGpuBatchOptions r{};
        if (std::getline(in, k, '\t') && (in >> r.capacity >> r.block_size >> r.sort_threshold) && k == key) {
            if (!(in >> r.schedule)) r.schedule = SOL_GPU_BATCH_WAVEFRONT;
            if (!(in >> r.ray_order)) r.ray_order = SOL_GPU_RAY_ORDER_DEFAULT;
            *o = r;
            found = true;
        }
    }
    return found;
}

}  // namespace

extern "C" {

int sol_gpu_batch_create(SolGpuScene* const* scenes, uint32_t num_scenes, const SolGpuBatchOptions* options,
                         SolGpuBatch** out) {
    if (!scenes || num_scenes == 0 || !out) return fail(SOL_GPU_ERR_INVALID_ARG, "scenes and out must not be NULL");
    *out = nullptr;
    const int device = scenes[0]->device;
    for (uint32_t i = 0; i < num_scenes; ++i) {
        if (!scenes[i]) return fail(SOL_GPU_ERR_INVALID_ARG, "scene must not be NULL");
        if (scenes[i]->device != device) return fail(SOL_GPU_ERR_INVALID_ARG, "all scenes of a batch must be on one device");
    }
    DeviceGuard guard(device);
    if (guard.err != cudaSuccess) return cuda_fail(guard.err, "cudaSetDevice");
    auto* b = new SolGpuBatch();
    b->device = device;
    b->scenes.assign(scenes, scenes + num_scenes);
    if (options) b->opts = *options;
    std::vector<SceneView> views(num_scenes);
    for (uint32_t i = 0; i < num_scenes; ++i) views[i] = scenes[i]->view;
    b->h_scenes = views;
    for (uint32_t i = 0; i < num_scenes && i < kWfMaxScenes; ++i) b->wf_table.v[i] = views[i];
    b->basic = std::all_of(b->scenes.begin(), b->scenes.end(), [](const SolGpuScene* s) { return s->basic_shading; });
    cudaError_t e = cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&b->d_params), sizeof(WfParams));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&b->d_ctr), sizeof(WfCounters));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&b->d_scenes), sizeof(SceneView) * num_scenes);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_scenes, views.data(), sizeof(SceneView) * num_scenes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        // Scene bounds for the reordering keys: the union of the root's two child boxes.
        std::vector<float4> boxes(2 * (size_t)num_scenes, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
        for (uint32_t i = 0; i < num_scenes && e == cudaSuccess; ++i) {
            boxes[2 * i + 1] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
            if (scenes[i]->view.num_nodes == 0) continue;
            DNode root{};
            e = cudaMemcpy(&root, scenes[i]->nodes, sizeof(DNode), cudaMemcpyDeviceToHost);
            boxes[2 * i] = make_float4(std::min(root.b0[0], root.b1[0]), std::min(root.b0[2], root.b1[2]),
                                       std::min(root.b2[0], root.b2[2]), 0.0f);
            boxes[2 * i + 1] = make_float4(std::max(root.b0[1], root.b1[1]), std::max(root.b0[3], root.b1[3]),
                                           std::max(root.b2[1], root.b2[3]), 0.0f);
        }
        if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&b->d_scene_box), sizeof(float4) * boxes.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(b->d_scene_box, boxes.data(), sizeof(float4) * boxes.size(), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&b->d_sort_bins), 2 * sizeof(uint32_t) * kWfSortBins);
    if (e == cudaSuccess) e = cudaMemset(b->d_sort_bins, 0, 2 * sizeof(uint32_t) * kWfSortBins);
    if (e == cudaSuccess) e = allow_sort_smem();
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&b->h_ctr), sizeof(WfCounters));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev_start);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev_stop);
    if (e != cudaSuccess) {
        int rc = cuda_fail(e, "batch create");
        sol_gpu_batch_destroy(b);
        return rc;
    }
    *out = b;
    return SOL_GPU_OK;
}

int sol_gpu_batch_destroy(SolGpuBatch* b) {
    if (!b) return fail(SOL_GPU_ERR_INVALID_ARG, "batch must not be NULL");
    DeviceGuard guard(b->device);
    cudaDeviceSynchronize();
    destroy_graph(b);
    cudaFree(b->pool);
    cudaFree(b->d_params);
    cudaFree(b->d_ctr);
    cudaFree(b->d_scenes);
    cudaFree(b->d_views);
    cudaFree(b->d_adj_views);
    cudaFree(b->d_dc);
    cudaFree(b->scratch);
    cudaFree(b->d_scene_box);
    cudaFree(b->d_sort_bins);
    if (b->h_ctr) cudaFreeHost(b->h_ctr);
    if (b->capture) cudaStreamDestroy(b->capture);
    if (b->ev_start) cudaEventDestroy(b->ev_start);
    if (b->ev_stop) cudaEventDestroy(b->ev_stop);
    delete b;
    return SOL_GPU_OK;
}

int sol_gpu_batch_render(SolGpuBatch* b, const SolGpuConfig* config, const SolGpuView* views, uint32_t num_views,
                         void* stream) {
    if (!b || !config || (num_views > 0 && !views)) return fail(SOL_GPU_ERR_INVALID_ARG, "batch, config and views must not be NULL");
    DeviceGuard guard(b->device);
    if (guard.err != cudaSuccess) return cuda_fail(guard.err, "cudaSetDevice");
    return render_batch(b, config, views, num_views, static_cast<cudaStream_t>(stream));
}

int sol_gpu_batch_forward_adjoint(SolGpuBatch* b, const SolGpuConfig* config, const SolGpuAdjointView* views,
                                  uint32_t n, void* stream) {
    if (!b || !config || (n > 0 && !views)) return fail(SOL_GPU_ERR_INVALID_ARG, "batch, config and views must not be NULL");
    if (config->max_path_len > (uint32_t)kAdjointMaxDepth)
        return fail(SOL_GPU_ERR_UNSUPPORTED, "the adjoint replays paths of at most 16 vertices");
    DeviceGuard guard(b->device);
    if (guard.err != cudaSuccess) return cuda_fail(guard.err, "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<AdjView> v(n);
    uint64_t items = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const SolGpuAdjointView& a = views[i];
        if (a.view.scene >= b->scenes.size()) return fail(SOL_GPU_ERR_INVALID_ARG, "view scene index out of range");
        if (a.view.width == 0 || a.view.height == 0 || a.view.sample_count == 0)
            return fail(SOL_GPU_ERR_INVALID_ARG, "view size and sample count must be positive");
        if (!a.view.film || !a.target || !a.grad || !a.loss) return fail(SOL_GPU_ERR_INVALID_ARG, "view buffers must not be NULL");
        AdjView& w = v[i];
        w.cam = to_camera(a.view.camera);
        w.scene = a.view.scene;
        w.width = a.view.width;
        w.height = a.view.height;
        w.sample_count = a.view.sample_count;
        w.sample_index = a.view.sample_index;
        w.film = a.view.film;
        w.target = a.target;
        w.grad = a.grad;
        w.loss = a.loss;
        w.item_begin = (uint32_t)items;
        w.group = fused_group(a.view.sample_count);
        items += fused_items(a.view.width, a.view.height, a.view.sample_count);
        if (items > 0xffffffffull) return fail(SOL_GPU_ERR_INVALID_ARG, "batch too large");
    }
    cudaError_t e = cudaSuccess;
    if (b->adj_views_cap < n) {
        cudaFree(b->d_adj_views);
        b->d_adj_views = nullptr;
        b->adj_views_cap = 0;
        e = cudaMalloc(reinterpret_cast<void**>(&b->d_adj_views), sizeof(AdjView) * std::max<size_t>(n, 32));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc views");
        b->adj_views_cap = std::max<size_t>(n, 32);
    }
    if (!b->d_dc) {
        e = cudaMalloc(reinterpret_cast<void**>(&b->d_dc), sizeof(DeviceCounters));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc counters");
    }
    if (n > 0) e = cudaMemcpyAsync(b->d_adj_views, v.data(), sizeof(AdjView) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_dc, 0, sizeof(DeviceCounters), st);
    if (e != cudaSuccess) return cuda_fail(e, "fused batch upload");
    const int per_sm = fused_blocks_per_sm();
    if (per_sm <= 0) return fail(SOL_GPU_ERR_CUDA, "fused kernel occupancy query failed");
    cudaEventRecord(b->ev_start, st);
    if (n > 0) {
        e = launch_fused_forward_adjoint(b->d_adj_views, n, (uint32_t)items, b->d_scenes, to_config(*config),
                                         b->d_dc, per_sm * b->num_sms, st);
        if (e != cudaSuccess) return cuda_fail(e, "fused forward/adjoint launch");
    }
    cudaEventRecord(b->ev_stop, st);
    b->rendered = true;
    b->last_dc = true;
    return SOL_GPU_OK;
}

int sol_gpu_batch_stats(SolGpuBatch* b, SolGpuRenderStats* out) {
    if (!b || !out) return fail(SOL_GPU_ERR_INVALID_ARG, "batch and out must not be NULL");
    std::memset(out, 0, sizeof(*out));
    if (!b->rendered) return SOL_GPU_OK;
    DeviceGuard guard(b->device);
    cudaError_t e = cudaEventSynchronize(b->ev_stop);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventSynchronize");
    if (b->last_dc) {
        DeviceCounters c;
        e = cudaMemcpy(&c, b->d_dc, sizeof(c), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "counters");
        out->paths = c.paths;
        out->rays = c.rays;
        out->shadow_rays = c.shadow_rays;
    } else {
        WfCounters c;
        e = cudaMemcpy(&c, b->d_ctr, sizeof(c), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "counters");
        out->paths = c.paths;
        out->rays = c.rays;
        out->shadow_rays = c.shadow_rays;
        out->launches = b->last_passes;
        if (c.error & kFaultPathLoop) {
            for (SolGpuScene* sc : b->scenes) check_fault(sc);   // clear what the stopped render left
            return fail(SOL_GPU_ERR_TIMEOUT, "the wavefront's bounce loop reached its iteration bound");
        }
        if (c.error) return fail(SOL_GPU_ERR_BAD_INDEX, "a wavefront self-check failed (flags " + std::to_string(c.error) + ")");
    }
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, b->ev_start, b->ev_stop) == cudaSuccess) out->kernel_ms = ms;
    for (SolGpuScene* sc : b->scenes) {
        int rc = check_fault(sc);
        if (rc != SOL_GPU_OK) return rc;
    }
    return SOL_GPU_OK;
}

int sol_gpu_batch_set_scratch_limit(SolGpuBatch* b, uint64_t bytes) {
    if (!b) return fail(SOL_GPU_ERR_INVALID_ARG, "batch must not be NULL");
    b->scratch_limit = bytes;
    return SOL_GPU_OK;
}

int sol_gpu_batch_set_iteration_limit(SolGpuBatch* b, uint64_t max_iterations) {
    if (!b) return fail(SOL_GPU_ERR_INVALID_ARG, "batch must not be NULL");
    b->max_iterations = max_iterations;
    return SOL_GPU_OK;
}

int sol_gpu_batch_autotune(SolGpuBatch* b, const SolGpuConfig* config, const SolGpuView* views, uint32_t num_views,
                           const char* cache_path, SolGpuBatchOptions* chosen) {
    if (!b || !config || !views || num_views == 0) return fail(SOL_GPU_ERR_INVALID_ARG, "batch, config and views are required");
    DeviceGuard guard(b->device);
    if (guard.err != cudaSuccess) return cuda_fail(guard.err, "cudaSetDevice");
    if (b->opts.schedule == SOL_GPU_BATCH_MEGAKERNEL) {   // nothing to choose
        if (chosen) *chosen = b->opts;
        return SOL_GPU_OK;
    }
    const bool both = b->opts.schedule == SOL_GPU_BATCH_AUTO;
    const std::string key = tune_key(b, views, num_views) + (both ? "|auto" : "|wavefront");
    SolGpuBatchOptions best = b->opts;
    if (cache_path && read_cache(cache_path, key, &best)) {
        best.host_loop = b->opts.host_loop;
        b->opts = best;
        if (chosen) *chosen = best;
        return SOL_GPU_OK;
    }
    // Probe: one sample per pixel of every view, into scratch films.
    std::vector<SolGpuView> probe(views, views + num_views);
    size_t floats = 0;
    for (auto& v : probe) floats += 3 * (size_t)v.width * v.height;
    float* scratch = nullptr;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&scratch), sizeof(float) * std::max<size_t>(floats, 1));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc autotune films");
    size_t off = 0;
    // Up to four samples per pixel: enough work items that the pool sizes differ.
    for (auto& v : probe) {
        v.film = scratch + off;
        off += 3 * (size_t)v.width * v.height;
        v.sample_count = std::min<uint32_t>(v.sample_count, 4);
    }
    cudaStream_t s = b->capture;
    // Pool capacities up to kMaxCapacity (64M slots, about 17 GB); those whose
    // pool would not fit in the device's free memory (plus the pool this
    // batch already holds) with 1 GiB to spare are skipped.
    const uint32_t caps[] = {1u << 21, 1u << 22, 1u << 23, 1u << 24, 1u << 25, 1u << 26};
    size_t free_bytes = 0, total_bytes = 0;
    e = cudaMemGetInfo(&free_bytes, &total_bytes);
    if (e != cudaSuccess) { cudaFree(scratch); return cuda_fail(e, "cudaMemGetInfo"); }
    const size_t room = free_bytes + (b->pool ? pool_bytes(b->allocated) : 0);
    const uint32_t blocks[] = {128, 256};
    const uint32_t sorts[] = {0u, 1u << 16, 0xffffffffu};
    const int32_t orders[] = {SOL_GPU_RAY_ORDER_QUEUE, SOL_GPU_RAY_ORDER_PACKED_SHADOWS};
    float best_ms = 1e30f;
    int rc = SOL_GPU_OK;
    const SolGpuBatchOptions saved = b->opts;
    for (uint32_t cap : caps) {
        if (cap > kMaxCapacity || pool_bytes(cap) + (size_t(1) << 30) > room) continue;
        for (uint32_t blk : blocks) {
            for (uint32_t srt : sorts) {
                for (int32_t order : orders) {
                    b->opts.capacity = cap;
                    b->opts.block_size = blk;
                    b->opts.sort_threshold = srt;
                    b->opts.ray_order = order;
                    float ms = 0.0f;
                    for (int rep = 0; rep < 2 && rc == SOL_GPU_OK; ++rep) {   // first run warms the graph
                        rc = render_batch(b, config, probe.data(), num_views, s);
                        if (rc == SOL_GPU_OK) {
                            e = cudaEventSynchronize(b->ev_stop);
                            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, b->ev_start, b->ev_stop);
                            if (e != cudaSuccess) rc = cuda_fail(e, "autotune timing");
                        }
                    }
                    if (rc != SOL_GPU_OK) break;
                    if (ms < best_ms) { best_ms = ms; best = b->opts; }
                }
            }
        }
    }
    if (rc == SOL_GPU_OK) {
        // Every candidate above ran as the wavefront; name it so.
        best.schedule = SOL_GPU_BATCH_WAVEFRONT;
    }
    if (rc == SOL_GPU_OK && both) {
        b->opts = saved;
        b->opts.schedule = SOL_GPU_BATCH_MEGAKERNEL;
        float ms = 0.0f;
        for (int rep = 0; rep < 2 && rc == SOL_GPU_OK; ++rep) {
            rc = render_batch(b, config, probe.data(), num_views, s);
            if (rc == SOL_GPU_OK) {
                e = cudaEventSynchronize(b->ev_stop);
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, b->ev_start, b->ev_stop);
                if (e != cudaSuccess) rc = cuda_fail(e, "autotune timing");
            }
        }
        if (rc == SOL_GPU_OK && ms < best_ms) { best_ms = ms; best = b->opts; }
    }
    cudaFree(scratch);
    if (rc != SOL_GPU_OK) { b->opts = saved; return rc; }
    best.host_loop = saved.host_loop;
    b->opts = best;
    if (chosen) *chosen = best;
    if (cache_path) {
        std::ofstream f(cache_path, std::ios::app);
        f << key << '\t' << best.capacity << ' ' << best.block_size << ' ' << best.sort_threshold << ' '
          << best.schedule << ' ' << best.ray_order << '\n';
    }
    return SOL_GPU_OK;
}

}  // extern "C"
