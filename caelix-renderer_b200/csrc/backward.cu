// The adjoint of the trace (path replay): gradients of an image loss with respect to the albedo
// of every material and the emitter power of every brick.
//
// The forward estimator is the per-frame kernel's (trace.cu trace_pixel, the reference's
// shaders/render/caelix_path_trace.hlsl:737-978 integrator). Its parameter-dependent factors are
//   * the primary albedo a0 and emission e0: pixel sample = e0 + a0 * sanitize(R);
//   * the albedo of every bounce vertex, a factor of the throughput of everything after it;
//   * the power of every emitting brick the path reaches: an emitter hit adds
//     power * throughput * w_mis, an NEE vertex adds power * s * throughput (s: the geometry,
//     pdf and MIS factors of the light sample).
// The sampling quantities (pdfs, MIS weights, Russian-roulette probabilities, every discrete
// decision) are held fixed (detached), so a sample is a polynomial in the parameters and
//   dL/da0[c]          = g[c] * sanitize(R)[c]
//   dL/de0             = g[0] + g[1] + g[2]
//   dL/dR[c]           = G[c] = g[c] * a0[c] (0 where sanitize clamps)
//   dL/dalbedo_j[c]    = G[c] * (R[c] - R_before_j[c]) / albedo_j[c]
//   dL/dpower_b        = sum_c G[c] * (throughput[c] * w_mis  or  s * throughput[c])
// with g = dL/d(pixel) / spp and R_before_j the radiance gathered before vertex j's albedo
// multiplies the throughput. The frame is traced twice with the wavefront kernels (wave.cu): a
// recording pass (bit-identical to the render) that keeps every sample's R (an image-sized
// buffer per sample index; nothing of the paths), then a replay of every path, in the same
// queues, that gathers the gradients: the power gradient of an NEE lamp is held in the path's
// slot until its shadow ray is found unoccluded. Albedo gradients are summed per CTA in shared
// memory, power gradients with global atomics.
#include <algorithm>
#include <cstdint>
#include <cstring>

#include "trace.cuh"

namespace cx {

namespace {

constexpr uint32_t kAdjointBlockWidth = 8;

uint64_t align256(uint64_t x) { return (x + 255u) & ~uint64_t{255}; }

}  // namespace

uint64_t adjoint_bytes(const TraceParams& p, uint32_t wave_capacity)
{
    WaveView v;
    std::memset(&v, 0, sizeof(v));
    v.params = p;
    v.blocks_x = (p.width + kAdjointBlockWidth - 1) / kAdjointBlockWidth;
    const WavePlan plan = wave_plan(&v, 1, kAdjointBlockWidth);
    const uint32_t items = plan.items.empty() ? 32 : plan.items[0];
    const uint32_t capacity = wave_capacity ? std::min(wave_capacity, items) : items;
    return 2 * align256(sizeof(WaveView)) + align256(4ull * plan.table.size()) +
           align256(12ull * p.spp * p.width * p.height) + wave_buffer_bytes(capacity);
}

cudaError_t adjoint_launch(const SceneView& s, const TraceParams& p, const float* d_radiance, float* image,
                           float* d_albedo, float* d_power, unsigned long long* ray_counts, void* memory,
                           uint32_t wave_capacity, uint32_t sm_count, cudaStream_t stream, uint32_t* launches)
{
    WaveView views[2];
    std::memset(views, 0, sizeof(views));
    views[0].scene = s;
    views[0].params = p;
    views[0].radiance = image;
    views[0].ray_counts = ray_counts;
    views[0].blocks_x = (p.width + kAdjointBlockWidth - 1) / kAdjointBlockWidth;
    views[1] = views[0];
    views[1].radiance = nullptr;    // the replay writes no image
    views[1].ray_counts = nullptr;  // and counts no rays
    const WavePlan plan = wave_plan(views, 1, kAdjointBlockWidth);
    const uint32_t items = plan.items.empty() ? 32 : plan.items[0];
    const uint32_t capacity = wave_capacity ? std::min(wave_capacity, items) : items;
    char* m = static_cast<char*>(memory);
    WaveView* d_record = reinterpret_cast<WaveView*>(m);
    m += align256(sizeof(WaveView));
    WaveView* d_replay = reinterpret_cast<WaveView*>(m);
    m += align256(sizeof(WaveView));
    uint32_t* d_table = reinterpret_cast<uint32_t*>(m);
    m += align256(4ull * plan.table.size());
    float* samples = reinterpret_cast<float*>(m);
    m += align256(12ull * p.spp * p.width * p.height);
    const WaveBuffers wb = wave_carve(m, capacity);
    CX_TRY(cudaMemcpyAsync(d_record, &views[0], sizeof(WaveView), cudaMemcpyHostToDevice, stream));
    CX_TRY(cudaMemcpyAsync(d_replay, &views[1], sizeof(WaveView), cudaMemcpyHostToDevice, stream));
    CX_TRY(cudaMemcpyAsync(d_table, plan.table.data(), 4 * plan.table.size(), cudaMemcpyHostToDevice, stream));
    WaveAdjoint adj;
    adj.d_radiance = d_radiance;
    adj.sample_radiance = samples;
    adj.d_albedo = d_albedo;
    adj.d_power = d_power;
    return wave_adjoint(s, d_record, d_replay, plan, d_table, wb, kAdjointBlockWidth, sm_count, adj, stream,
                        launches);
}

}  // namespace cx
