// C-ABI host runtime: contexts, device workspaces, host<->device staging and
// kernel launches for the entry points declared in include/lcbinint_b200.h.
#include "../../include/lcbinint_b200.h"
#include "lcbi_context.h"
#include "lcbi_kernels.h"

#include <cstdio>
#include <cstring>
#include <new>
#include <string>

using lcbi::Context;

namespace lcbi {

bool Context::fail(const char* what, cudaError_t e)
{
    error = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}

bool Context::fail(const std::string& what)
{
    error = what;
    return false;
}

bool Context::ensure(Buffer& b, size_t bytes)
{
    if (b.bytes >= bytes) return true;
    if (b.ptr) {
        cudaFree(b.ptr);
        b.ptr = nullptr;
        b.bytes = 0;
    }
    size_t want = bytes < 4096 ? 4096 : bytes;
    want = (want + 0xffff) & ~size_t(0xffff);
    const cudaError_t e = cudaMalloc(&b.ptr, want);
    if (e != cudaSuccess) return fail("cudaMalloc", e);
    b.bytes = want;
    return true;
}

bool Context::check(const char* what, cudaError_t e)
{
    if (e == cudaSuccess) return true;
    return fail(what, e);
}

Context::~Context()
{
    cudaSetDevice(device);
    for (Buffer* b : all_buffers()) {
        if (b->ptr) cudaFree(b->ptr);
    }
    if (pinned) cudaFreeHost(pinned);
    for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
    for (auto& p : pending) {
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
    }
    if (fork_event) cudaEventDestroy(fork_event);
    if (join_event) cudaEventDestroy(join_event);
    if (side_stream) cudaStreamDestroy(side_stream);
    if (early_fork) cudaEventDestroy(early_fork);
    if (early_join) cudaEventDestroy(early_join);
    if (early_seeded) cudaEventDestroy(early_seeded);
    for (cudaEvent_t e : marks)
        if (e) cudaEventDestroy(e);
    if (early_stream) cudaStreamDestroy(early_stream);
    if (own_stream) cudaStreamDestroy(own_stream);
}

void Context::stage_begin(int stage, cudaEvent_t* ev)
{
    (void)stage;
    *ev = nullptr;
    if (!timing) return;
    if (event_pool.empty()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        event_pool.push_back(e);
    }
    *ev = event_pool.back();
    event_pool.pop_back();
    cudaEventRecord(*ev, stream);
}

void Context::stage_end(int stage, cudaEvent_t begin)
{
    if (!timing || begin == nullptr) return;
    cudaEvent_t e;
    if (event_pool.empty()) {
        if (cudaEventCreate(&e) != cudaSuccess) return;
    } else {
        e = event_pool.back();
        event_pool.pop_back();
    }
    cudaEventRecord(e, stream);
    pending.push_back({stage, {begin, e}});
}

void Context::collect_timing()
{
    for (auto& p : pending) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, p.second.first, p.second.second) == cudaSuccess && p.first >= 0 &&
            p.first < kStages) {
            stage_ms[p.first] += ms;
            stage_launches[p.first] += 1;
        }
        event_pool.push_back(p.second.first);
        event_pool.push_back(p.second.second);
    }
    pending.clear();
}

// Stages `count` elements of an input array: device pointers pass through,
// host arrays are copied into `buf`.
template <typename T>
bool Context::stage_in(Buffer& buf, const T* src, size_t count, bool device_ptrs, const T** out)
{
    if (device_ptrs) {
        *out = src;
        return true;
    }
    if (!ensure(buf, count * sizeof(T))) return false;
    if (count && !check("cudaMemcpyAsync H2D",
                        cudaMemcpyAsync(buf.ptr, src, count * sizeof(T), cudaMemcpyHostToDevice, stream)))
        return false;
    *out = static_cast<const T*>(buf.ptr);
    return true;
}

template <typename T>
bool Context::stage_out(Buffer& buf, T* dst, size_t count, bool device_ptrs, T** out)
{
    if (device_ptrs || dst == nullptr) {
        *out = dst;
        return true;
    }
    if (!ensure(buf, count * sizeof(T))) return false;
    *out = static_cast<T*>(buf.ptr);
    return true;
}

template <typename T>
bool Context::copy_back(T* dst, const T* dev, size_t count, bool device_ptrs)
{
    if (device_ptrs || dst == nullptr || count == 0) return true;
    return check("cudaMemcpyAsync D2H", cudaMemcpyAsync(dst, dev, count * sizeof(T), cudaMemcpyDeviceToHost, stream));
}

bool Context::finish()
{
    const bool ok = check("cudaStreamSynchronize", cudaStreamSynchronize(stream));
    if (ok) collect_timing();
    return ok;
}

template bool Context::stage_in<double>(Buffer&, const double*, size_t, bool, const double**);
template bool Context::stage_in<int>(Buffer&, const int*, size_t, bool, const int**);
template bool Context::stage_out<double>(Buffer&, double*, size_t, bool, double**);
template bool Context::stage_out<int>(Buffer&, int*, size_t, bool, int**);
template bool Context::copy_back<double>(double*, const double*, size_t, bool);
template bool Context::copy_back<int>(int*, const int*, size_t, bool);

// Point-source batches from host memory of at least two chunks: chunks of
// kPsChunk positions go round-robin to the context's three streams, each
// chunk's copies in, kernel and copies out in order on its stream, so the
// copies of some chunks run on the copy engines while the kernels of others
// run on the SMs.  Every position's result is the kernel's, so the results
// are those of one launch over the whole batch.  (With pinned host memory
// the copies are asynchronous; pageable memory still gives correct results,
// with less overlap.)
constexpr size_t kPsChunk = size_t(1) << 18;

int ps_pipelined(Context* ctx, size_t N, const double* s, const double* q, const double* y1, const double* y2,
                 double* A, int32_t* image_count, int32_t* status)
{
    if (!ctx->ensure(ctx->in[0], N * sizeof(double)) || !ctx->ensure(ctx->in[1], N * sizeof(double)) ||
        !ctx->ensure(ctx->in[2], N * sizeof(double)) || !ctx->ensure(ctx->in[3], N * sizeof(double)) ||
        !ctx->ensure(ctx->out[0], N * sizeof(double)) ||
        (image_count && !ctx->ensure(ctx->out[1], N * sizeof(int))) ||
        (status && !ctx->ensure(ctx->out[2], N * sizeof(int))))
        return LCBI_GPU_ERROR;
    cudaStream_t streams[3] = {ctx->stream, ctx->side_stream, ctx->early_stream};
    if (!ctx->check("fork", cudaEventRecord(ctx->fork_event, ctx->stream)) ||
        !ctx->check("fork", cudaStreamWaitEvent(ctx->side_stream, ctx->fork_event, 0)) ||
        !ctx->check("fork", cudaStreamWaitEvent(ctx->early_stream, ctx->fork_event, 0)))
        return LCBI_GPU_ERROR;
    const double* hin[4] = {s, q, y1, y2};
    bool ok = true;
    size_t c = 0;
    for (size_t off = 0; off < N && ok; off += kPsChunk, ++c) {
        const size_t m = N - off < kPsChunk ? N - off : kPsChunk;
        cudaStream_t st = streams[c % 3];
        double* din[4];
        for (int k = 0; k < 4 && ok; ++k) {
            din[k] = static_cast<double*>(ctx->in[k].ptr) + off;
            ok = ctx->check("cudaMemcpyAsync H2D",
                            cudaMemcpyAsync(din[k], hin[k] + off, m * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        double* dA = static_cast<double*>(ctx->out[0].ptr) + off;
        int* dn = image_count ? static_cast<int*>(ctx->out[1].ptr) + off : nullptr;
        int* dst = status ? static_cast<int*>(ctx->out[2].ptr) + off : nullptr;
        ok = ok && ctx->check("ps_batch_kernel", launch_ps_batch(din[0], din[1], din[2], din[3], dA, dn, dst,
                                                                 static_cast<long long>(m), ctx->sm_count, st));
        ok = ok && ctx->check("cudaMemcpyAsync D2H",
                              cudaMemcpyAsync(A + off, dA, m * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (dn)
            ok = ok && ctx->check("cudaMemcpyAsync D2H", cudaMemcpyAsync(image_count + off, dn, m * sizeof(int),
                                                                         cudaMemcpyDeviceToHost, st));
        if (dst)
            ok = ok && ctx->check("cudaMemcpyAsync D2H",
                                  cudaMemcpyAsync(status + off, dst, m * sizeof(int), cudaMemcpyDeviceToHost, st));
        ctx->launches += 1;
    }
    // Joined even after a failure, so the context's stream never runs ahead
    // of work queued beside it.
    const bool joined = ctx->check("join", cudaEventRecord(ctx->join_event, ctx->side_stream)) &&
                        ctx->check("join", cudaStreamWaitEvent(ctx->stream, ctx->join_event, 0)) &&
                        ctx->check("join", cudaEventRecord(ctx->early_join, ctx->early_stream)) &&
                        ctx->check("join", cudaStreamWaitEvent(ctx->stream, ctx->early_join, 0));
    if (!joined || !ctx->finish() || !ok) return LCBI_GPU_ERROR;
    return LCBI_OK;
}

} // namespace lcbi

using lcbi::kPsChunk;
using lcbi::ps_pipelined;

extern "C" {

int lcbi_gpu_create(int device, lcbi_gpu_context** out)
{
    if (out == nullptr) return LCBI_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return LCBI_GPU_ERROR;
    }
    Context* ctx = new (std::nothrow) Context();
    if (!ctx) return LCBI_GPU_ERROR;
    ctx->device = device;
    int least = 0, greatest = 0;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ctx->side_stream, cudaStreamNonBlocking, greatest) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->fork_event, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->join_event, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ctx->early_stream, cudaStreamNonBlocking, greatest) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->early_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->early_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->early_seeded, cudaEventDisableTiming) != cudaSuccess ||
        cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return LCBI_GPU_ERROR;
    }
    ctx->stream = ctx->own_stream;
    *out = reinterpret_cast<lcbi_gpu_context*>(ctx);
    return LCBI_OK;
}

int lcbi_gpu_set_stream(lcbi_gpu_context* c, void* stream)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx) return LCBI_INVALID_ARGUMENT;
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    return LCBI_OK;
}

int lcbi_gpu_set_timing(lcbi_gpu_context* c, int enable)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx) return LCBI_INVALID_ARGUMENT;
    ctx->timing = enable != 0;
    for (int i = 0; i < Context::kStages; ++i) {
        ctx->stage_ms[i] = 0.0;
        ctx->stage_launches[i] = 0;
    }
    return LCBI_OK;
}

int lcbi_gpu_set_item_cycles(lcbi_gpu_context* c, int enable)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx) return LCBI_INVALID_ARGUMENT;
    ctx->item_cycles = enable != 0;
    return LCBI_OK;
}

int lcbi_gpu_set_cell_budget(lcbi_gpu_context* c, int64_t cells)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || cells < 0) return LCBI_INVALID_ARGUMENT;
    ctx->cell_budget = cells;
    ctx->cell_budget_set = true;
    return LCBI_OK;
}

int lcbi_gpu_set_seed_block_after(lcbi_gpu_context* c, int32_t sources)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || sources < 0) return LCBI_INVALID_ARGUMENT;
    ctx->seed_block_after = sources;
    return LCBI_OK;
}

int lcbi_gpu_set_ray_precision(lcbi_gpu_context* c, int32_t bits)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || (bits != 32 && bits != 64)) return LCBI_INVALID_ARGUMENT;
    ctx->f32_rays = bits == 32;
    return LCBI_OK;
}

int lcbi_gpu_set_grad_resolution(lcbi_gpu_context* c, int32_t cells_per_radius)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || cells_per_radius < 8 || cells_per_radius > 512) return LCBI_INVALID_ARGUMENT;
    ctx->grad_bins = cells_per_radius;
    return LCBI_OK;
}

int lcbi_gpu_set_stream_marks(lcbi_gpu_context* c, int enable)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx) return LCBI_INVALID_ARGUMENT;
    if (enable && ctx->marks[0] == nullptr) {
        if (cudaSetDevice(ctx->device) != cudaSuccess) return LCBI_GPU_ERROR;
        for (cudaEvent_t& e : ctx->marks)
            if (cudaEventCreate(&e) != cudaSuccess) {
                cudaGetLastError();
                return LCBI_GPU_ERROR;
            }
    }
    ctx->marks_on = enable != 0;
    ctx->marks_set = 0;
    return LCBI_OK;
}

int lcbi_gpu_stream_marks(lcbi_gpu_context* c, double* ms, int32_t n)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || !ms || n < 0) return LCBI_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return LCBI_GPU_ERROR;
    for (int i = 0; i < n && i < 3; ++i) {
        ms[i] = -1.0;
        float f = 0.0f;
        if ((ctx->marks_set & 1u) && (ctx->marks_set & (2u << i)) &&
            cudaEventSynchronize(ctx->marks[i + 1]) == cudaSuccess &&
            cudaEventElapsedTime(&f, ctx->marks[0], ctx->marks[i + 1]) == cudaSuccess)
            ms[i] = f;
    }
    return LCBI_OK;
}

int lcbi_gpu_set_early_helpers(lcbi_gpu_context* c, int enable)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx) return LCBI_INVALID_ARGUMENT;
    ctx->early_helpers = enable != 0;
    return LCBI_OK;
}

int lcbi_gpu_set_polar_tiles(lcbi_gpu_context* c, int enable)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx) return LCBI_INVALID_ARGUMENT;
    ctx->polar_tiles = enable != 0;
    return LCBI_OK;
}

int lcbi_gpu_set_workspace(lcbi_gpu_context* c, int32_t warps_per_sm, int32_t second_pass_blocks,
                           int64_t tile_capacity)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || second_pass_blocks < 0) return LCBI_INVALID_ARGUMENT;
    if (tile_capacity > 0 && (tile_capacity & (tile_capacity - 1)) != 0) return LCBI_INVALID_ARGUMENT;
    if (warps_per_sm > 0) ctx->warps_per_sm = warps_per_sm;  // the scratch is re-sized on the next call
    if (second_pass_blocks != ctx->retry_blocks) {
        ctx->retry_blocks = second_pass_blocks;
        ctx->big_ready = false;
    }
    if (tile_capacity > 0) ctx->tile_capacity = tile_capacity;
    return LCBI_OK;
}

int lcbi_gpu_stage_times(const lcbi_gpu_context* c, double* ms, int64_t* launches, int32_t n)
{
    const Context* ctx = reinterpret_cast<const Context*>(c);
    if (!ctx || !ms || n < 0) return LCBI_INVALID_ARGUMENT;
    for (int i = 0; i < n && i < Context::kStages; ++i) {
        ms[i] = ctx->stage_ms[i];
        if (launches) launches[i] = ctx->stage_launches[i];
    }
    return LCBI_OK;
}

void lcbi_gpu_destroy(lcbi_gpu_context* c)
{
    delete reinterpret_cast<Context*>(c);
}

const char* lcbi_gpu_last_error(const lcbi_gpu_context* c)
{
    return c ? reinterpret_cast<const Context*>(c)->error.c_str() : "null context";
}

int64_t lcbi_gpu_launch_count(const lcbi_gpu_context* c)
{
    return c ? reinterpret_cast<const Context*>(c)->launches : 0;
}

int lcbi_gpu_kernel_binary_version(int32_t* version)
{
    if (!version) return LCBI_INVALID_ARGUMENT;
    int v = 0;
    if (lcbi::kernel_binary_version(&v) != cudaSuccess) {
        cudaGetLastError();
        return LCBI_GPU_ERROR;
    }
    *version = v;
    return LCBI_OK;
}

int64_t lcbi_gpu_workspace_bytes(lcbi_gpu_context* c)
{
    if (!c) return -1;
    Context* ctx = reinterpret_cast<Context*>(c);
    int64_t total = 0;
    for (const lcbi::Buffer* b : ctx->all_buffers()) total += static_cast<int64_t>(b->bytes);
    return total;
}

int lcbi_gpu_binary_mag0(lcbi_gpu_context* c, int64_t n, const double* s, const double* q, const double* y1,
                         const double* y2, double* A, int32_t* image_count, int32_t* status, unsigned flags)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || n < 0) return LCBI_INVALID_ARGUMENT;
    if (n == 0) return LCBI_OK;
    if (!s || !q || !y1 || !y2 || !A) return LCBI_INVALID_ARGUMENT;
    ctx->error.clear();
    cudaSetDevice(ctx->device);
    const bool dev = (flags & LCBI_GPU_DEVICE_POINTERS) != 0;
    const size_t N = static_cast<size_t>(n);
    if (!dev && !ctx->timing && N >= 2 * kPsChunk) return ps_pipelined(ctx, N, s, q, y1, y2, A, image_count, status);
    const double *ds, *dq, *dy1, *dy2;
    double* dA;
    int *dn, *dst;
    if (!ctx->stage_in(ctx->in[0], s, N, dev, &ds) || !ctx->stage_in(ctx->in[1], q, N, dev, &dq) ||
        !ctx->stage_in(ctx->in[2], y1, N, dev, &dy1) || !ctx->stage_in(ctx->in[3], y2, N, dev, &dy2) ||
        !ctx->stage_out(ctx->out[0], A, N, dev, &dA) ||
        !ctx->stage_out(ctx->out[1], reinterpret_cast<int*>(image_count), N, dev, &dn) ||
        !ctx->stage_out(ctx->out[2], reinterpret_cast<int*>(status), N, dev, &dst))
        return LCBI_GPU_ERROR;
    cudaEvent_t t0;
    ctx->stage_begin(5, &t0);
    if (!ctx->check("ps_batch_kernel", lcbi::launch_ps_batch(ds, dq, dy1, dy2, dA, dn, dst, n, ctx->sm_count,
                                                             ctx->stream)))
        return LCBI_GPU_ERROR;
    ctx->stage_end(5, t0);
    ctx->launches += 1;
    if (!ctx->copy_back(A, dA, N, dev) || !ctx->copy_back(reinterpret_cast<int*>(image_count), dn, N, dev) ||
        !ctx->copy_back(reinterpret_cast<int*>(status), dst, N, dev) || !ctx->finish())
        return LCBI_GPU_ERROR;
    return LCBI_OK;
}

int lcbi_gpu_binary_images_mag(lcbi_gpu_context* c, int64_t n, const double* s, const double* q, const double* y1,
                               const double* y2, double* A, int32_t* image_count, unsigned flags)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || n < 0) return LCBI_INVALID_ARGUMENT;
    if (n == 0) return LCBI_OK;
    if (!s || !q || !y1 || !y2 || !A) return LCBI_INVALID_ARGUMENT;
    ctx->error.clear();
    cudaSetDevice(ctx->device);
    const bool dev = (flags & LCBI_GPU_DEVICE_POINTERS) != 0;
    const size_t N = static_cast<size_t>(n);
    const double *ds, *dq, *dy1, *dy2;
    double* dA;
    int* dn;
    if (!ctx->stage_in(ctx->in[0], s, N, dev, &ds) || !ctx->stage_in(ctx->in[1], q, N, dev, &dq) ||
        !ctx->stage_in(ctx->in[2], y1, N, dev, &dy1) || !ctx->stage_in(ctx->in[3], y2, N, dev, &dy2) ||
        !ctx->stage_out(ctx->out[0], A, N, dev, &dA) ||
        !ctx->stage_out(ctx->out[1], reinterpret_cast<int*>(image_count), N, dev, &dn))
        return LCBI_GPU_ERROR;
    if (!ctx->check("ps_images_kernel", lcbi::launch_ps_images(ds, dq, dy1, dy2, dA, dn, n, ctx->sm_count,
                                                               ctx->stream)))
        return LCBI_GPU_ERROR;
    ctx->launches += 1;
    if (!ctx->copy_back(A, dA, N, dev) || !ctx->copy_back(reinterpret_cast<int*>(image_count), dn, N, dev) ||
        !ctx->finish())
        return LCBI_GPU_ERROR;
    return LCBI_OK;
}

int lcbi_gpu_binary_image_candidates(lcbi_gpu_context* c, int64_t n, const double* s, const double* q,
                                     const double* y1, const double* y2, double* candidates, int32_t* n_physical,
                                     unsigned flags)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || n < 0) return LCBI_INVALID_ARGUMENT;
    if (n == 0) return LCBI_OK;
    if (!s || !q || !y1 || !y2 || !candidates || !n_physical) return LCBI_INVALID_ARGUMENT;
    ctx->error.clear();
    cudaSetDevice(ctx->device);
    const bool dev = (flags & LCBI_GPU_DEVICE_POINTERS) != 0;
    const size_t N = static_cast<size_t>(n);
    const double *ds, *dq, *dy1, *dy2;
    double* dcand;
    int* dn;
    if (!ctx->stage_in(ctx->in[0], s, N, dev, &ds) || !ctx->stage_in(ctx->in[1], q, N, dev, &dq) ||
        !ctx->stage_in(ctx->in[2], y1, N, dev, &dy1) || !ctx->stage_in(ctx->in[3], y2, N, dev, &dy2) ||
        !ctx->stage_out(ctx->out[0], candidates, 20 * N, dev, &dcand) ||
        !ctx->stage_out(ctx->out[1], reinterpret_cast<int*>(n_physical), N, dev, &dn))
        return LCBI_GPU_ERROR;
    if (!ctx->check("ps_candidates_kernel",
                    lcbi::launch_ps_candidates(ds, dq, dy1, dy2, reinterpret_cast<double4*>(dcand), dn, n,
                                               ctx->sm_count, ctx->stream)))
        return LCBI_GPU_ERROR;
    ctx->launches += 1;
    if (!ctx->copy_back(candidates, dcand, 20 * N, dev) ||
        !ctx->copy_back(reinterpret_cast<int*>(n_physical), dn, N, dev) || !ctx->finish())
        return LCBI_GPU_ERROR;
    return LCBI_OK;
}

int lcbi_gpu_binary_mag0_derivatives(lcbi_gpu_context* c, int64_t n, const double* s, const double* q,
                                     const double* y1, const double* y2, double* A, int32_t* image_count,
                                     double* indicator, unsigned flags)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || n < 0) return LCBI_INVALID_ARGUMENT;
    if (n == 0) return LCBI_OK;
    if (!s || !q || !y1 || !y2 || !A || !image_count || !indicator) return LCBI_INVALID_ARGUMENT;
    ctx->error.clear();
    cudaSetDevice(ctx->device);
    const bool dev = (flags & LCBI_GPU_DEVICE_POINTERS) != 0;
    const size_t N = static_cast<size_t>(n);
    const double *ds, *dq, *dy1, *dy2;
    double *dA, *dind;
    int* dn;
    if (!ctx->stage_in(ctx->in[0], s, N, dev, &ds) || !ctx->stage_in(ctx->in[1], q, N, dev, &dq) ||
        !ctx->stage_in(ctx->in[2], y1, N, dev, &dy1) || !ctx->stage_in(ctx->in[3], y2, N, dev, &dy2) ||
        !ctx->stage_out(ctx->out[0], A, N, dev, &dA) ||
        !ctx->stage_out(ctx->out[1], reinterpret_cast<int*>(image_count), N, dev, &dn) ||
        !ctx->stage_out(ctx->out[2], indicator, N, dev, &dind))
        return LCBI_GPU_ERROR;
    if (!ctx->check("ps_deriv_kernel",
                    lcbi::launch_ps_deriv(ds, dq, dy1, dy2, dA, dn, dind, n, ctx->sm_count, ctx->stream)))
        return LCBI_GPU_ERROR;
    ctx->launches += 1;
    if (!ctx->copy_back(A, dA, N, dev) || !ctx->copy_back(reinterpret_cast<int*>(image_count), dn, N, dev) ||
        !ctx->copy_back(indicator, dind, N, dev) || !ctx->finish())
        return LCBI_GPU_ERROR;
    return LCBI_OK;
}

} // extern "C"
