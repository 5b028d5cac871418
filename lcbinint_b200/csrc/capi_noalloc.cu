// lcbi_gpu_binary_mag_noalloc: the finite-source pipeline of lcbi_gpu_binary_mag
// for one lens model and one settings struct, with every working buffer carved
// out of one fixed, file-scope device array instead of context workspaces.
//
// Who needs it: a caller that cannot let the library allocate in the middle of
// its run.  Examples are a sampler that has already handed all free device
// memory to its own pool (a cudaMalloc there fails, or forces the pool to give
// memory back), and a caller whose other streams are busy, since cudaFree --
// which the context workspaces call when a batch outgrows them -- waits for the
// whole device and stalls their work.  This entry point makes no device
// allocation, no cudaFree, and calls no allocating library: after the one-time
// setup per device it only issues memsets, copies of small host structs and
// kernel launches on the context's stream.
//
// Limits of the fixed area (LCBI_NOALLOC_* in the public header): caustic_bins
// at most 2048 (larger requests are rejected); adaptive local refinement
// (adaptive_source_bins with a tolerance) is refused with LCBI_UNSUPPORTED; 2048 image seeds per point
// (status 17 beyond, as in lcbi_gpu_binary_mag); 8192 rows per Cartesian seed
// scan and 16384 polar segments in flight in the first pass (one warp per
// point), with a second pass on four blocks (one point per block) at 65536
// rows / 131072 segments for the points that overflow (status 18 / 19 beyond
// that, where lcbi_gpu_binary_mag goes on further).  Points are processed 256 at a time, so n itself is unbounded.
//
// What must start at zero: the work-list counters (reset with a memset at the
// start of every 256-point chunk).  The row and segment tables of the scans must
// start with no slot carrying the current scan's tag; every pass resets them to
// all-ones bytes, a tag no scan produces.  Nothing else is read before it is
// written, so the area needs no initialisation by the caller.
//
// Calls on one device share the one area: two calls that overlap in time (from
// two host threads, or on two streams with no ordering between them) race on it
// and corrupt each other's results.  Serialise them.
#include "../../include/lcbinint_b200.h"
#include "lcbi_context.h"
#include "lcbi_fs_kernels.h"

#include <cuda.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <mutex>

namespace lcbi {
namespace {

constexpr int kMaxBins = LCBI_NOALLOC_MAX_CAUSTIC_BINS;
constexpr int kPoints = 256;          // points per pipeline pass
constexpr int kSeedCap = 2048;        // image seeds per point
constexpr int kCandCap = 4 * kMaxBins;
constexpr int kWarps = 32;            // persistent warps of the first pass
constexpr int kRows = 8192;           // Cartesian rows per seed scan, first pass
constexpr int kQueue = 1 << 14;       // polar segments in flight, first pass
constexpr int kHash = 1 << 15;        // polar visited-segment slots, first pass
constexpr int kRetryBlocks = 4;       // second pass: blocks of kBigWarps warps
constexpr int kRowsRetry = 1 << 16;
constexpr int kQueueRetry = 1 << 17;
constexpr int kHashRetry = 1 << 18;
// The first-pass scan kernels run 4 warps per block and give every launched
// warp its own share of the scratch, so the warp count must be a multiple of 4.
static_assert(kWarps % 4 == 0, "whole blocks only");
constexpr int kTrig = 1400 + 400 + 64 + 16;
constexpr double kHostPi = 3.14159265358979323846;
constexpr int kMaxDevices = 64;

constexpr size_t up256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t max3(size_t a, size_t b, size_t c) { return a > b ? (a > c ? a : c) : (b > c ? b : c); }

// Byte offsets of the pieces of the area.
constexpr size_t kOffSettings = 0;
constexpr size_t kOffModel = kOffSettings + up256(sizeof(FsSettingsDev));
constexpr size_t kOffRawOffset = kOffModel + up256(sizeof(CausticModel));
constexpr size_t kOffLdCoeff = kOffRawOffset + 256;
constexpr size_t kOffCounters = kOffLdCoeff + 256;
constexpr size_t kOffPhases = kOffCounters + 256;
constexpr size_t kOffRaw = kOffPhases + up256(sizeof(double2) * kMaxBins);
constexpr size_t kOffBranches = kOffRaw + up256(sizeof(P2) * 4 * kMaxBins);
constexpr size_t kOffLd = kOffBranches + up256(sizeof(P2) * 4 * kMaxBins);
constexpr size_t kOffItems = kOffLd + up256(sizeof(double) * (kLdTable + 1));
constexpr size_t kOffRays = kOffItems + up256(sizeof(FsItem) * kPoints);
constexpr size_t kOffLists = kOffRays + up256(sizeof(unsigned long long) * kPoints);
constexpr size_t kOffSeeds = kOffLists + up256(sizeof(int) * 4 * kPoints);
constexpr size_t kOffScratch = kOffSeeds + up256(sizeof(P2) * kPoints * kSeedCap);
constexpr size_t kCandPerWarp = (size_t)2 * kCandCap * (sizeof(long long) + sizeof(P2));
constexpr size_t kScratchBytes = 36u << 20;  // checked against the scan sizes at setup

} // namespace
} // namespace lcbi

// The fixed working area (one instance per device, reserved when the library's
// module is loaded on that device) and the constant angle tables.
static __device__ __align__(256) unsigned char g_noalloc_area[LCBI_NOALLOC_AREA_BYTES];
static __device__ __align__(256) double2 g_noalloc_trig[lcbi::kTrig];

static_assert(lcbi::kOffScratch + lcbi::kScratchBytes <= LCBI_NOALLOC_AREA_BYTES, "fixed area layout");

namespace lcbi {
namespace {

struct DeviceArea {
    unsigned char* area;
    double2* trig;
    unsigned long long context_id;  // the CUDA context the tables were uploaded in
    bool ready;
};
DeviceArea g_devices[kMaxDevices];
std::mutex g_setup_mutex;

// Per-warp scan sizes must fit the scratch part of the area.
bool scratch_fits(size_t* main_cart, size_t* main_polar, size_t* retry_cart, size_t* retry_polar)
{
    *main_cart = up256(cartesian_scratch_bytes(kRows, kSeedCap));
    *main_polar = up256(polar_scratch_bytes(kQueue, kHash));
    *retry_cart = up256(cartesian_scratch_bytes(kRowsRetry, kSeedCap));
    *retry_polar = up256(polar_scratch_bytes(kQueueRetry, kHashRetry));
    const size_t first = kWarps * max3(*main_cart, *main_polar, kCandPerWarp);
    const size_t second = kRetryBlocks * (*retry_cart > *retry_polar ? *retry_cart : *retry_polar);
    return first <= kScratchBytes && second <= kScratchBytes;
}

// The unique id of the current CUDA context (cuCtxGetId, reached through the
// runtime's driver entry points so that nothing links libcuda); 0 if unknown.
// A cudaDeviceReset ends the device's primary context, and the next one gets
// a new id.
unsigned long long current_context_id()
{
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, nullptr) == cudaSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, nullptr) == cudaSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    });
    if (!get_current || !get_id) return 0;
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current(&c) != CUDA_SUCCESS || c == nullptr || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Set-up for the context's device (the device must be current), checked on
// every call: looks up the device addresses of the fixed arrays (cheap once
// the library's device code is loaded) and uploads the angle tables,
// evaluated with the host C library exactly as the workspace path evaluates
// them, whenever the device has not been set up in its current CUDA context:
// on the device's first call, and again after a cudaDeviceReset, which loads
// the device code afresh (the arrays may sit elsewhere and have lost their
// contents).  The upload is a synchronous cudaMemcpy.
bool setup(Context* ctx)
{
    if (ctx->device < 0 || ctx->device >= kMaxDevices) return ctx->fail("device index beyond the fixed-area table");
    void* area = nullptr;
    void* trig = nullptr;
    if (!ctx->check("cudaGetSymbolAddress(fixed area)", cudaGetSymbolAddress(&area, g_noalloc_area)) ||
        !ctx->check("cudaGetSymbolAddress(angle tables)", cudaGetSymbolAddress(&trig, g_noalloc_trig)))
        return false;
    const unsigned long long cid = current_context_id();
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceArea& d = g_devices[ctx->device];
    if (d.ready && d.area == area && d.trig == trig && d.context_id == cid) return true;
    size_t a, b, c, e;
    if (!scratch_fits(&a, &b, &c, &e)) return ctx->fail("fixed-area scan sizes exceed the scratch part");
    static double2 host[kTrig];
    int k = 0;
    const double phase_step = 2.0 * kHostPi / static_cast<double>(1400);
    for (int i = 0; i < 1400; ++i) {
        const std::complex<double> p = std::polar(1.0, phase_step * static_cast<double>(i));
        host[k++] = make_double2(p.real(), p.imag());
    }
    for (int i = 0; i < 400; ++i) {
        const double phi = 2.0 * kHostPi * static_cast<double>(i) / static_cast<double>(400);
        host[k++] = make_double2(std::cos(phi), std::sin(phi));
    }
    for (int i = 0; i < 64; ++i) {
        const double phi = 2.0 * kHostPi * static_cast<double>(i) / static_cast<double>(64);
        host[k++] = make_double2(std::cos(phi), std::sin(phi));
    }
    for (int i = 0; i < 16; ++i) {
        const double th = 2.0 * kHostPi * static_cast<double>(i) / static_cast<double>(16);
        host[k++] = make_double2(std::cos(th), std::sin(th));
    }
    d.ready = false;
    if (!ctx->check("angle tables upload", cudaMemcpy(trig, host, sizeof(host), cudaMemcpyHostToDevice))) return false;
    d.area = static_cast<unsigned char*>(area);
    d.trig = static_cast<double2*>(trig);
    d.context_id = cid;
    d.ready = true;
    return true;
}

__global__ void noalloc_items_kernel(const double* y1, const double* y2, const double* rho, double s, double q,
                                     FsItem* items, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    FsItem it;
    it.s = s;
    it.q = q;
    it.x = y1[i];
    it.y = y2[i];
    it.rho = rho[i];
    it.a_ps = 0.0;
    it.settings = 0;
    it.model = 0;
    it.flags = kItemPsExact | kItemPsOnDevice;
    it.pad = 0;
    items[i] = it;
}

FsSettingsDev settings_of(const lcbi_fs_settings& s)
{
    FsSettingsDev d;
    d.source_bins = s.source_bins;
    d.caustic_bins = s.caustic_bins;
    d.grid_ratio = s.grid_ratio;
    d.polar_source_bins = s.polar_source_bins;
    d.polar_grid_ratio = s.polar_grid_ratio;
    d.finite_mode = s.finite_mode;
    d.kinji_threshold = s.kinji_threshold;
    d.hex_threshold = s.hex_threshold;
    d.adaptive_hex_threshold = s.adaptive_hex_threshold;
    d.ld_c = s.limb_darkening_c;
    d.ld_d = s.limb_darkening_d;
    d.adaptive_source_bins = s.adaptive_source_bins;
    d.max_source_bins = s.max_source_bins;
    d.tol = s.finite_source_tol;
    d.reltol = s.finite_source_reltol;
    d.ld_table = 0;
    d.pad = 0;
    return d;
}

template <typename T>
T* at(unsigned char* area, size_t off)
{
    return reinterpret_cast<T*>(area + off);
}

} // namespace
} // namespace lcbi

using namespace lcbi;

extern "C" int lcbi_gpu_binary_mag_noalloc(lcbi_gpu_context* c, const lcbi_fs_settings* settings, double s, double q,
                                           int64_t n, const double* y1, const double* y2, const double* rho,
                                           lcbi_fs_result* results)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || !settings || n < 0) return LCBI_INVALID_ARGUMENT;
    ctx->error.clear();
    if (settings->caustic_bins > kMaxBins) {
        char msg[160];
        std::snprintf(msg, sizeof(msg), "caustic_bins %d exceeds the fixed working area's maximum of %d",
                      settings->caustic_bins, kMaxBins);
        ctx->fail(msg);
        return LCBI_INVALID_ARGUMENT;
    }
    if (settings->adaptive_source_bins != 0 &&
        (settings->finite_source_tol > 0.0 || settings->finite_source_reltol > 0.0)) {
        ctx->fail("adaptive source bins (local refinement) is not implemented");
        return LCBI_UNSUPPORTED;
    }
    if (settings->finite_mode == 3) {
        ctx->fail("finite_mode 3 (experimental spine integrator) is not implemented");
        return LCBI_UNSUPPORTED;
    }
    if (!ctx->check("cudaSetDevice", cudaSetDevice(ctx->device)) || !setup(ctx)) return LCBI_GPU_ERROR;
    if (n == 0) return LCBI_OK;
    if (!y1 || !y2 || !rho || !results) return LCBI_INVALID_ARGUMENT;
    unsigned char* area;
    const double2* trig;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        area = g_devices[ctx->device].area;
        trig = g_devices[ctx->device].trig;
    }
    cudaStream_t st = ctx->stream;

    // Per-call constants: settings, the lens model with its phase table, the
    // limb-darkening table, the sampled caustic.
    const int bins = settings->caustic_bins > 32 ? settings->caustic_bins : 32;
    const FsSettingsDev sd = settings_of(*settings);
    CausticModel md{};
    md.s = s;
    md.q = q;
    md.bins = bins;
    md.phase_offset = 0;
    md.branch_offset = 0;
    const long long raw_offset = 0;
    const double2 ld_coeff = make_double2(settings->limb_darkening_c, settings->limb_darkening_d);
    double2 phases[kMaxBins];
    for (int i = 0; i < bins; ++i) {
        const double a = 2.0 * kHostPi * static_cast<double>(i) / static_cast<double>(bins);
        const std::complex<double> p = std::polar(1.0, a);
        phases[i] = make_double2(p.real(), p.imag());
    }
    FsSettingsDev* d_settings = at<FsSettingsDev>(area, kOffSettings);
    CausticModel* d_model = at<CausticModel>(area, kOffModel);
    long long* d_raw_offset = at<long long>(area, kOffRawOffset);
    double2* d_ld_coeff = at<double2>(area, kOffLdCoeff);
    double2* d_phases = at<double2>(area, kOffPhases);
    P2* d_raw = at<P2>(area, kOffRaw);
    P2* d_branches = at<P2>(area, kOffBranches);
    double* d_ld = at<double>(area, kOffLd);
    if (!ctx->check("settings H2D", cudaMemcpyAsync(d_settings, &sd, sizeof(sd), cudaMemcpyHostToDevice, st)) ||
        !ctx->check("model H2D", cudaMemcpyAsync(d_model, &md, sizeof(md), cudaMemcpyHostToDevice, st)) ||
        !ctx->check("offset H2D", cudaMemcpyAsync(d_raw_offset, &raw_offset, sizeof(raw_offset),
                                                  cudaMemcpyHostToDevice, st)) ||
        !ctx->check("ld coeff H2D", cudaMemcpyAsync(d_ld_coeff, &ld_coeff, sizeof(ld_coeff), cudaMemcpyHostToDevice,
                                                    st)) ||
        !ctx->check("phases H2D", cudaMemcpyAsync(d_phases, phases, sizeof(double2) * bins, cudaMemcpyHostToDevice,
                                                  st)))
        return LCBI_GPU_ERROR;
    if (!ctx->check("ld tables", launch_ld_tables(d_ld_coeff, 1, d_ld, st)) ||
        !ctx->check("caustics", launch_caustics(d_model, 1, bins, d_phases, d_raw_offset, d_raw, d_branches, st)))
        return LCBI_GPU_ERROR;
    ctx->launches += 3;

    size_t main_cart, main_polar, retry_cart, retry_polar;
    scratch_fits(&main_cart, &main_polar, &retry_cart, &retry_polar);
    char* scratch = reinterpret_cast<char*>(area + kOffScratch);
    int* counters = at<int>(area, kOffCounters);
    int* lists = at<int>(area, kOffLists);
    FsItem* items = at<FsItem>(area, kOffItems);
    for (long long c0 = 0; c0 < n; c0 += kPoints) {
        const int cn = static_cast<int>((n - c0) < kPoints ? (n - c0) : kPoints);
        if (!ctx->check("items", cudaMemsetAsync(counters, 0, 64 * sizeof(int), st)))
            return LCBI_GPU_ERROR;
        noalloc_items_kernel<<<(cn + 127) / 128, 128, 0, st>>>(y1 + c0, y2 + c0, rho + c0, s, q, items, cn);
        if (!ctx->check("items", cudaGetLastError())) return LCBI_GPU_ERROR;
        FsWork w{};
        w.items = items;
        w.settings = d_settings;
        w.models = d_model;
        w.raw_offset = d_raw_offset;
        w.raw = d_raw;
        w.branches = d_branches;
        w.ld_tables = d_ld;
        w.trig = TrigTables{trig, trig + 1400, trig + 1800, trig + 1864};
        w.out = reinterpret_cast<FsOut*>(results + c0);
        w.n_items = cn;
        w.ir_count = counters;
        w.next_item = counters + 8;
        w.ir_cart = lists;
        w.ir_polar = lists + kPoints;
        w.retry_cart = lists + 2 * kPoints;
        w.retry_polar = lists + 3 * kPoints;
        w.seeds = at<P2>(area, kOffSeeds);
        w.seed_cap = kSeedCap;
        w.cand_cap = kCandCap;
        w.rays = at<unsigned long long>(area, kOffRays);
        w.cycles = nullptr;
        w.retry_pass = 0;
        w.scratch = scratch;
        w.scratch_per_warp = static_cast<long long>(main_cart);
        w.scratch_polar = scratch;
        w.scratch_polar_per_warp = static_cast<long long>(main_polar);
        w.row_cap = kRows;
        w.queue_cap = kQueue;
        w.hash_cap = kHash;
        const int warps = kWarps < cn ? kWarps : cn;
        // Seed-probe candidates: all warps' keys, then all warps' probes.
        long long* cand_keys = reinterpret_cast<long long*>(scratch);
        P2* cand_probes = reinterpret_cast<P2*>(scratch + (size_t)kWarps * 2 * kCandCap * sizeof(long long));
        if (!ctx->check("decide", launch_decide(w, ctx->sm_count, st)) ||
            !ctx->check("seeds", launch_seeds(w, ctx->sm_count, st, cand_keys, cand_probes, warps)))
            return LCBI_GPU_ERROR;
        // Cartesian and polar scans, then the second pass for the points whose
        // first-pass scan outgrew its share; the same bytes serve every scan, so
        // each starts from freshly reset tables.
        const size_t first = kWarps * (main_cart > main_polar ? main_cart : main_polar);
        const size_t second = kRetryBlocks * (retry_cart > retry_polar ? retry_cart : retry_polar);
        if (!ctx->check("table reset", cudaMemsetAsync(scratch, 0xff, first, st)) ||
            !ctx->check("cartesian", launch_cartesian(w, warps, st, 1)) ||
            !ctx->check("table reset", cudaMemsetAsync(scratch, 0xff, first, st)) ||
            !ctx->check("polar", launch_polar(w, warps, st, 1)))
            return LCBI_GPU_ERROR;
        FsWork r = w;
        r.retry_pass = 1;
        r.scratch_per_warp = static_cast<long long>(retry_cart);
        r.scratch_polar_per_warp = static_cast<long long>(retry_polar);
        r.row_cap = kRowsRetry;
        r.queue_cap = kQueueRetry;
        r.hash_cap = kHashRetry;
        if (!ctx->check("table reset", cudaMemsetAsync(scratch, 0xff, second, st)) ||
            !ctx->check("cartesian retry", launch_cartesian(r, kRetryBlocks, st, 1)) ||
            !ctx->check("table reset", cudaMemsetAsync(scratch, 0xff, second, st)) ||
            !ctx->check("polar retry", launch_polar(r, kRetryBlocks, st, 1)))
            return LCBI_GPU_ERROR;
        ctx->launches += 7;
    }
    return ctx->finish() ? LCBI_OK : LCBI_GPU_ERROR;
}
