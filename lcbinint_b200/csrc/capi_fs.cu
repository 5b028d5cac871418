// C-ABI host runtime of the finite-source pipeline:
//   caustic models -> decision kernel -> seeding -> Cartesian / polar inverse ray.
// The host only plans (de-duplicates lens models, builds constant angle tables
// with the host C library) and launches; all physics runs in the kernels.
#include <algorithm>
#include "../../include/lcbinint_b200.h"
#include "lcbi_context.h"
#include "lcbi_fs_kernels.h"
#include "lcbi_internal.h"
#include "lcbi_kernels.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <tuple>
#include <unordered_map>
#include <vector>

using lcbi::Context;

namespace lcbi {
namespace {

static_assert(sizeof(FsOut) == sizeof(lcbi_fs_result), "result layout");
static_assert(sizeof(FsItem) == sizeof(lcbi_fs_point), "point layout");

constexpr int kChunk = 16384;
constexpr double kHostPi = 3.14159265358979323846;

// Constant angle tables, evaluated exactly as the reference evaluates them.
bool ensure_trig(Context* ctx)
{
    if (ctx->trig_ready) return true;
    std::vector<double2> t;
    t.reserve(1400 + 400 + 64 + 16);
    const double phase_step = 2.0 * kHostPi / static_cast<double>(1400);
    for (int k = 0; k < 1400; ++k) {
        const std::complex<double> p = std::polar(1.0, phase_step * static_cast<double>(k));
        t.push_back(make_double2(p.real(), p.imag()));
    }
    for (int i = 0; i < 400; ++i) {
        const double phi = 2.0 * kHostPi * static_cast<double>(i) / static_cast<double>(400);
        t.push_back(make_double2(std::cos(phi), std::sin(phi)));
    }
    for (int i = 0; i < 64; ++i) {
        const double phi = 2.0 * kHostPi * static_cast<double>(i) / static_cast<double>(64);
        t.push_back(make_double2(std::cos(phi), std::sin(phi)));
    }
    for (int i = 0; i < 16; ++i) {
        const double th = 2.0 * kHostPi * static_cast<double>(i) / static_cast<double>(16);
        t.push_back(make_double2(std::cos(th), std::sin(th)));
    }
    if (!ctx->ensure(ctx->fs_trig, t.size() * sizeof(double2))) return false;
    if (!ctx->check("trig upload", cudaMemcpy(ctx->fs_trig.ptr, t.data(), t.size() * sizeof(double2),
                                              cudaMemcpyHostToDevice)))
        return false;
    ctx->trig_ready = true;
    return true;
}

TrigTables trig_of(Context* ctx)
{
    const double2* b = static_cast<const double2*>(ctx->fs_trig.ptr);
    return TrigTables{b, b + 1400, b + 1800, b + 1864};
}

// Persistent-warp scratch, sized once per context and initialised to 0xff
// (no generation tag matches it).
bool ensure_scratch(Context* ctx)
{
    const int warps = ctx->sm_count * ctx->warps_per_sm;
    if (ctx->fs_warps == warps) return true;
    const size_t cart = (cartesian_scratch_bytes(ctx->row_cap, ctx->seed_cap) + 255) & ~size_t(255);
    const size_t pol = (polar_scratch_bytes(ctx->queue_cap, ctx->hash_cap) + 255) & ~size_t(255);
    if (!ctx->ensure(ctx->fs_scratch, cart * warps) || !ctx->ensure(ctx->fs_scratch_polar, pol * warps) ||
        !ctx->ensure(ctx->fs_cand_keys, seed_candidate_bytes_per_warp(ctx->cand_cap) * warps))
        return false;
    if (!ctx->check("scratch init", cudaMemsetAsync(ctx->fs_scratch.ptr, 0xff, cart * warps, ctx->stream)) ||
        !ctx->check("scratch init", cudaMemsetAsync(ctx->fs_scratch_polar.ptr, 0xff, pol * warps, ctx->stream)))
        return false;
    ctx->fs_warps = warps;
    // The scan tags restart with the epoch, so the second-pass scratch, which
    // still holds tags of the epochs before, is cleared as well (by
    // ensure_big_scratch, which every caller runs next).  A tag left over
    // from an earlier scan would otherwise pass for one of the current scan:
    // rows of another point would join the overlap chains.
    ctx->big_ready = false;
    ctx->epoch = 0;
    return true;
}

size_t cart_bytes_big(const Context* c) { return (cartesian_scratch_bytes(c->row_cap_big, c->seed_cap) + 255) & ~size_t(255); }
size_t split_bytes(const Context* c) { return (cartesian_scratch_bytes(kSplitRowCap, c->seed_cap) + 255) & ~size_t(255); }
size_t polar_bytes_big(const Context* c) { return (polar_scratch_bytes(c->queue_cap_big, c->hash_cap_big) + 255) & ~size_t(255); }

int retry_blocks(const Context* c) { return c->retry_blocks > 0 ? c->retry_blocks : c->sm_count; }

// The early pass's blocks and unit row areas: kEarlyBlocks and kSplitSlots
// (units take areas in list order, largest points first, until the pool is
// used up; the points after that run their seeds on their finishing block.
// On the 4,096-point batch, pools of 256, 384, 512, 768, 1,536 and 2,560
// areas measured 186, 188, 192, 190, 197 and 200 ms per step: splitting
// more points adds merges and repeated first rows and takes nothing off a
// step that the whole GPU's throughput bounds),
// or, when the caller has set a number of second-pass blocks, as many early
// blocks as second-pass blocks (at least 2) and 32 unit areas per early block.
int early_blocks(const Context* c)
{
    return c->retry_blocks > 0 ? std::min(kEarlyBlocks, std::max(2, c->retry_blocks)) : kEarlyBlocks;
}
int split_slots(const Context* c) { return std::min(kSplitSlots, 32 * early_blocks(c)); }

bool ensure_big_scratch(Context* ctx)
{
    if (ctx->big_ready) return true;
    // Cartesian: the second pass's blocks, then the early pass's blocks.
    const size_t cb = cart_bytes_big(ctx) * (retry_blocks(ctx) + early_blocks(ctx));
    const size_t pb = polar_bytes_big(ctx) * retry_blocks(ctx);
    // The units of the split early points: one small row scratch each.
    const size_t sb = split_bytes(ctx) * split_slots(ctx);
    if (!ctx->ensure(ctx->fs_scratch_big, cb) || !ctx->ensure(ctx->fs_scratch_polar_big, pb) ||
        !ctx->ensure(ctx->fs_split, sb) || !ctx->ensure(ctx->fs_split_info, kSplitUnits * sizeof(SplitInfo)) ||
        !ctx->ensure(ctx->fs_seed_info, (size_t)kEarlyMax * kSplitSeeds * sizeof(SeedInfo)))
        return false;
    if (!ctx->check("scratch init", cudaMemsetAsync(ctx->fs_scratch_big.ptr, 0xff, cb, ctx->stream)) ||
        !ctx->check("scratch init", cudaMemsetAsync(ctx->fs_scratch_polar_big.ptr, 0xff, pb, ctx->stream)) ||
        !ctx->check("scratch init", cudaMemsetAsync(ctx->fs_split.ptr, 0xff, sb, ctx->stream)))
        return false;
    ctx->big_ready = true;
    return true;
}

FsSettingsDev to_dev(const lcbi_fs_settings& s, int ld_index)
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
    d.ld_table = ld_index;
    d.pad = 0;
    return d;
}

struct Plan {
    std::vector<double2> ld_coeffs;  // distinct (c, d) pairs, one 20,001-entry table each
    std::vector<FsSettingsDev> settings;
    std::vector<CausticModel> models;
    std::vector<long long> raw_offset;
    std::vector<double2> phases;
    int max_bins = 0;
};

// Adds the caustic model (s, q, max(bins, 32)) and its phase table; returns its index.
struct ModelTable {
    Plan* plan;
    std::map<std::tuple<uint64_t, uint64_t, int>, int> index;
    std::map<int, int> phase_offset;
    long long raw_total = 0;

    int get(double s, double q, int caustic_bins)
    {
        const int bins = caustic_bins > 32 ? caustic_bins : 32;
        uint64_t bs, bq;
        std::memcpy(&bs, &s, 8);
        std::memcpy(&bq, &q, 8);
        const auto key = std::make_tuple(bs, bq, bins);
        auto it = index.find(key);
        if (it != index.end()) return it->second;
        const int id = add(s, q, bins);
        index[key] = id;
        return id;
    }

    // As get, but keyed only on the previous call's key: runs of points with
    // the same (s, q, bins) share one model and any other point gets its own.
    // Equal keys sample equal caustics, so a repeat costs only its sampling;
    // this keeps the table linear in time when every point has its own
    // separation (lens orbital motion).
    int get_sequential(double s, double q, int caustic_bins)
    {
        const int bins = caustic_bins > 32 ? caustic_bins : 32;
        uint64_t bs, bq;
        std::memcpy(&bs, &s, 8);
        std::memcpy(&bq, &q, 8);
        const auto key = std::make_tuple(bs, bq, bins);
        if (last_id >= 0 && key == last_key) return last_id;
        last_key = key;
        last_id = add(s, q, bins);
        return last_id;
    }

    std::tuple<uint64_t, uint64_t, int> last_key{};
    int last_id = -1;

    // Starts a new pass: later models get branch offsets from 0 in a fresh
    // table of samples, and no key is shared with earlier models.
    void restart_pass()
    {
        index.clear();
        last_id = -1;
        raw_total = 0;
    }

    int add(double s, double q, int bins)
    {
        auto po = phase_offset.find(bins);
        int off;
        if (po == phase_offset.end()) {
            off = static_cast<int>(plan->phases.size());
            for (int i = 0; i < bins; ++i) {
                const double a = 2.0 * kHostPi * static_cast<double>(i) / static_cast<double>(bins);
                const std::complex<double> p = std::polar(1.0, a);
                plan->phases.push_back(make_double2(p.real(), p.imag()));
            }
            phase_offset[bins] = off;
        } else {
            off = po->second;
        }
        CausticModel m{};
        m.s = s;
        m.q = q;
        m.bins = bins;
        m.phase_offset = off;
        m.branch_offset = raw_total;
        plan->raw_offset.push_back(raw_total);
        raw_total += 4ll * bins;
        if (bins > plan->max_bins) plan->max_bins = bins;
        const int id = static_cast<int>(plan->models.size());
        plan->models.push_back(m);
        return id;
    }
};

// Adds settings with their limb-darkening table slot, sharing tables between
// settings with the same (c, d).
void add_settings(Plan& plan, const lcbi_fs_settings* s, int n)
{
    for (int i = 0; i < n; ++i) {
        int slot = -1;
        for (size_t k = 0; k < plan.ld_coeffs.size(); ++k) {
            if (plan.ld_coeffs[k].x == s[i].limb_darkening_c && plan.ld_coeffs[k].y == s[i].limb_darkening_d) {
                slot = static_cast<int>(k);
                break;
            }
        }
        if (slot < 0) {
            slot = static_cast<int>(plan.ld_coeffs.size());
            plan.ld_coeffs.push_back(make_double2(s[i].limb_darkening_c, s[i].limb_darkening_d));
        }
        plan.settings.push_back(to_dev(s[i], slot));
    }
}

template <typename T>
bool upload(Context* ctx, Buffer& b, const std::vector<T>& v)
{
    if (!ctx->ensure(b, v.size() * sizeof(T) + 16)) return false;
    if (v.empty()) return true;
    return ctx->check("upload", cudaMemcpyAsync(b.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice,
                                                ctx->stream));
}

size_t cart_bytes_of(const Context* c) { return (cartesian_scratch_bytes(c->row_cap, c->seed_cap) + 255) & ~size_t(255); }
size_t polar_bytes_of(const Context* c) { return (polar_scratch_bytes(c->queue_cap, c->hash_cap) + 255) & ~size_t(255); }

// The parts of a work description every stage shares; callers set the points,
// results, caustic tables, work lists and counters.
FsWork common_work(Context* ctx)
{
    FsWork w{};
    w.settings = static_cast<const FsSettingsDev*>(ctx->fs_settings.ptr);
    w.ld_tables = static_cast<const double*>(ctx->fs_ld.ptr);
    w.trig = trig_of(ctx);
    w.seeds = static_cast<P2*>(ctx->fs_seeds.ptr);
    w.seed_cap = ctx->seed_cap;
    w.scratch = static_cast<char*>(ctx->fs_scratch.ptr);
    w.scratch_per_warp = static_cast<long long>(cart_bytes_of(ctx));
    w.scratch_polar = static_cast<char*>(ctx->fs_scratch_polar.ptr);
    w.scratch_polar_per_warp = static_cast<long long>(polar_bytes_of(ctx));
    w.row_cap = ctx->row_cap;
    w.queue_cap = ctx->queue_cap;
    w.hash_cap = ctx->hash_cap;
    w.retry_pass = 0;
    w.cand_cap = ctx->cand_cap;
    // Too few inverse-ray points to fill the GPU with one warp per point (a
    // single light curve, say, or a large batch that is mostly point
    // sources) run every point on a whole block.
    w.cell_budget = ctx->cell_budget;
    w.few_points = ctx->cell_budget_set ? 0 : 4 * ctx->sm_count;
    w.f32_rays = ctx->f32_rays ? 1 : 0;
    w.tape = ctx->tape_on ? static_cast<TapeCell*>(ctx->fs_tape.ptr) : nullptr;
    w.seed_block_after = ctx->seed_block_after;
    w.seed_scratch = static_cast<char*>(ctx->fs_seed_block.ptr);
    w.seed_scratch_per_block = static_cast<long long>(seed_candidate_bytes_per_warp(ctx->cand_cap));
    w.wait_limit = ctx->wait_limit;
    w.wait_timeouts = static_cast<int*>(ctx->fs_waits.ptr);
    return w;
}

void set_lists(FsWork& w, int* counters, int* lists, int* retry, long long cap_cart, long long cap_retry)
{
    w.ir_count = counters;
    w.next_item = counters + 8;
    w.ir_cart = lists;
    w.ir_polar = lists + cap_cart;
    w.retry_cart = retry;
    w.retry_polar = retry + cap_retry;
    w.retry_seeds = retry ? retry + 2 * cap_retry : nullptr;
    w.early_cart = counters + kEarlyOff;  // the layout: lcbi_fs_kernels.h
}

// The decision of every point of w (work lists and counters reset first).
bool stage_decide(Context* ctx, const FsWork& w)
{
    if (!ctx->check("counters", cudaMemsetAsync(w.ir_count, 0, kCounterInts * sizeof(int), ctx->stream))) return false;
    cudaEvent_t ev;
    ctx->stage_begin(1, &ev);
    if (!ctx->check("decide", launch_decide(w, ctx->sm_count, ctx->stream))) return false;
    ctx->stage_end(1, ev);
    return true;
}

// Scan tags of a new integration (the Cartesian and polar scratch areas
// carry them); at the wrap every area is cleared.
bool next_epoch(Context* ctx)
{
    if (++ctx->epoch < 0xfff0ull) return true;
    ctx->big_ready = false;
    if (!ensure_big_scratch(ctx)) return false;
    if (!ctx->check("scratch reset", cudaMemsetAsync(ctx->fs_scratch.ptr, 0xff, cart_bytes_of(ctx) * ctx->fs_warps,
                                                     ctx->stream)) ||
        !ctx->check("scratch reset", cudaMemsetAsync(ctx->fs_scratch_polar.ptr, 0xff,
                                                     polar_bytes_of(ctx) * ctx->fs_warps, ctx->stream)))
        return false;
    ctx->epoch = 1;
    return true;
}

// Cartesian points predicted to count more than half the first pass's cell
// budget (pi nbin^2 max(|A_ps|, 1) cells) would often spend the whole budget
// on their warp before starting again on a block after the first pass, and
// a point of a few million cells on one block sets the step.  They run on
// blocks from the start instead, largest first, at most kEarlyMax, each
// seed's two directional scans as units on blocks of their own (the early
// pass's blocks have their own scratch after the second pass's); the first
// pass skips them.  Adaptive refinement keeps one tape per group and does
// not use this path.
bool early_routing(const Context* ctx, const FsWork& w)
{
    return ctx->cell_budget > 0 && w.tape == nullptr && w.early_cart != nullptr;
}

FsWork early_work(Context* ctx, const FsWork& w)
{
    FsWork e = w;
    e.retry_pass = 1;
    e.early_pass = 1;
    e.scratch = static_cast<char*>(ctx->fs_scratch_big.ptr) +
                (long long)retry_blocks(ctx) * static_cast<long long>(cart_bytes_big(ctx));
    e.scratch_per_warp = static_cast<long long>(cart_bytes_big(ctx));
    e.row_cap = ctx->row_cap_big;
    e.split_scratch = static_cast<char*>(ctx->fs_split.ptr);
    e.split_bytes = static_cast<long long>(split_bytes(ctx));
    e.split_info = static_cast<SplitInfo*>(ctx->fs_split_info.ptr);
    e.split_slots = split_slots(ctx);
    e.seed_info = static_cast<SeedInfo*>(ctx->fs_seed_info.ptr);
    return e;
}

// Seeds of every inverse-ray point of w's work lists (at most max_points).
// With early routing, the routed points are seeded on the early stream and
// their block pass starts right after, beside the seeding of the others
// (stage_integrate joins it); with stage timing on, everything stays on the
// context's stream and stage_integrate runs the early pass first.
bool stage_seeds(Context* ctx, const FsWork& w, int max_points)
{
    const int warps = ctx->fs_warps < max_points ? ctx->fs_warps : max_points;
    if (warps <= 0) return true;
    // Early work a failed call left behind is finished before anything reuses its buffers.
    if (ctx->early_live && !ctx->check("join", cudaStreamWaitEvent(ctx->stream, ctx->early_join, 0))) return false;
    if (!next_epoch(ctx)) return false;
    ctx->early_live = false;
    ctx->marks_set = 0;
    ctx->mark(0, ctx->stream);
    ctx->early_serial = false;
    // Candidate keys and probes share one allocation: all warps' keys, then all probes.
    const size_t per = seed_candidate_bytes_per_warp(ctx->cand_cap);
    const size_t key_bytes = per * 8 / (8 + 16);
    cudaEvent_t ev;
    const bool early = early_routing(ctx, w);
    if (early) {
        if (!ctx->check("route", launch_route_early(w, 0.5 * static_cast<double>(ctx->cell_budget),
                                                    ctx->fs_route.ptr, max_points, ctx->sm_count, ctx->stream)))
            return false;
        FsWork es = w;
        es.seed_slots = w.early_cart;
        es.seed_count = w.ir_count + 5;
        es.seed_next = w.next_item + 7;
        es.seed_block_after = 0;
        char* eb = static_cast<char*>(ctx->fs_seed_early.ptr);
        long long* ek = reinterpret_cast<long long*>(eb);
        P2* ep = reinterpret_cast<P2*>(eb + key_bytes * kEarlyMax);
        if (!ctx->timing && ctx->early_stream != nullptr) {
            if (!ctx->check("fork", cudaEventRecord(ctx->early_fork, ctx->stream)) ||
                !ctx->check("fork", cudaStreamWaitEvent(ctx->early_stream, ctx->early_fork, 0)))
                return false;
            const bool ok =
                ctx->check("seeds early", launch_seeds(es, ctx->sm_count, ctx->early_stream, ek, ep, kEarlyMax)) &&
                ctx->check("early seeded", cudaEventRecord(ctx->early_seeded, ctx->early_stream)) &&
                ctx->check("cartesian early",
                           launch_cartesian(early_work(ctx, w), early_blocks(ctx), ctx->early_stream, ctx->epoch));
            // Recorded even after a failed launch: the context's stream must
            // never run ahead of work already queued beside it.
            ctx->mark(1, ctx->early_stream);
            if (!ctx->check("join", cudaEventRecord(ctx->early_join, ctx->early_stream))) return false;
            ctx->early_live = true;
            if (!ok) return false;
        } else {
            ctx->stage_begin(2, &ev);
            if (!ctx->check("seeds early", launch_seeds(es, ctx->sm_count, ctx->stream, ek, ep, kEarlyMax)))
                return false;
            ctx->stage_end(2, ev);
            ctx->early_serial = true;
        }
        ctx->launches += 4;
    }
    FsWork wm = w;
    wm.seed_skip_early = early ? 1 : 0;
    char* cb = static_cast<char*>(ctx->fs_cand_keys.ptr);
    ctx->stage_begin(2, &ev);
    if (!ctx->check("seeds", launch_seeds(wm, ctx->sm_count, ctx->stream, reinterpret_cast<long long*>(cb),
                                          reinterpret_cast<P2*>(cb + key_bytes * ctx->fs_warps), warps)))
        return false;
    // The points the one-warp pass handed over (their disks hold many
    // critical sources), one block each.
    if (wm.seed_block_after > 0 && wm.retry_seeds != nullptr && wm.seed_scratch != nullptr) {
        if (!ctx->check("seeds blocks", launch_seeds_blocks(wm, retry_blocks(ctx), ctx->stream))) return false;
        ctx->launches += 1;
    }
    ctx->stage_end(2, ev);
    return true;
}

// Inverse ray of every point of w's work lists: a first pass on warps (the
// polar points on tiles), then a second on blocks for the points that passed
// the cell budget or outgrew the first pass's scratch.  max_points bounds the
// lists' lengths.
bool stage_integrate(Context* ctx, const FsWork& w, int max_points)
{
    if (max_points <= 0) return true;
    const int warps = ctx->fs_warps < max_points ? ctx->fs_warps : max_points;
    const bool overlap = !ctx->timing && ctx->side_stream != nullptr;
    cudaEvent_t ev;
    if (ctx->early_serial) {
        // Stage timing on: the early block pass (stage_seeds) runs here, first.
        ctx->stage_begin(3, &ev);
        if (!ctx->check("cartesian early", launch_cartesian(early_work(ctx, w), early_blocks(ctx), ctx->stream, ctx->epoch)))
            return false;
        ctx->stage_end(3, ev);
    }
    if (!overlap) {
        ctx->stage_begin(3, &ev);
        if (!ctx->check("cartesian", launch_cartesian(w, warps, ctx->stream, ctx->epoch))) return false;
        ctx->stage_end(3, ev);
    }
    FsWork r = w;
    r.retry_pass = 1;
    // The second pass's groups (blocks) have the tapes after the first pass's warps.
    if (r.tape) r.tape += (long long)ctx->fs_warps * kTapeMax;
    r.scratch = static_cast<char*>(ctx->fs_scratch_big.ptr);
    r.scratch_per_warp = static_cast<long long>(cart_bytes_big(ctx));
    r.scratch_polar = static_cast<char*>(ctx->fs_scratch_polar_big.ptr);
    r.scratch_polar_per_warp = static_cast<long long>(polar_bytes_big(ctx));
    r.row_cap = ctx->row_cap_big;
    r.queue_cap = ctx->queue_cap_big;
    r.hash_cap = ctx->hash_cap_big;
    // Without stage timing the Cartesian passes (the first on warps, then the
    // second on blocks) run on the side stream, beside the polar passes, which
    // need nothing from them: each alone leaves much of the GPU idle while its
    // largest points finish.  The two touch disjoint work lists, counters
    // (Cartesian: ir_count[0], [2], next_item[1], [3]; polar: ir_count[1],
    // [3], next_item[2], [4]), outputs and scratch areas, so the results do
    // not depend on how they interleave.  With stage timing on, the stages run
    // one after another so that each stage's time is its own.
    if (overlap) {
        if (!ctx->check("fork", cudaEventRecord(ctx->fork_event, ctx->stream)) ||
            !ctx->check("fork", cudaStreamWaitEvent(ctx->side_stream, ctx->fork_event, 0)))
            return false;
        bool ok =
            ctx->check("cartesian", launch_cartesian(w, warps, ctx->side_stream, ctx->epoch)) &&
            ctx->check("cartesian retry", launch_cartesian(r, retry_blocks(ctx), ctx->side_stream, ctx->epoch));
        // Then the side stream's blocks join the early pass: the early pass's
        // units and points are claimed from one counter, so blocks launched
        // later take whatever is left, and the SMs the first and second passes
        // leave idle scan early units instead of waiting for the early
        // stream's blocks.  They use the second pass's scratch areas, free
        // once it has finished on this stream, with row-key generations above
        // the second pass's.  Which block runs a unit does not change its
        // result.
        if (ok && ctx->early_live && ctx->early_helpers) {
            FsWork h = early_work(ctx, w);
            h.scratch = static_cast<char*>(ctx->fs_scratch_big.ptr);
            h.gen_base = 0x40000000u;
            ok = ctx->check("early seeded", cudaStreamWaitEvent(ctx->side_stream, ctx->early_seeded, 0)) &&
                 ctx->check("cartesian early", launch_cartesian(h, retry_blocks(ctx), ctx->side_stream, ctx->epoch));
            ctx->launches += 1;
        }
        // The join is recorded even after a failed launch, so that the
        // context's stream never runs ahead of work already queued beside it.
        ctx->mark(2, ctx->side_stream);
        if (!ctx->check("join", cudaEventRecord(ctx->join_event, ctx->side_stream)) || !ok) return false;
    }
    ctx->stage_begin(4, &ev);
    bool polar_ok;
    if (ctx->polar_tiles) {
        polar_ok = ctx->check("polar", launch_polar_tiles(w, ctx->fs_tiles.ptr, ctx->tile_capacity, max_points,
                                                          ctx->tile_blocks, ctx->stream));
    } else {
        polar_ok = ctx->check("polar", launch_polar(w, warps, ctx->stream, ctx->epoch));
    }
    ctx->stage_end(4, ev);
    if (polar_ok && !overlap) {
        ctx->stage_begin(3, &ev);
        polar_ok = ctx->check("cartesian retry", launch_cartesian(r, retry_blocks(ctx), ctx->stream, ctx->epoch));
        ctx->stage_end(3, ev);
    }
    if (polar_ok) {
        ctx->stage_begin(4, &ev);
        polar_ok = ctx->check("polar retry", launch_polar(r, retry_blocks(ctx), ctx->stream, ctx->epoch));
        ctx->stage_end(4, ev);
    }
    ctx->mark(3, ctx->stream);
    if (overlap && !ctx->check("join", cudaStreamWaitEvent(ctx->stream, ctx->join_event, 0))) return false;
    if (ctx->early_live && !ctx->check("join", cudaStreamWaitEvent(ctx->stream, ctx->early_join, 0))) return false;
    ctx->early_live = false;
    if (!polar_ok) return false;
    ctx->launches += 8;
    return true;
}

// Everything before the caustic sampling: constant tables, the settings and
// limb-darkening tables, and the per-context scratch.
bool prepare_tables(Context* ctx, const Plan& plan)
{
    // Candidate lists of the caustic-branch seed probes hold one entry per sampled point.
    if (4 * plan.max_bins > ctx->cand_cap) {
        ctx->cand_cap = 4 * plan.max_bins;
        ctx->fs_warps = 0;  // re-size the per-warp areas
    }
    if (!ensure_trig(ctx) || !ensure_scratch(ctx) || !ensure_big_scratch(ctx) ||
        !ctx->ensure(ctx->fs_seed_block, seed_candidate_bytes_per_warp(ctx->cand_cap) * retry_blocks(ctx)) ||
        !ctx->ensure(ctx->fs_route, route_bytes()) ||
        !ctx->ensure(ctx->fs_seed_early, seed_candidate_bytes_per_warp(ctx->cand_cap) * kEarlyMax))
        return false;
    const int nld = static_cast<int>(plan.ld_coeffs.size());
    if (!upload(ctx, ctx->fs_settings, plan.settings) || !upload(ctx, ctx->fs_models, plan.models) ||
        !upload(ctx, ctx->fs_raw_offset, plan.raw_offset) || !upload(ctx, ctx->fs_phases, plan.phases) ||
        !upload(ctx, ctx->fs_ld_coeffs, plan.ld_coeffs) ||
        !ctx->ensure(ctx->fs_ld, (size_t)(nld + 1) * (kLdTable + 1) * sizeof(double)) ||
        !ctx->ensure(ctx->fs_counters, kCounterInts * sizeof(int)))
        return false;
    if (ctx->tile_blocks == 0) ctx->tile_blocks = polar_tile_blocks_per_sm() * ctx->sm_count;
    // Adaptive local refinement needs a tape per scratch group.
    ctx->tape_on = false;
    for (const auto& st : plan.settings)
        if (st.adaptive_source_bins != 0 && (st.tol > 0.0 || st.reltol > 0.0)) ctx->tape_on = true;
    if (ctx->tape_on &&
        !ctx->ensure(ctx->fs_tape, (size_t)(ctx->fs_warps + retry_blocks(ctx)) * kTapeMax * sizeof(TapeCell)))
        return false;
    if (!ctx->check("ld tables", launch_ld_tables(static_cast<double2*>(ctx->fs_ld_coeffs.ptr), nld,
                                                  static_cast<double*>(ctx->fs_ld.ptr), ctx->stream)))
        return false;
    ctx->launches += 1;
    return true;
}

// Per-point ray counts (and cycles) of n points, zeroed.
bool prepare_counts(Context* ctx, long long n)
{
    if (!ctx->ensure(ctx->fs_waits, sizeof(int)) ||
        !ctx->check("waits init", cudaMemsetAsync(ctx->fs_waits.ptr, 0, sizeof(int), ctx->stream)))
        return false;
    if (!ctx->ensure(ctx->fs_levels, (size_t)(n + 1) * sizeof(int)) ||
        !ctx->check("levels init", cudaMemsetAsync(ctx->fs_levels.ptr, 0, (size_t)n * sizeof(int), ctx->stream)))
        return false;
    if (!ctx->ensure(ctx->fs_rays, (size_t)(n + 1) * sizeof(unsigned long long)) ||
        (ctx->item_cycles && !ctx->ensure(ctx->fs_cycles, (size_t)(n + 1) * sizeof(long long))))
        return false;
    if (!ctx->check("rays init", cudaMemsetAsync(ctx->fs_rays.ptr, 0, (size_t)n * sizeof(unsigned long long),
                                                 ctx->stream)))
        return false;
    if (ctx->item_cycles &&
        !ctx->check("cycles init", cudaMemsetAsync(ctx->fs_cycles.ptr, 0, (size_t)n * sizeof(long long), ctx->stream)))
        return false;
    return true;
}

// Runs the pipeline on device-resident items (ctx->fs_items) and writes device
// results to ctx->fs_out.  Everything is asynchronous on ctx->stream.
bool run_pipeline(Context* ctx, const Plan& plan, long long n, double* grads = nullptr)
{
    if (!prepare_tables(ctx, plan) || !prepare_counts(ctx, n)) return false;
    const int nmod = static_cast<int>(plan.models.size());
    long long raw_total = 0;
    for (const auto& m : plan.models) raw_total += 4ll * m.bins;
    if (!ctx->ensure(ctx->fs_raw, (raw_total + 1) * sizeof(P2)) ||
        !ctx->ensure(ctx->fs_branches, (raw_total + 1) * sizeof(P2)) ||
        !ctx->ensure(ctx->fs_ir, (size_t)2 * kChunk * sizeof(int)) ||
        !ctx->ensure(ctx->fs_retry, (size_t)3 * kChunk * sizeof(int)) ||
        !ctx->ensure(ctx->fs_seeds, (size_t)kChunk * ctx->seed_cap * sizeof(P2)) ||
        !ctx->ensure(ctx->fs_tiles, tile_bytes(ctx->tile_capacity, kChunk)))
        return false;
    cudaEvent_t t0;
    ctx->stage_begin(0, &t0);
    if (nmod > 0) {
        if (!ctx->check("caustics", launch_caustics(static_cast<CausticModel*>(ctx->fs_models.ptr), nmod, plan.max_bins,
                                                    static_cast<double2*>(ctx->fs_phases.ptr),
                                                    static_cast<long long*>(ctx->fs_raw_offset.ptr),
                                                    static_cast<P2*>(ctx->fs_raw.ptr), static_cast<P2*>(ctx->fs_branches.ptr),
                                                    ctx->stream)))
            return false;
        ctx->launches += 2;
    }
    ctx->stage_end(0, t0);
    for (long long c0 = 0; c0 < n; c0 += kChunk) {
        const int cn = static_cast<int>((n - c0) < kChunk ? (n - c0) : kChunk);
        FsWork w = common_work(ctx);
        w.items = static_cast<const FsItem*>(ctx->fs_items.ptr) + c0;
        w.models = static_cast<const CausticModel*>(ctx->fs_models.ptr);
        w.raw_offset = static_cast<const long long*>(ctx->fs_raw_offset.ptr);
        w.raw = static_cast<const P2*>(ctx->fs_raw.ptr);
        w.branches = static_cast<const P2*>(ctx->fs_branches.ptr);
        w.out = static_cast<FsOut*>(ctx->fs_out.ptr) + c0;
        w.n_items = cn;
        set_lists(w, static_cast<int*>(ctx->fs_counters.ptr), static_cast<int*>(ctx->fs_ir.ptr),
                  static_cast<int*>(ctx->fs_retry.ptr), kChunk, kChunk);
        w.rays = static_cast<unsigned long long*>(ctx->fs_rays.ptr) + c0;
        w.levels = static_cast<int*>(ctx->fs_levels.ptr) + c0;
        w.cycles = ctx->item_cycles ? static_cast<long long*>(ctx->fs_cycles.ptr) + c0 : nullptr;
        if (!stage_decide(ctx, w) || !stage_seeds(ctx, w, cn) || !stage_integrate(ctx, w, cn)) return false;
        if (grads) {
            if (!ctx->ensure(ctx->fs_grad_tiles, grad_tile_bytes(ctx->tile_capacity, kChunk))) return false;
            if (ctx->grad_blocks == 0) ctx->grad_blocks = grad_flood_blocks_per_sm() * ctx->sm_count;
            if (!ctx->check("gradient", launch_grad(w, ctx->fs_grad_tiles.ptr, ctx->tile_capacity, cn,
                                                    ctx->grad_blocks, ctx->grad_bins, ctx->sm_count, grads + c0 * 8,
                                                    ctx->stream)))
                return false;
            ctx->launches += 6;
        }
    }
    return true;
}

int finish_results(Context* ctx, lcbi_fs_result* results, long long n)
{
    if (!ctx->check("results D2H", cudaMemcpyAsync(results, ctx->fs_out.ptr, n * sizeof(lcbi_fs_result),
                                                   cudaMemcpyDeviceToHost, ctx->stream)) ||
        !ctx->finish())
        return LCBI_GPU_ERROR;
    return LCBI_OK;
}

bool check_settings(Context* ctx, const lcbi_fs_settings* s, int n)
{
    for (int i = 0; i < n; ++i) {
        if (s[i].adaptive_source_bins != 0 && (s[i].finite_source_tol > 0.0 || s[i].finite_source_reltol > 0.0) &&
            s[i].max_source_bins >= kTapeMax)
            return ctx->fail("adaptive refinement records at most 4096 boundary cells: max_source_bins must be below "
                             "4096");
        if (s[i].finite_mode == 3) return ctx->fail("finite_mode 3 (experimental spine integrator) is not implemented");
    }
    return true;
}

} // namespace
} // namespace lcbi

using namespace lcbi;

extern "C" {

namespace lcbi {
namespace {
int binary_mag_impl(Context* ctx, const lcbi_fs_settings* settings, int32_t n_settings, const lcbi_lens_model* models,
                    int32_t n_models, int64_t n, const lcbi_fs_point* points, lcbi_fs_result* results, double* grads,
                    unsigned flags);
}
} // namespace lcbi

int lcbi_gpu_binary_mag(lcbi_gpu_context* c, const lcbi_fs_settings* settings, int32_t n_settings,
                        const lcbi_lens_model* models, int32_t n_models, int64_t n, const lcbi_fs_point* points,
                        lcbi_fs_result* results, unsigned flags)
{
    return binary_mag_impl(reinterpret_cast<Context*>(c), settings, n_settings, models, n_models, n, points, results,
                           nullptr, flags);
}

int lcbi_gpu_binary_mag_grad(lcbi_gpu_context* c, const lcbi_fs_settings* settings, int32_t n_settings,
                             const lcbi_lens_model* models, int32_t n_models, int64_t n, const lcbi_fs_point* points,
                             lcbi_fs_result* results, double* grads, unsigned flags)
{
    if (!grads) return LCBI_INVALID_ARGUMENT;
    return binary_mag_impl(reinterpret_cast<Context*>(c), settings, n_settings, models, n_models, n, points, results,
                           grads, flags);
}

} // extern "C"

namespace lcbi {
namespace {
int binary_mag_impl(Context* ctx, const lcbi_fs_settings* settings, int32_t n_settings, const lcbi_lens_model* models,
                    int32_t n_models, int64_t n, const lcbi_fs_point* points, lcbi_fs_result* results, double* grads,
                    unsigned flags)
{
    if (!ctx || n < 0 || !settings || n_settings <= 0) return LCBI_INVALID_ARGUMENT;
    if (n == 0) return LCBI_OK;
    if (!points || !results) return LCBI_INVALID_ARGUMENT;
    ctx->error.clear();
    cudaSetDevice(ctx->device);
    if (!check_settings(ctx, settings, n_settings)) return LCBI_UNSUPPORTED;
    const bool dev = (flags & LCBI_GPU_DEVICE_POINTERS) != 0;
    const bool given = (flags & LCBI_GPU_MODELS_GIVEN) != 0;
    if (dev && !given) return LCBI_INVALID_ARGUMENT;
    Plan plan;
    add_settings(plan, settings, n_settings);
    ModelTable mt{&plan};
    std::vector<FsItem> items;
    if (given) {
        for (int m = 0; m < n_models; ++m) mt.get(models[m].s, models[m].q, models[m].caustic_bins);
    }
    if (!dev) {
        items.resize(static_cast<size_t>(n));
        std::memcpy(items.data(), points, n * sizeof(FsItem));
        for (auto& it : items) {
            if (it.settings < 0 || it.settings >= n_settings) return LCBI_INVALID_ARGUMENT;
            if (given) {
                if (it.model < 0 || it.model >= n_models) return LCBI_INVALID_ARGUMENT;
            } else if (it.rho > 0.0 && settings[it.settings].finite_mode > 0) {
                it.model = mt.get(it.s, it.q, settings[it.settings].caustic_bins);
            } else {
                it.model = 0;
            }
        }
        if (!upload(ctx, ctx->fs_items, items)) return LCBI_GPU_ERROR;
    } else {
        if (!ctx->ensure(ctx->fs_items, n * sizeof(FsItem)) ||
            !ctx->check("items D2D", cudaMemcpyAsync(ctx->fs_items.ptr, points, n * sizeof(FsItem),
                                                     cudaMemcpyDeviceToDevice, ctx->stream)))
            return LCBI_GPU_ERROR;
    }
    if (!ctx->ensure(ctx->fs_out, n * sizeof(FsOut))) return LCBI_GPU_ERROR;
    double* dgrads = nullptr;
    if (grads) {
        if (dev) {
            dgrads = grads;
        } else {
            if (!ctx->ensure(ctx->fs_grad, (size_t)n * 8 * sizeof(double))) return LCBI_GPU_ERROR;
            dgrads = static_cast<double*>(ctx->fs_grad.ptr);
        }
    }
    if (!run_pipeline(ctx, plan, n, dgrads)) return LCBI_GPU_ERROR;
    if (dev) {
        if (!ctx->check("results D2D", cudaMemcpyAsync(results, ctx->fs_out.ptr, n * sizeof(FsOut),
                                                       cudaMemcpyDeviceToDevice, ctx->stream)) ||
            !ctx->finish())
            return LCBI_GPU_ERROR;
        return LCBI_OK;
    }
    if (grads && !ctx->check("gradients D2H", cudaMemcpyAsync(grads, dgrads, (size_t)n * 8 * sizeof(double),
                                                               cudaMemcpyDeviceToHost, ctx->stream)))
        return LCBI_GPU_ERROR;
    return finish_results(ctx, results, n);
}
} // namespace
} // namespace lcbi

extern "C" {

int lcbi_gpu_autotune(lcbi_gpu_context* c, const lcbi_fs_settings* settings, int32_t n_settings,
                      const lcbi_lens_model* models, int32_t n_models, int64_t n, const lcbi_fs_point* points,
                      lcbi_fs_result* results, unsigned flags, int32_t* shape, double* best_ms)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || !settings || n_settings <= 0 || n <= 0 || !points || !results) return LCBI_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    cudaEvent_t e0, e1;
    if (!ctx->check("event", cudaEventCreate(&e0)) || !ctx->check("event", cudaEventCreate(&e1))) return LCBI_GPU_ERROR;
    struct Events {
        cudaEvent_t a, b;
        ~Events() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } guard{e0, e1};
    const int sm = ctx->sm_count;
    const int occupancy = polar_tile_blocks_per_sm();
    // One shape: {tile flood blocks per SM, first-pass warps per SM, second-pass blocks}.
    auto apply = [&](const int* sh) {
        ctx->tile_blocks = sh[0] * sm;
        ctx->warps_per_sm = sh[1];
        if (sh[2] != ctx->retry_blocks) {
            ctx->retry_blocks = sh[2];
            ctx->big_ready = false;
        }
    };
    // Time of one call with a shape, after one untimed call (allocations, caches).
    auto measure = [&](const int* sh, double* ms) -> int {
        apply(sh);
        int rc = binary_mag_impl(ctx, settings, n_settings, models, n_models, n, points, results, nullptr, flags);
        if (rc != LCBI_OK) return rc;
        if (!ctx->check("event", cudaEventRecord(e0, ctx->stream))) return LCBI_GPU_ERROR;
        rc = binary_mag_impl(ctx, settings, n_settings, models, n_models, n, points, results, nullptr, flags);
        if (rc != LCBI_OK) return rc;
        float t = 0.0f;
        if (!ctx->check("event", cudaEventRecord(e1, ctx->stream)) ||
            !ctx->check("event", cudaEventSynchronize(e1)) || !ctx->check("event", cudaEventElapsedTime(&t, e0, e1)))
            return LCBI_GPU_ERROR;
        *ms = t;
        return LCBI_OK;
    };
    // Coordinate search: flood blocks, then first-pass warps, then second-pass blocks.
    int best[3] = {occupancy, ctx->warps_per_sm, ctx->retry_blocks > 0 ? ctx->retry_blocks : sm};
    double best_t = 0.0;
    int rc = measure(best, &best_t);
    if (rc != LCBI_OK) return rc;
    const int floods[4] = {1, 2, 4, occupancy};
    const int warps[2] = {4, 8};
    const int seconds[2] = {sm, 2 * sm};
    for (int axis = 0; axis < 3; ++axis) {
        const int* cand = axis == 0 ? floods : (axis == 1 ? warps : seconds);
        const int nc = axis == 0 ? 4 : 2;
        for (int i = 0; i < nc; ++i) {
            int sh[3] = {best[0], best[1], best[2]};
            sh[axis] = cand[i];
            if (sh[axis] == best[axis] || sh[axis] <= 0) continue;
            double t = 0.0;
            rc = measure(sh, &t);
            if (rc != LCBI_OK) return rc;
            if (t < best_t) {
                best_t = t;
                best[0] = sh[0];
                best[1] = sh[1];
                best[2] = sh[2];
            }
        }
    }
    apply(best);
    if (shape) {
        shape[0] = best[0];
        shape[1] = best[1];
        shape[2] = best[2];
    }
    if (best_ms) *best_ms = best_t;
    return LCBI_OK;
}

int lcbi_gpu_binary_inverse_ray(lcbi_gpu_context* c, const lcbi_fs_settings* settings, int64_t n, const double* s,
                                const double* q, const double* y1, const double* y2, const double* rho, double* A,
                                int32_t* method, int32_t* status)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || !settings || n < 0) return LCBI_INVALID_ARGUMENT;
    if (n == 0) return LCBI_OK;
    if (!s || !q || !y1 || !y2 || !rho || !A) return LCBI_INVALID_ARGUMENT;
    lcbi_fs_settings st = *settings;
    st.kinji_threshold = 1e18;
    st.hex_threshold = 0.0;
    st.adaptive_hex_threshold = 0.0;
    std::vector<lcbi_fs_point> pts(static_cast<size_t>(n));
    for (long long i = 0; i < n; ++i) {
        lcbi_fs_point& p = pts[i];
        p.s = s[i];
        p.q = q[i];
        p.y1 = y1[i];
        p.y2 = y2[i];
        p.rho = std::fabs(rho[i]);
        p.point_source_magnification = 0.0;
        p.settings = 0;
        p.model = 0;
        p.flags = LCBI_FS_PS_EXACT | LCBI_FS_PS_ON_DEVICE;
        p.reserved = 0;
    }
    std::vector<lcbi_fs_result> res(static_cast<size_t>(n));
    const int rc = lcbi_gpu_binary_mag(c, &st, 1, nullptr, 0, n, pts.data(), res.data(), 0);
    if (rc != LCBI_OK) return rc;
    for (long long i = 0; i < n; ++i) {
        A[i] = res[i].magnification;
        if (method) method[i] = res[i].method;
        if (status) status[i] = res[i].status;
    }
    return LCBI_OK;
}

int lcbi_gpu_light_curves(lcbi_gpu_context* c, const lcbi_fs_settings* settings, int32_t n_models,
                          const double* params, const int64_t* first, const int32_t* count, const double* times,
                          int64_t n_times, double* A, int32_t* method, int32_t* status)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || !settings || n_models < 0 || n_times < 0) return LCBI_INVALID_ARGUMENT;
    if (n_models == 0 || n_times == 0) return LCBI_OK;
    if (!params || !first || !count || !times || !A) return LCBI_INVALID_ARGUMENT;
    ctx->error.clear();
    cudaSetDevice(ctx->device);
    if (!check_settings(ctx, settings, 1)) return LCBI_UNSUPPORTED;
    Plan plan;
    add_settings(plan, settings, 1);
    ModelTable mt{&plan};
    std::vector<LcModel> lcm(static_cast<size_t>(n_models));
    for (int m = 0; m < n_models; ++m) {
        const double* p = params + 7 * m;
        if (first[m] < 0 || count[m] < 0 || first[m] + count[m] > n_times) return LCBI_INVALID_ARGUMENT;
        LcModel& L = lcm[m];
        L.t0 = p[0];
        L.tE = p[1];
        L.u0 = p[2];
        L.cos_alpha = std::cos(p[3]);
        L.sin_alpha = std::sin(p[3]);
        L.s = p[4];
        L.q_core = p[5] != 0.0 ? 1.0 / p[5] : p[5];
        L.rho = p[6];
        L.first = first[m];
        L.count = count[m];
        L.settings = 0;
        L.model = (p[6] != 0.0 && settings->finite_mode > 0) ? mt.get(L.s, L.q_core, settings->caustic_bins) : 0;
        L.pad = 0;
    }
    if (!upload(ctx, ctx->fs_lc_models, lcm) || !ctx->ensure(ctx->fs_times, n_times * sizeof(double)) ||
        !ctx->check("times H2D", cudaMemcpyAsync(ctx->fs_times.ptr, times, n_times * sizeof(double),
                                                 cudaMemcpyHostToDevice, ctx->stream)) ||
        !ctx->ensure(ctx->fs_items, n_times * sizeof(FsItem)) || !ctx->ensure(ctx->fs_out, n_times * sizeof(FsOut)))
        return LCBI_GPU_ERROR;
    if (!ctx->check("lc items", launch_lc_items(static_cast<LcModel*>(ctx->fs_lc_models.ptr), n_models,
                                                static_cast<double*>(ctx->fs_times.ptr),
                                                static_cast<FsItem*>(ctx->fs_items.ptr), n_times, ctx->stream)))
        return LCBI_GPU_ERROR;
    ctx->launches += 1;
    if (!run_pipeline(ctx, plan, n_times)) return LCBI_GPU_ERROR;
    std::vector<lcbi_fs_result> res(static_cast<size_t>(n_times));
    const int rc = finish_results(ctx, res.data(), n_times);
    if (rc != LCBI_OK) return rc;
    for (long long i = 0; i < n_times; ++i) {
        A[i] = res[i].magnification;
        if (method) method[i] = res[i].method;
        if (status) status[i] = res[i].status;
    }
    return LCBI_OK;
}

namespace {
// lcbi_gpu_light_curves_grad with the per-epoch arrays (times, A, dA, method,
// status) on the host (dev = false) or on the device (dev = true).  The
// model parameters, first and count are host arrays either way: they define
// the caustic models and the work the host plans.
int light_curves_grad_impl(Context* ctx, const lcbi_fs_settings* settings, int32_t n_models, const double* params,
                           const int64_t* first, const int32_t* count, const double* times, int64_t n_times,
                           double* A, double* dA, int32_t* method, int32_t* status, bool dev)
{
    if (!ctx || !settings || n_models < 0 || n_times < 0) return LCBI_INVALID_ARGUMENT;
    if (n_models == 0 || n_times == 0) return LCBI_OK;
    if (!params || !first || !count || !times || !A) return LCBI_INVALID_ARGUMENT;
    ctx->error.clear();
    cudaSetDevice(ctx->device);
    if (!check_settings(ctx, settings, 1)) return LCBI_UNSUPPORTED;
    // One settings entry per distinct Gamma (the models' linear limb darkening).
    std::vector<lcbi_fs_settings> sts;
    std::vector<int> model_settings(static_cast<size_t>(n_models));
    for (int m = 0; m < n_models; ++m) {
        const double g = params[8 * m + 7];
        int idx = -1;
        for (size_t k = 0; k < sts.size(); ++k)
            if (sts[k].limb_darkening_c == g) idx = static_cast<int>(k);
        if (idx < 0) {
            lcbi_fs_settings st = settings[0];
            st.limb_darkening_c = g;
            st.limb_darkening_d = 0.0;
            idx = static_cast<int>(sts.size());
            sts.push_back(st);
        }
        model_settings[m] = idx;
    }
    Plan plan;
    add_settings(plan, sts.data(), static_cast<int>(sts.size()));
    ModelTable mt{&plan};
    std::vector<LcModel> lcm(static_cast<size_t>(n_models));
    for (int m = 0; m < n_models; ++m) {
        const double* p = params + 8 * m;
        if (first[m] < 0 || count[m] < 0 || first[m] + count[m] > n_times) return LCBI_INVALID_ARGUMENT;
        LcModel& L = lcm[m];
        L.t0 = p[0];
        L.tE = p[1];
        L.u0 = p[2];
        L.cos_alpha = std::cos(p[3]);
        L.sin_alpha = std::sin(p[3]);
        L.s = p[4];
        L.q_core = p[5] != 0.0 ? 1.0 / p[5] : p[5];
        L.rho = p[6];
        L.first = first[m];
        L.count = count[m];
        L.settings = model_settings[m];
        L.model = (p[6] != 0.0 && settings->finite_mode > 0) ? mt.get(L.s, L.q_core, settings->caustic_bins) : 0;
        L.pad = 0;
    }
    const double* dt = times;
    if (!upload(ctx, ctx->fs_lc_models, lcm) || !ctx->ensure(ctx->fs_items, n_times * sizeof(FsItem)) ||
        !ctx->ensure(ctx->fs_out, n_times * sizeof(FsOut)) ||
        !ctx->ensure(ctx->fs_grad, (size_t)n_times * 8 * sizeof(double)) ||
        !ctx->ensure(ctx->fs_grad_lc, (size_t)n_times * 8 * sizeof(double)))
        return LCBI_GPU_ERROR;
    if (!dev) {
        if (!ctx->ensure(ctx->fs_times, n_times * sizeof(double)) ||
            !ctx->check("times H2D", cudaMemcpyAsync(ctx->fs_times.ptr, times, n_times * sizeof(double),
                                                     cudaMemcpyHostToDevice, ctx->stream)))
            return LCBI_GPU_ERROR;
        dt = static_cast<double*>(ctx->fs_times.ptr);
    }
    const LcModel* dm = static_cast<LcModel*>(ctx->fs_lc_models.ptr);
    if (!ctx->check("lc items", launch_lc_items(dm, n_models, dt, static_cast<FsItem*>(ctx->fs_items.ptr), n_times,
                                                ctx->stream)))
        return LCBI_GPU_ERROR;
    ctx->launches += 1;
    double* pg = dA ? static_cast<double*>(ctx->fs_grad.ptr) : nullptr;
    if (!run_pipeline(ctx, plan, n_times, pg)) return LCBI_GPU_ERROR;
    if (dA) {
        double* chain_out = dev ? dA : static_cast<double*>(ctx->fs_grad_lc.ptr);
        if (!ctx->check("gradient chain", launch_lc_grad_chain(dm, n_models, dt, pg, chain_out, n_times, ctx->stream)))
            return LCBI_GPU_ERROR;
        ctx->launches += 1;
        if (!dev && !ctx->check("gradients D2H", cudaMemcpyAsync(dA, ctx->fs_grad_lc.ptr,
                                                                  (size_t)n_times * 8 * sizeof(double),
                                                                  cudaMemcpyDeviceToHost, ctx->stream)))
            return LCBI_GPU_ERROR;
    }
    if (dev) {
        if (!ctx->check("results", launch_unpack_results(static_cast<const FsOut*>(ctx->fs_out.ptr), A, method, status,
                                                         n_times, ctx->stream)) ||
            !ctx->finish())
            return LCBI_GPU_ERROR;
        ctx->launches += 1;
        return LCBI_OK;
    }
    std::vector<lcbi_fs_result> res(static_cast<size_t>(n_times));
    const int rc = finish_results(ctx, res.data(), n_times);
    if (rc != LCBI_OK) return rc;
    for (long long i = 0; i < n_times; ++i) {
        A[i] = res[i].magnification;
        if (method) method[i] = res[i].method;
        if (status) status[i] = res[i].status;
    }
    return LCBI_OK;
}
} // namespace

int lcbi_gpu_light_curves_grad(lcbi_gpu_context* c, const lcbi_fs_settings* settings, int32_t n_models,
                               const double* params, const int64_t* first, const int32_t* count, const double* times,
                               int64_t n_times, double* A, double* dA, int32_t* method, int32_t* status)
{
    return light_curves_grad_impl(reinterpret_cast<Context*>(c), settings, n_models, params, first, count, times,
                                  n_times, A, dA, method, status, false);
}

int lcbi_gpu_light_curves_grad_device(lcbi_gpu_context* c, const lcbi_fs_settings* settings, int32_t n_models,
                                      const double* params, const int64_t* first, const int32_t* count,
                                      const double* times, int64_t n_times, double* A, double* dA, int32_t* method,
                                      int32_t* status)
{
    return light_curves_grad_impl(reinterpret_cast<Context*>(c), settings, n_models, params, first, count, times,
                                  n_times, A, dA, method, status, true);
}

} // extern "C"

namespace lcbi {

// Grows b to at least `bytes`, keeping its contents (stream-ordered copy).
bool grow_keep(Context* ctx, Buffer& b, size_t bytes)
{
    if (b.bytes >= bytes) return true;
    Buffer nb;
    size_t want = b.bytes * 2 > bytes ? b.bytes * 2 : bytes;
    want = (want + 0xffff) & ~size_t(0xffff);
    if (!ctx->check("cudaMalloc", cudaMalloc(&nb.ptr, want))) return false;
    nb.bytes = want;
    if (b.ptr) {
        if (!ctx->check("store copy", cudaMemcpyAsync(nb.ptr, b.ptr, b.bytes, cudaMemcpyDeviceToDevice, ctx->stream)))
            return false;
        cudaFree(b.ptr);  // waits for the copy
    }
    b = nb;
    return true;
}

// Large batches in which every point may have its own separation (lens
// orbital motion): the caustic sampling and the decision run pass by pass, a
// pass's caustic samples being dropped once it is decided, and the few
// inverse-ray points of all passes are seeded and integrated together at the
// end, so that no pass waits for its slowest inverse-ray point.  Two passes
// are in flight: while the GPU samples and decides pass p, the host collects
// the inverse-ray points of pass p - 1 and has their caustic models copied
// into a store that outlives the pass.
int binary_mag_images(lcbi_gpu_context* c, const lcbi_fs_settings* settings, int n_settings,
                      const lcbi_fs_point* points, long long n, lcbi_fs_result* results, double* a_ps,
                      int32_t* image_count, int32_t* levels)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || n < 0 || !settings || n_settings <= 0) return LCBI_INVALID_ARGUMENT;
    if (n == 0) return LCBI_OK;
    if (!points || !results || !a_ps || !image_count || n > (1ll << 30)) return LCBI_INVALID_ARGUMENT;
    for (long long i = 0; i < n; ++i)
        if (points[i].settings < 0 || points[i].settings >= n_settings) return LCBI_INVALID_ARGUMENT;
    ctx->error.clear();
    cudaSetDevice(ctx->device);
    if (!check_settings(ctx, settings, n_settings)) return LCBI_UNSUPPORTED;

    // Host: the points and every pass's caustic models (indices relative to the pass).
    const long long n_pass = (n + kChunk - 1) / kChunk;
    std::vector<FsItem> items(static_cast<size_t>(n));
    std::memcpy(items.data(), points, n * sizeof(FsItem));
    Plan plan;
    add_settings(plan, settings, n_settings);
    ModelTable mt{&plan};
    std::vector<int> model_base(static_cast<size_t>(n_pass + 1));
    long long max_raw = 0;
    for (long long p = 0; p < n_pass; ++p) {
        mt.restart_pass();
        model_base[p] = static_cast<int>(plan.models.size());
        const long long e1 = (p + 1) * kChunk < n ? (p + 1) * kChunk : n;
        for (long long i = p * kChunk; i < e1; ++i) {
            FsItem& it = items[i];
            const lcbi_fs_settings& st = settings[it.settings];
            it.a_ps = 0.0;
            it.flags = kItemPsExact | kItemSeedHints;
            it.model = (it.rho > 0.0 && st.finite_mode > 0)
                           ? mt.get_sequential(it.s, it.q, st.caustic_bins) - model_base[p]
                           : 0;
        }
        if (mt.raw_total > max_raw) max_raw = mt.raw_total;
    }
    model_base[n_pass] = static_cast<int>(plan.models.size());

    // Device: tables, all points and their point-source values.
    if (!prepare_tables(ctx, plan) || !prepare_counts(ctx, n) || !upload(ctx, ctx->fs_items, items) ||
        !ctx->ensure(ctx->fs_out, n * sizeof(FsOut)) || !ctx->ensure(ctx->fs_all_aps, n * sizeof(double)) ||
        !ctx->ensure(ctx->fs_all_nimg, n * sizeof(int)))
        return LCBI_GPU_ERROR;
    FsItem* d_items = static_cast<FsItem*>(ctx->fs_items.ptr);
    FsOut* d_out = static_cast<FsOut*>(ctx->fs_out.ptr);
    CausticModel* d_models = static_cast<CausticModel*>(ctx->fs_models.ptr);
    const long long* d_ro = static_cast<const long long*>(ctx->fs_raw_offset.ptr);
    if (!ctx->check("images", launch_item_images(d_items, n, static_cast<double*>(ctx->fs_all_aps.ptr),
                                                 static_cast<int*>(ctx->fs_all_nimg.ptr), ctx->sm_count, ctx->stream)))
        return LCBI_GPU_ERROR;
    ctx->launches += 1;
    // Points that provably take the decision's bounding-box exit need no
    // caustic samples; only the models of the others are sampled.
    const size_t n_models_all = plan.models.size();
    if (!upload(ctx, ctx->fs_model_base, model_base) || !ctx->ensure(ctx->fs_needed, n_models_all + 1) ||
        !ctx->check("needed init", cudaMemsetAsync(ctx->fs_needed.ptr, 0, n_models_all + 1, ctx->stream)) ||
        !ctx->check("certify", launch_certify(d_items, n, static_cast<const FsSettingsDev*>(ctx->fs_settings.ptr),
                                              static_cast<const int*>(ctx->fs_model_base.ptr), kChunk,
                                              static_cast<unsigned char*>(ctx->fs_needed.ptr), ctx->sm_count,
                                              ctx->stream)))
        return LCBI_GPU_ERROR;
    ctx->launches += 1;
    const unsigned char* d_needed = static_cast<const unsigned char*>(ctx->fs_needed.ptr);

    // Pass buffers (two sets) and page-locked staging of their lists and jobs.
    const size_t list_ints = 2 * static_cast<size_t>(kChunk);
    const size_t job_bytes = static_cast<size_t>(kChunk) * (sizeof(StashJob) + sizeof(StashRemap));
    const size_t stage_bytes = (64 + list_ints) * sizeof(int) + job_bytes;
    for (int k = 0; k < 2; ++k) {
        if (!ctx->ensure(ctx->pass_raw[k], (max_raw + 1) * sizeof(P2)) ||
            !ctx->ensure(ctx->pass_branches[k], (max_raw + 1) * sizeof(P2)) ||
            !ctx->ensure(ctx->pass_lists[k], list_ints * sizeof(int)) ||
            !ctx->ensure(ctx->pass_counters[k], kCounterInts * sizeof(int)) || !ctx->ensure(ctx->pass_jobs[k], job_bytes))
            return LCBI_GPU_ERROR;
    }
    if (ctx->pinned_bytes < 2 * stage_bytes) {
        if (ctx->pinned) cudaFreeHost(ctx->pinned);
        ctx->pinned = nullptr;
        ctx->pinned_bytes = 0;
        if (!ctx->check("cudaMallocHost", cudaMallocHost(&ctx->pinned, 2 * stage_bytes))) return LCBI_GPU_ERROR;
        ctx->pinned_bytes = 2 * stage_bytes;
    }
    auto stage_of = [&](int k) { return static_cast<char*>(ctx->pinned) + k * stage_bytes; };
    cudaEvent_t pass_done[2];
    for (int k = 0; k < 2; ++k)
        if (!ctx->check("event", cudaEventCreateWithFlags(&pass_done[k], cudaEventDisableTiming))) return LCBI_GPU_ERROR;
    struct Events {
        cudaEvent_t* e;
        ~Events() { cudaEventDestroy(e[0]); cudaEventDestroy(e[1]); }
    } events_guard{pass_done};

    std::vector<int> g_cart, g_polar;
    long long store_models = 0, store_points = 0;
    std::vector<int> dst_of;  // per model of the pass being collected: store index, or -1

    auto enqueue_pass = [&](long long p) -> bool {
        const int k = static_cast<int>(p & 1);
        const long long c0 = p * kChunk;
        const int cn = static_cast<int>((n - c0) < kChunk ? (n - c0) : kChunk);
        const int base = model_base[p];
        const int nmod = model_base[p + 1] - base;
        cudaEvent_t ev;
        ctx->stage_begin(0, &ev);
        if (nmod > 0) {
            if (!ctx->check("caustics", launch_caustics(d_models + base, nmod, plan.max_bins,
                                                        static_cast<double2*>(ctx->fs_phases.ptr), d_ro + base,
                                                        static_cast<P2*>(ctx->pass_raw[k].ptr),
                                                        static_cast<P2*>(ctx->pass_branches[k].ptr), ctx->stream,
                                                        d_needed + base)))
                return false;
            ctx->launches += 2;
        }
        ctx->stage_end(0, ev);
        FsWork w = common_work(ctx);
        w.items = d_items + c0;
        w.models = d_models + base;
        w.raw_offset = d_ro + base;
        w.raw = static_cast<const P2*>(ctx->pass_raw[k].ptr);
        w.branches = static_cast<const P2*>(ctx->pass_branches[k].ptr);
        w.out = d_out + c0;
        w.n_items = cn;
        set_lists(w, static_cast<int*>(ctx->pass_counters[k].ptr), static_cast<int*>(ctx->pass_lists[k].ptr),
                  nullptr, kChunk, 0);
        w.rays = static_cast<unsigned long long*>(ctx->fs_rays.ptr) + c0;
        w.cycles = ctx->item_cycles ? static_cast<long long*>(ctx->fs_cycles.ptr) + c0 : nullptr;
        if (!stage_decide(ctx, w)) return false;
        int* st = reinterpret_cast<int*>(stage_of(k));
        return ctx->check("lists D2H", cudaMemcpyAsync(st, ctx->pass_counters[k].ptr, 64 * sizeof(int),
                                                       cudaMemcpyDeviceToHost, ctx->stream)) &&
               ctx->check("lists D2H", cudaMemcpyAsync(st + 64, ctx->pass_lists[k].ptr, list_ints * sizeof(int),
                                                       cudaMemcpyDeviceToHost, ctx->stream)) &&
               ctx->check("event", cudaEventRecord(pass_done[k], ctx->stream));
    };

    auto collect_pass = [&](long long p) -> bool {
        const int k = static_cast<int>(p & 1);
        const long long c0 = p * kChunk;
        const int base = model_base[p];
        if (!ctx->check("pass wait", cudaEventSynchronize(pass_done[k]))) return false;
        const int* st = reinterpret_cast<const int*>(stage_of(k));
        const int nc = st[0], np = st[1];
        const int* lists = st + 64;
        StashJob* jobs = reinterpret_cast<StashJob*>(stage_of(k) + (64 + list_ints) * sizeof(int));
        StashRemap* remaps = reinterpret_cast<StashRemap*>(jobs + kChunk);
        dst_of.assign(static_cast<size_t>(model_base[p + 1] - base), -1);
        int n_jobs = 0, n_remaps = 0;
        for (int j = 0; j < nc + np; ++j) {
            const int it = j < nc ? lists[j] : lists[kChunk + (j - nc)];
            const long long g = c0 + it;
            const int m = items[g].model;
            if (dst_of[m] < 0) {
                dst_of[m] = static_cast<int>(store_models++);
                jobs[n_jobs++] = StashJob{m, dst_of[m], store_points};
                store_points += 4ll * plan.models[base + m].bins;
            }
            remaps[n_remaps++] = StashRemap{g, dst_of[m], 0};
            (j < nc ? g_cart : g_polar).push_back(static_cast<int>(g));
        }
        if (n_jobs == 0) return true;
        if (!grow_keep(ctx, ctx->ir_models, (size_t)store_models * sizeof(CausticModel)) ||
            !grow_keep(ctx, ctx->ir_branches, (size_t)store_points * sizeof(P2)))
            return false;
        char* dj = static_cast<char*>(ctx->pass_jobs[k].ptr);
        if (!ctx->check("jobs H2D", cudaMemcpyAsync(dj, jobs, n_jobs * sizeof(StashJob), cudaMemcpyHostToDevice,
                                                    ctx->stream)) ||
            !ctx->check("jobs H2D", cudaMemcpyAsync(dj + kChunk * sizeof(StashJob), remaps,
                                                    n_remaps * sizeof(StashRemap), cudaMemcpyHostToDevice,
                                                    ctx->stream)))
            return false;
        ctx->launches += 1;
        return ctx->check("stash", launch_stash(d_models + base, static_cast<const P2*>(ctx->pass_branches[k].ptr),
                                                reinterpret_cast<const StashJob*>(dj), n_jobs,
                                                static_cast<CausticModel*>(ctx->ir_models.ptr),
                                                static_cast<P2*>(ctx->ir_branches.ptr),
                                                reinterpret_cast<const StashRemap*>(dj + kChunk * sizeof(StashJob)),
                                                n_remaps, d_items, ctx->stream));
    };

    for (long long p = 0; p < n_pass; ++p) {
        if (!enqueue_pass(p)) return LCBI_GPU_ERROR;
        if (p > 0 && !collect_pass(p - 1)) return LCBI_GPU_ERROR;
    }
    if (!collect_pass(n_pass - 1)) return LCBI_GPU_ERROR;

    // All inverse-ray points: seeds, then the integration.
    const int n_cart = static_cast<int>(g_cart.size());
    const int n_polar = static_cast<int>(g_polar.size());
    const int n_ir = n_cart + n_polar;
    if (n_ir > 0) {
        std::vector<int> lists(g_cart);
        lists.insert(lists.end(), g_polar.begin(), g_polar.end());
        std::vector<int> counters(kCounterInts, 0);
        counters[0] = n_cart;
        counters[1] = n_polar;
        if (!upload(ctx, ctx->ir_lists, lists) || !upload(ctx, ctx->ir_counters, counters) ||
            !ctx->ensure(ctx->ir_retry, (size_t)3 * n_ir * sizeof(int)) ||
            !ctx->ensure(ctx->fs_seeds, (size_t)n_ir * ctx->seed_cap * sizeof(P2)) ||
            !ctx->ensure(ctx->fs_tiles, tile_bytes(ctx->tile_capacity, n_ir)))
            return LCBI_GPU_ERROR;
        FsWork w = common_work(ctx);
        w.items = d_items;
        w.models = static_cast<const CausticModel*>(ctx->ir_models.ptr);
        w.branches = static_cast<const P2*>(ctx->ir_branches.ptr);
        w.out = d_out;
        w.n_items = 0;
        set_lists(w, static_cast<int*>(ctx->ir_counters.ptr), static_cast<int*>(ctx->ir_lists.ptr),
                  static_cast<int*>(ctx->ir_retry.ptr), n_cart, n_ir);
        w.rays = static_cast<unsigned long long*>(ctx->fs_rays.ptr);
        w.levels = static_cast<int*>(ctx->fs_levels.ptr);
        w.cycles = ctx->item_cycles ? static_cast<long long*>(ctx->fs_cycles.ptr) : nullptr;
        if (!stage_seeds(ctx, w, n_ir) || !stage_integrate(ctx, w, n_ir)) return LCBI_GPU_ERROR;
    }
    if (!ctx->check("results D2H", cudaMemcpyAsync(results, d_out, n * sizeof(lcbi_fs_result),
                                                   cudaMemcpyDeviceToHost, ctx->stream)) ||
        !ctx->check("a_ps D2H", cudaMemcpyAsync(a_ps, ctx->fs_all_aps.ptr, n * sizeof(double), cudaMemcpyDeviceToHost,
                                                ctx->stream)) ||
        !ctx->check("images D2H", cudaMemcpyAsync(image_count, ctx->fs_all_nimg.ptr, n * sizeof(int32_t),
                                                  cudaMemcpyDeviceToHost, ctx->stream)) ||
        (levels && !ctx->check("levels D2H", cudaMemcpyAsync(levels, ctx->fs_levels.ptr, n * sizeof(int32_t),
                                                             cudaMemcpyDeviceToHost, ctx->stream))) ||
        !ctx->finish())
        return LCBI_GPU_ERROR;
    return LCBI_OK;
}

} // namespace lcbi

extern "C" {

int lcbi_gpu_binary_geometry(lcbi_gpu_context* c, double s, double q, int32_t n_points, int32_t caustic,
                             double* xy, int32_t* points_per_branch)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || !xy || n_points < 8) return LCBI_INVALID_ARGUMENT;
    if (!std::isfinite(s) || !std::isfinite(q) || s == 0.0 || q == 0.0) return LCBI_INVALID_ARGUMENT;
    ctx->error.clear();
    cudaSetDevice(ctx->device);
    Plan plan;
    ModelTable mt{&plan};
    mt.add(s, q, n_points);
    if (!upload(ctx, ctx->fs_models, plan.models) || !upload(ctx, ctx->fs_raw_offset, plan.raw_offset) ||
        !upload(ctx, ctx->fs_phases, plan.phases) ||
        !ctx->ensure(ctx->fs_raw, (4ll * n_points + 1) * sizeof(P2)) ||
        !ctx->ensure(ctx->fs_branches, (4ll * n_points + 1) * sizeof(P2)))
        return LCBI_GPU_ERROR;
    if (!ctx->check("geometry", launch_caustics(static_cast<CausticModel*>(ctx->fs_models.ptr), 1, n_points,
                                                static_cast<double2*>(ctx->fs_phases.ptr),
                                                static_cast<long long*>(ctx->fs_raw_offset.ptr),
                                                static_cast<P2*>(ctx->fs_raw.ptr),
                                                static_cast<P2*>(ctx->fs_branches.ptr), ctx->stream, nullptr,
                                                caustic == 0)))
        return LCBI_GPU_ERROR;
    ctx->launches += 2;
    if (!ctx->check("geometry D2H", cudaMemcpyAsync(xy, ctx->fs_branches.ptr, 4ll * n_points * sizeof(P2),
                                                    cudaMemcpyDeviceToHost, ctx->stream)) ||
        !ctx->finish())
        return LCBI_GPU_ERROR;
    if (points_per_branch) *points_per_branch = n_points;
    return LCBI_OK;
}

int lcbi_gpu_last_item_cycles(lcbi_gpu_context* c, int64_t n, int64_t* cycles)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || !cycles || n < 0) return LCBI_INVALID_ARGUMENT;
    if (n == 0) return LCBI_OK;
    if (!ctx->item_cycles || ctx->fs_cycles.ptr == nullptr || (size_t)n * sizeof(int64_t) > ctx->fs_cycles.bytes)
        return LCBI_INVALID_ARGUMENT;
    if (!ctx->check("cycles D2H", cudaMemcpyAsync(cycles, ctx->fs_cycles.ptr, n * sizeof(int64_t),
                                                  cudaMemcpyDeviceToHost, ctx->stream)) ||
        !ctx->finish())
        return LCBI_GPU_ERROR;
    return LCBI_OK;
}

int lcbi_gpu_last_ray_counts(lcbi_gpu_context* c, int64_t n, uint64_t* rays)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || !rays || n < 0) return LCBI_INVALID_ARGUMENT;
    if (n == 0) return LCBI_OK;
    if (ctx->fs_rays.ptr == nullptr || (size_t)n * sizeof(uint64_t) > ctx->fs_rays.bytes) return LCBI_INVALID_ARGUMENT;
    if (!ctx->check("rays D2H", cudaMemcpyAsync(rays, ctx->fs_rays.ptr, n * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                                ctx->stream)) ||
        !ctx->finish())
        return LCBI_GPU_ERROR;
    return LCBI_OK;
}

int lcbi_gpu_set_wait_limit(lcbi_gpu_context* c, uint32_t polls)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx) return LCBI_INVALID_ARGUMENT;
    ctx->wait_limit = polls;
    return LCBI_OK;
}

int lcbi_gpu_last_wait_timeouts(lcbi_gpu_context* c, int32_t* count)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || !count) return LCBI_INVALID_ARGUMENT;
    *count = 0;
    if (ctx->fs_waits.ptr == nullptr) return LCBI_OK;
    if (!ctx->check("waits D2H", cudaMemcpyAsync(count, ctx->fs_waits.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                                 ctx->stream)) ||
        !ctx->finish())
        return LCBI_GPU_ERROR;
    return LCBI_OK;
}

int lcbi_gpu_last_refinement_levels(lcbi_gpu_context* c, int64_t n, int32_t* levels)
{
    Context* ctx = reinterpret_cast<Context*>(c);
    if (!ctx || !levels || n < 0) return LCBI_INVALID_ARGUMENT;
    if (n == 0) return LCBI_OK;
    if (ctx->fs_levels.ptr == nullptr || (size_t)n * sizeof(int32_t) > ctx->fs_levels.bytes)
        return LCBI_INVALID_ARGUMENT;
    if (!ctx->check("levels D2H", cudaMemcpyAsync(levels, ctx->fs_levels.ptr, n * sizeof(int32_t),
                                                  cudaMemcpyDeviceToHost, ctx->stream)) ||
        !ctx->finish())
        return LCBI_GPU_ERROR;
    return LCBI_OK;
}

} // extern "C"
