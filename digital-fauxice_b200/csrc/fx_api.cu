// fx_api.cu -- C ABI, device memory and per-frame pipelines.
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <mutex>
#include <thread>
#include <algorithm>
#include <vector>

#include <openssl/evp.h>

#include "fx_internal.cuh"

namespace fx {

static Geometry make_geometry(int h, int w) {
    Geometry g;
    g.h = h;
    g.w = w;
    g.th = (h + kTileH - 1) / kTileH;
    g.tw = (w + kTileW - 1) / kTileW;
    g.hp = g.th * kTileH;
    g.wp = g.tw * kTileW;
    g.prow = g.hp + 2 * kPad;
    g.pitch = ((g.wp + 2 * kPad) + 31) / 32 * 32;
    g.sites = 6 * (int64_t)w + (int64_t)h * w;
    g.segments = (g.sites + kSegment - 1) / kSegment;
    return g;
}

static int64_t default_amb_capacity(const Geometry &g) {
    const int64_t c = g.sites / 2;
    return c < 65536 ? 65536 : c;
}

// One frame's device buffers, carved from a single allocation.
struct Arena {
    void *base = nullptr;
    size_t bytes = 0;
    uint16_t *rgbi = nullptr;
    fx_stage *stages = nullptr;
    float *aux = nullptr, *hs = nullptr, *hwa = nullptr, *hwr = nullptr;
    double *cand = nullptr;
    uint8_t *meta = nullptr;
    uint32_t *seg_base = nullptr, *seg_amb = nullptr;
    uint32_t *seg_raw = nullptr;  // seg_raw_words(segments): per-segment and per-block sums
    AmbEntry *entries = nullptr;
    uint32_t *pos = nullptr, *extra = nullptr;
    uint8_t *chunk_two = nullptr;
    void *producer = nullptr;
    float *rows = nullptr;
    uint16_t *out = nullptr;
    uint8_t *changed = nullptr;
    void *counters = nullptr;
    uint32_t *err = nullptr;
    void *walk = nullptr;
    int64_t amb_capacity = 0;
};

static int g_per_wave = 444;  // window blocks per wave: walk_per_wave(SM count)

static size_t arena_layout(const Geometry &g, int64_t amb_cap, Arena *a) {
    size_t off = 0;
    auto take = [&](size_t n) {
        const size_t o = off;
        off += (n + 255) & ~(size_t)255;
        return o;
    };
    const int64_t px = (int64_t)g.h * g.w;
    const int64_t plane = (int64_t)g.prow * g.pitch;
    const size_t o_rgbi = take(px * 8);
    const size_t o_stages = take((g.h + 6) * sizeof(fx_stage));
    const size_t o_aux = take(plane * 4);  // padded, edge-replicated
    const size_t o_hs = take(plane * 4);
    const size_t o_hwa = take(plane * 4);
    const size_t o_hwr = take(3 * plane * 4);
    const size_t o_cand = take(g.sites * 24);
    const size_t o_meta = take(g.sites);
    const size_t o_sb = take((g.segments + 1) * 4);
    const size_t o_sa = take((g.segments + 1) * 4);
    const size_t o_sr = take(seg_raw_words(g.segments) * 4);
    const size_t o_ent = take(amb_cap * sizeof(AmbEntry) + 64);
    const size_t o_pos = take(amb_cap * 4);
    const size_t o_ext = take(amb_cap * 4);
    const size_t o_two = take(walk_chunks(amb_cap));
    const size_t o_prod = take(producer_bytes(g.h, g.w));
    const size_t o_rows = take(4 * (size_t)g.h * 4);
    const size_t o_out = take(px * 6);
    const size_t o_chg = take(px);
    const size_t o_ctr = take(dev_counters_bytes());
    const size_t o_err = take(16);
    const size_t o_walk = take(walk_scratch_bytes(amb_cap, g_per_wave));
    if (a) {
        char *b = reinterpret_cast<char *>(a->base);
        a->rgbi = (uint16_t *)(b + o_rgbi);
        a->stages = (fx_stage *)(b + o_stages);
        a->aux = (float *)(b + o_aux);
        a->hs = (float *)(b + o_hs);
        a->hwa = (float *)(b + o_hwa);
        a->hwr = (float *)(b + o_hwr);
        a->cand = (double *)(b + o_cand);
        a->meta = (uint8_t *)(b + o_meta);
        a->seg_base = (uint32_t *)(b + o_sb);
        a->seg_amb = (uint32_t *)(b + o_sa);
        a->seg_raw = (uint32_t *)(b + o_sr);
        a->entries = (AmbEntry *)(b + o_ent);
        a->pos = (uint32_t *)(b + o_pos);
        a->extra = (uint32_t *)(b + o_ext);
        a->chunk_two = (uint8_t *)(b + o_two);
        a->producer = (void *)(b + o_prod);
        a->rows = (float *)(b + o_rows);
        a->out = (uint16_t *)(b + o_out);
        a->changed = (uint8_t *)(b + o_chg);
        a->counters = (void *)(b + o_ctr);
        a->err = (uint32_t *)(b + o_err);
        a->walk = (void *)(b + o_walk);
        a->amb_capacity = amb_cap;
    }
    return off;
}

struct Slot {
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;  // k_startup, beside the stencil (greatest priority)
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaStream_t last_stream = nullptr;  // stream of the last device-buffer pass
    cudaEvent_t done = nullptr;
    Arena arena;
    // pinned staging for asynchronous requests
    void *h_in = nullptr;
    size_t h_in_bytes = 0;
    void *h_out = nullptr;
    size_t h_out_bytes = 0;
    void *h_ctr = nullptr;  // DevCounters copy + error word
    // cancel word: pinned host memory the pass's stage gates read through
    // its device mapping (fx_cancel sets it; a new request clears it)
    volatile uint32_t *cancel_host = nullptr;
    uint32_t *cancel_dev = nullptr;
    cudaEvent_t chunk_done[16] = {};  // staged downloads (fx_process)
    // request in flight
    bool busy = false;
    int64_t ticket = -1;
    fx_frame frame{};
    fx_params params{};
    std::vector<fx_stage> stages;
    bool has_stages = false;
    Geometry g{};
    bool stage_score = false, stage_changed = false;  // planes staged in h_out
    // device-buffer request (fx_submit_device): caller-owned device memory
    bool device = false;
    const uint16_t *d_in = nullptr;
    uint16_t *d_out = nullptr;
    float *d_score = nullptr;
    uint8_t *d_changed = nullptr;
};

}  // namespace fx

struct fx_context {
    int device = 0;
    bool profile = false;
    bool parallel_walk = true;
    int walk_wave = 0;  // window segments per wave; 0: g_per_wave (three per SM)
    double walk_sigmas = fx::kDefaultWindowSigmas;  // walk window half-width
    int stencil_rows = 8;  // stencil tile height: 8 (four blocks per SM) or 16 (two)
    double list_per_site = 0.0;  // longest RNG-dependent list per site a pass has needed
    int top_priority = 0;     // the device's greatest launch priority
    bool use_priority = true;  // chain and walk launched at top_priority
    int64_t list_capacity = 0;  // RNG-dependent list entries per frame; 0: sites / 2
    std::vector<std::vector<cudaEvent_t>> pending;  // recorded, not yet read
    std::vector<std::vector<cudaEvent_t>> spare;
    double profile_ms[fx::kProfileStages] = {0};
    int64_t profile_passes = 0;
    float *lut = nullptr;
    uint32_t *high = nullptr, *low = nullptr;
    uint16_t *ident = nullptr;  // emit(lut[v]) for every raw value v
    uint32_t *ident_bad = nullptr;
    bool tables = false;
    std::vector<fx::Slot> slots;
    int64_t next_ticket = 1;
    std::mutex mu;
    char error[512] = {0};
    bool hash_output = false;      // fx_process: SHA-256 of the RGB16 output
    bool digest_valid = false;
    unsigned char digest[32] = {0};
};

namespace fx {

// RNG-dependent list capacity of a frame: the override of
// fx_set_list_capacity when one is set, else sites / 2 (at least 65536).
static int64_t amb_capacity(const fx_context *ctx, const Geometry &g) {
    return ctx->list_capacity > 0 ? ctx->list_capacity : default_amb_capacity(g);
}

// The list capacity of a pass: the frame's own (amb_capacity), raised to
// the longest list per site any pass of this context has needed, so that
// once a frame has overflowed (heavy damage) the next such frame, on any
// slot and at any size, does not.  Never above three channels per site, the
// most a frame can list.  The fx_set_list_capacity override is taken as
// given.
static int64_t pass_capacity(const fx_context *ctx, const Geometry &g) {
    const int64_t cap = amb_capacity(ctx, g);
    if (ctx->list_capacity > 0 || ctx->list_per_site <= 0.0) return cap;
    const int64_t most = 3 * g.sites;
    int64_t learned = (int64_t)std::ceil(ctx->list_per_site * (double)g.sites) + 1;
    if (learned > most) learned = most;
    return learned > cap ? learned : cap;
}

// After an overflow: later passes list at least `cap` channels per
// `g.sites` sites.
static void note_capacity(fx_context *ctx, const Geometry &g, int64_t cap) {
    const double r = (double)cap / (double)g.sites;
    if (r > ctx->list_per_site) ctx->list_per_site = r;
}

static char g_error[512];

static int fail(fx_context *ctx, int code, const char *fmt, ...) {
    char *buf = ctx ? ctx->error : g_error;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, 512, fmt, ap);
    va_end(ap);
    return code;
}

#define FX_CUDA(ctx, call)                                                                 \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail((ctx), FX_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

static int ensure_arena(fx_context *ctx, Slot &s, const Geometry &g, int64_t amb_cap) {
    const size_t need = arena_layout(g, amb_cap, nullptr);
    if (s.arena.base && s.arena.bytes >= need) {
        const size_t bytes = s.arena.bytes;
        void *base = s.arena.base;
        s.arena = Arena();
        s.arena.base = base;
        s.arena.bytes = bytes;
        arena_layout(g, amb_cap, &s.arena);
        return FX_OK;
    }
    if (s.arena.base) {
        cudaStreamSynchronize(s.stream);
        cudaFree(s.arena.base);
        s.arena = Arena();
    }
    void *base = nullptr;
    const cudaError_t e = cudaMalloc(&base, need);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, FX_ERR_OUT_OF_MEMORY, "device allocation of %zu bytes failed: %s", need,
                    cudaGetErrorString(e));
    }
    s.arena.base = base;
    s.arena.bytes = need;
    arena_layout(g, amb_cap, &s.arena);
    return FX_OK;
}

static int check_frame(fx_context *ctx, const fx_params *p, int h, int w) {
    if (!ctx) return FX_ERR_INVALID_ARGUMENT;
    if (!ctx->tables) return fail(ctx, FX_ERR_TABLES, "fx_set_tables has not been called");
    if (!p || h < 1 || w < 1) return fail(ctx, FX_ERR_INVALID_ARGUMENT, "bad frame arguments");
    if ((int64_t)h * w > (int64_t)1 << 30)
        return fail(ctx, FX_ERR_INVALID_ARGUMENT, "frame too large");
    if (p->visible_channel < 0 || p->visible_channel > 2 || p->radius < 1 || p->radius > 4)
        return fail(ctx, FX_ERR_INVALID_ARGUMENT, "bad parameters");
    // streaming.py:391-392 and startup.py:210-213 / fast_cpu/engine.py:148-154
    if (h < 4) return fail(ctx, FX_ERR_GEOMETRY, "streaming startup requires at least four main rows");
    if (p->cross_neighbor && h < 5)
        return fail(ctx, FX_ERR_GEOMETRY, "cross-neighbor startup requires the first five real rows");
    if (p->cross_neighbor && w < 4)
        return fail(ctx, FX_ERR_GEOMETRY, "cross-neighbor startup requires at least four columns");
    if (!isfinite(p->dither_low) || !isfinite(p->dither_high))
        return fail(ctx, FX_ERR_DITHER_INPUT, "dither inputs must be finite");
    for (int c = 0; c < 3; ++c)
        if (!isfinite(p->dither_scales[c]))
            return fail(ctx, FX_ERR_DITHER_INPUT, "dither inputs must be finite");
    return FX_OK;
}

// Enqueue the whole pass for one frame whose input already sits in
// s.arena.rgbi (or `d_in`).  Outputs land in the arena (or `d_out`).
// `cancellable` passes (fx_submit, fx_submit_device) get stage gates that
// read the slot's cancel word.
static int enqueue_pass(fx_context *ctx, Slot &s, const Geometry &g, const fx_params &p,
                        const fx_stage *host_stages, uint32_t rng, const uint16_t *d_in,
                        uint16_t *d_out, uint8_t *d_changed, bool producer_rows,
                        bool cancellable = false) {
    Arena &a = s.arena;
    cudaStream_t st = s.stream;
    Marks marks;
    if (ctx->profile) {
        std::vector<cudaEvent_t> ev;
        if (!ctx->spare.empty()) {
            ev = std::move(ctx->spare.back());
            ctx->spare.pop_back();
        } else {
            ev.resize(kProfileStages + 1);
            for (auto &e : ev) FX_CUDA(ctx, cudaEventCreate(&e));
        }
        ctx->pending.push_back(std::move(ev));
        marks.events = ctx->pending.back().data();
    }
    FX_CUDA(ctx, cudaMemsetAsync(a.err, 0, 16, st));
    marks.mark(0, st);
    if (host_stages) {
        FX_CUDA(ctx, cudaMemcpyAsync(a.stages, host_stages, (g.h + 6) * sizeof(fx_stage),
                                     cudaMemcpyHostToDevice, st));
    } else {
        FX_CUDA(ctx, launch_producer(d_in, g.h, g.w, ctx->lut, a.producer, a.stages,
                                     producer_rows ? a.rows : nullptr, a.err, st,
                                     ctx->use_priority ? ctx->top_priority : 0));
    }
    marks.mark(1, st);
    const uint32_t *cancel = cancellable ? s.cancel_dev : nullptr;
    FX_CUDA(ctx, launch_gate(cancel, a.err, st));
    FX_CUDA(ctx, launch_analysis(d_in, g, ctx->lut, a.stages, p, a.aux, a.hs, a.hwa, a.hwr,
                                 (int64_t)g.prow * g.pitch, a.cand, a.meta, a.err, st, marks,
                                 ctx->stencil_rows, s.side, s.fork, s.join));
    // the walk scratch is sized for g_per_wave; a narrower wave uses part of it
    const int wave = (ctx->walk_wave > 0 && ctx->walk_wave < g_per_wave) ? ctx->walk_wave
                                                                         : g_per_wave;
    WriterBuffers wb{a.seg_base, a.seg_amb, a.seg_raw, a.entries, a.pos, a.extra, a.counters,
                     a.amb_capacity, a.walk, wave, ctx->parallel_walk, ctx->walk_sigmas, cancel,
                     a.chunk_two, ctx->use_priority ? ctx->top_priority : 0};
    FX_CUDA(ctx, launch_writer(g, a.meta, a.cand, d_in, ctx->lut, ctx->high, ctx->low, ctx->ident, a.stages,
                               p, rng, wb, d_out, d_changed, a.err, st, marks));
    return FX_OK;
}

static int error_from_device(fx_context *ctx, uint32_t code) {
    switch (code) {
    case FX_ERR_CANCELLED:
        return fail(ctx, (int)code, "the request was cancelled");
    case FX_ERR_NONFINITE_AUX:
        return fail(ctx, (int)code, "auxiliary score input must be a finite HxW plane");
    case FX_ERR_NONFINITE_WORK:
        return fail(ctx, (int)code, "work RGB must be finite");
    case FX_ERR_COMBINER_INPUT:
        return fail(ctx, (int)code, "combiner inputs must be finite");
    case FX_ERR_DITHER_INPUT:
        return fail(ctx, (int)code, "dither inputs must be finite");
    case FX_ERR_SETTER_ONE:
        return fail(ctx, (int)code, "X3A setter scale cannot equal one");
    case FX_ERR_STAGE_NONFINITE:
        return fail(ctx, (int)code, "stage calibration contains a non-finite value");
    case FX_ERR_ALPHA_ONE_UNBOUND:
        return fail(ctx, (int)code,
                    "alpha==1 requires the runtime-configured auxiliary replacement");
    default:
        return fail(ctx, FX_ERR_INTERNAL, "device consistency check failed (code %u)", code);
    }
}

// Context accessors for entry points defined in other files.
int context_device(const fx_context *ctx) { return ctx->device; }

const float *context_lut(const fx_context *ctx) { return ctx->tables ? ctx->lut : nullptr; }

int context_fail(fx_context *ctx, int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(ctx->error, sizeof(ctx->error), fmt, ap);
    va_end(ap);
    return code;
}

int context_device_error(fx_context *ctx, uint32_t code) { return error_from_device(ctx, code); }

void context_lock(fx_context *ctx) { ctx->mu.lock(); }
void context_unlock(fx_context *ctx) { ctx->mu.unlock(); }

// Counters + error word of the slot, after the stream completed.
static int finish_counters(fx_context *ctx, Slot &s, const void *ctr_copy, uint32_t err,
                           fx_counters *out, bool *overflow) {
    *overflow = false;
    if (err) return error_from_device(ctx, err);
    if ((int64_t)counters_n_amb(ctr_copy) > s.arena.amb_capacity) {
        *overflow = true;
        return FX_OK;
    }
    if (out) counters_to_host(ctr_copy, out);
    return FX_OK;
}

static Slot &slot0(fx_context *ctx) { return ctx->slots[0]; }

// The synchronous entry points run on slot 0; a request of fx_submit /
// fx_submit_device may hold it, and its buffers must not move under it.
static int check_slot0_free(fx_context *ctx) {
    if (slot0(ctx).busy)
        return fail(ctx, FX_PENDING, "slot 0 holds a request in flight: wait for it first");
    return FX_OK;
}

static int ensure_slots(fx_context *ctx, int n) {
    while ((int)ctx->slots.size() < n) {
        ctx->slots.emplace_back();
        Slot &s = ctx->slots.back();
        FX_CUDA(ctx, cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
        FX_CUDA(ctx, cudaStreamCreateWithPriority(&s.side, cudaStreamNonBlocking,
                                                  ctx->top_priority));
        FX_CUDA(ctx, cudaEventCreateWithFlags(&s.fork, cudaEventDisableTiming));
        FX_CUDA(ctx, cudaEventCreateWithFlags(&s.join, cudaEventDisableTiming));
        FX_CUDA(ctx, cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
        FX_CUDA(ctx, cudaMallocHost(&s.h_ctr, dev_counters_bytes() + 64));  // + err + count
        void *word = nullptr;
        FX_CUDA(ctx, cudaHostAlloc(&word, 64, cudaHostAllocMapped));
        s.cancel_host = static_cast<volatile uint32_t *>(word);
        *s.cancel_host = 0u;
        void *dev = nullptr;
        FX_CUDA(ctx, cudaHostGetDevicePointer(&dev, word, 0));
        s.cancel_dev = static_cast<uint32_t *>(dev);
    }
    return FX_OK;
}

// Synchronous pass over device buffers on the slot's stream, with the
// amb-capacity retry.
static int run_device(fx_context *ctx, Slot &s, const Geometry &g, const fx_params &p,
                      const fx_stage *stages, uint32_t rng, const uint16_t *d_in, uint16_t *d_out,
                      uint8_t *d_changed, fx_counters *counters, bool producer_rows) {
    int64_t cap = pass_capacity(ctx, g);
    for (int attempt = 0; attempt < 2; ++attempt) {
        // keep caller-side device pointers stable: the arena may move only
        // when the input/outputs live in it
        int rc = ensure_arena(ctx, s, g, cap);
        if (rc) return rc;
        const uint16_t *in = d_in ? d_in : s.arena.rgbi;
        uint16_t *out = d_out ? d_out : s.arena.out;
        uint8_t *chg = d_changed ? d_changed : s.arena.changed;
        rc = enqueue_pass(ctx, s, g, p, stages, rng, in, out, chg, producer_rows);
        if (rc) return rc;
        char *hc = reinterpret_cast<char *>(s.h_ctr);
        FX_CUDA(ctx, cudaMemcpyAsync(hc, s.arena.counters, dev_counters_bytes(),
                                     cudaMemcpyDeviceToHost, s.stream));
        FX_CUDA(ctx, cudaMemcpyAsync(hc + dev_counters_bytes(), s.arena.err, 4,
                                     cudaMemcpyDeviceToHost, s.stream));
        FX_CUDA(ctx, cudaStreamSynchronize(s.stream));
        uint32_t err;
        std::memcpy(&err, hc + dev_counters_bytes(), 4);
        bool overflow;
        rc = finish_counters(ctx, s, hc, err, counters, &overflow);
        if (rc) return rc;
        if (!overflow) {
            if (counters) counters->capacity_reruns = attempt;
            return FX_OK;
        }
        cap = (int64_t)counters_n_amb(hc) + 1024;
        note_capacity(ctx, g, cap);
        if (!d_in) return fail(ctx, FX_ERR_INTERNAL, "amb capacity retry needs the input");
    }
    return fail(ctx, FX_ERR_INTERNAL, "amb capacity retry failed");
}

}  // namespace fx

using namespace fx;

extern "C" {

FX_API int fx_version(void) { return FX_ABI_VERSION; }

FX_API int fx_device_check(int device, char *reason, size_t reason_len) {
    auto say = [&](int code, const char *msg) {
        if (reason && reason_len) snprintf(reason, reason_len, "%s", msg);
        return code;
    };
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return say(FX_ERR_NO_DEVICE, "no CUDA device is visible");
    }
    if (device < 0 || device >= count) return say(FX_ERR_NO_DEVICE, "device index out of range");
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess)
        return say(FX_ERR_NO_DEVICE, "cannot query the CUDA device");
    if (prop.major != 10 || prop.minor != 0) {
        char buf[384];
        snprintf(buf, sizeof(buf), "device %s is sm_%d%d; this library is built for sm_100a",
                 prop.name, prop.major, prop.minor);
        return say(FX_ERR_UNSUPPORTED_DEVICE, buf);
    }
    return say(FX_OK, "ok");
}

FX_API int fx_context_create(int device, fx_context **out) {
    if (!out) return FX_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    char reason[160];
    const int rc = fx_device_check(device, reason, sizeof(reason));
    if (rc) return fail(nullptr, rc, "%s", reason);
    fx_context *ctx = new fx_context();
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete ctx;
        return fail(nullptr, FX_ERR_CUDA, "cudaSetDevice failed");
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess &&
        sms > 0)
        g_per_wave = walk_per_wave(sms);
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess)
        ctx->top_priority = greatest;
    if (analysis_init() != cudaSuccess || ensure_slots(ctx, 1) != FX_OK ||
        cudaMalloc(&ctx->lut, 65536 * 4) != cudaSuccess ||
        cudaMalloc(&ctx->high, 256 * 4) != cudaSuccess ||
        cudaMalloc(&ctx->low, 256 * 4) != cudaSuccess ||
        cudaMalloc(&ctx->ident, 65536 * 2) != cudaSuccess ||
        cudaMalloc(&ctx->ident_bad, 4) != cudaSuccess) {
        cudaGetLastError();
        fx_context_destroy(ctx);
        return fail(nullptr, FX_ERR_CUDA, "context initialisation failed");
    }
    *out = ctx;
    return FX_OK;
}

FX_API void fx_context_destroy(fx_context *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    for (Slot &s : ctx->slots) {
        if (s.stream) cudaStreamSynchronize(s.stream);
        if (s.arena.base) cudaFree(s.arena.base);
        if (s.h_in) cudaFreeHost(s.h_in);
        if (s.h_out) cudaFreeHost(s.h_out);
        if (s.h_ctr) cudaFreeHost(s.h_ctr);
        if (s.cancel_host) cudaFreeHost(const_cast<uint32_t *>(s.cancel_host));
        if (s.done) cudaEventDestroy(s.done);
        if (s.fork) cudaEventDestroy(s.fork);
        if (s.join) cudaEventDestroy(s.join);
        for (cudaEvent_t e : s.chunk_done)
            if (e) cudaEventDestroy(e);
        if (s.side) {
            cudaStreamSynchronize(s.side);
            cudaStreamDestroy(s.side);
        }
        if (s.stream) cudaStreamDestroy(s.stream);
    }
    for (auto &v : ctx->pending)
        for (auto e : v) cudaEventDestroy(e);
    for (auto &v : ctx->spare)
        for (auto e : v) cudaEventDestroy(e);
    if (ctx->lut) cudaFree(ctx->lut);
    if (ctx->high) cudaFree(ctx->high);
    if (ctx->low) cudaFree(ctx->low);
    if (ctx->ident) cudaFree(ctx->ident);
    if (ctx->ident_bad) cudaFree(ctx->ident_bad);
    delete ctx;
}

FX_API int fx_last_error(const fx_context *ctx, char *buf, size_t len) {
    if (!buf || !len) return FX_ERR_INVALID_ARGUMENT;
    snprintf(buf, len, "%s", ctx ? ctx->error : g_error);
    return FX_OK;
}

FX_API int fx_set_tables(fx_context *ctx, const float *lut, const uint32_t *high,
                         const uint32_t *low) {
    if (!ctx || !lut || !high || !low) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    FX_CUDA(ctx, cudaMemcpy(ctx->lut, lut, 65536 * 4, cudaMemcpyHostToDevice));
    FX_CUDA(ctx, cudaMemcpy(ctx->high, high, 256 * 4, cudaMemcpyHostToDevice));
    FX_CUDA(ctx, cudaMemcpy(ctx->low, low, 256 * 4, cudaMemcpyHostToDevice));
    FX_CUDA(ctx, writer_identity_table(ctx->lut, ctx->high, ctx->low, ctx->ident, ctx->ident_bad, 0));
    uint32_t bad = 0;
    FX_CUDA(ctx, cudaMemcpy(&bad, ctx->ident_bad, 4, cudaMemcpyDeviceToHost));
    if (bad) {
        ctx->tables = false;
        return fail(ctx, FX_ERR_NONFINITE_WORK, "work RGB must be finite: the LUT holds a non-finite value");
    }
    ctx->tables = true;
    return FX_OK;
}

FX_API int fx_reduce_prepass(const uint16_t *prepass, int32_t h, int32_t w, const float *lut,
                             uint8_t payload[64], int64_t *valid, int64_t *tiles) {
    if (!prepass || !lut || !payload || h < 1 || w < 1) return FX_ERR_INVALID_ARGUMENT;
    return host_reduce_prepass(prepass, h, w, lut, payload, valid, tiles);
}

FX_API int fx_stage_table(int32_t h, const float *p1, const float *p2, const float *mv,
                          const float *mi, float factor_b, fx_stage *stages) {
    if (h < 1 || !p1 || !p2 || !mv || !mi || !stages) return FX_ERR_INVALID_ARGUMENT;
    return host_stage_table(h, p1, p2, mv, mi, factor_b, stages);
}

FX_API int fx_producer_rows(fx_context *ctx, const uint16_t *main_rgbi, int32_t h, int32_t w,
                            float *p1, float *p2, float *mv, float *mi) {
    if (!ctx || !main_rgbi || h < 1 || w < 8 || !p1 || !p2 || !mv || !mi)
        return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    if (!ctx->tables) return fail(ctx, FX_ERR_TABLES, "fx_set_tables has not been called");
    int rc = check_slot0_free(ctx);
    if (rc) return rc;
    Slot &s = slot0(ctx);
    const Geometry g = make_geometry(h, w);
    rc = ensure_arena(ctx, s, g, default_amb_capacity(g));
    if (rc) return rc;
    FX_CUDA(ctx, cudaMemsetAsync(s.arena.err, 0, 16, s.stream));
    FX_CUDA(ctx, cudaMemcpyAsync(s.arena.rgbi, main_rgbi, (size_t)h * w * 8,
                                 cudaMemcpyHostToDevice, s.stream));
    FX_CUDA(ctx, launch_producer(s.arena.rgbi, h, w, ctx->lut, s.arena.producer, s.arena.stages,
                                 s.arena.rows, s.arena.err, s.stream));
    std::vector<float> rows(4 * (size_t)h);
    uint32_t err = 0;
    FX_CUDA(ctx, cudaMemcpyAsync(rows.data(), s.arena.rows, rows.size() * 4,
                                 cudaMemcpyDeviceToHost, s.stream));
    FX_CUDA(ctx, cudaMemcpyAsync(&err, s.arena.err, 4, cudaMemcpyDeviceToHost, s.stream));
    FX_CUDA(ctx, cudaStreamSynchronize(s.stream));
    std::memcpy(p1, rows.data(), h * 4);
    std::memcpy(p2, rows.data() + h, h * 4);
    std::memcpy(mv, rows.data() + 2 * (size_t)h, h * 4);
    std::memcpy(mi, rows.data() + 3 * (size_t)h, h * 4);
    if (err && err != FX_ERR_SETTER_ONE && err != FX_ERR_STAGE_NONFINITE)
        return error_from_device(ctx, err);
    return FX_OK;
}

// Host <-> device copies of caller (pageable) buffers through the slot's
// pinned staging: the frame moves in chunks, host threads copying one chunk
// between the caller's buffer and pinned memory while the DMA engine moves
// another.
constexpr int kCopyChunks = 16;

static int copy_threads() {
    const unsigned n = std::thread::hardware_concurrency();
    return n >= 8 ? 8 : (n > 0 ? (int)n : 1);
}

// memcpy of a large buffer split over the copy threads (one host thread
// cannot saturate the memory bus; frames here are 100-200 MB).
static void parallel_memcpy(void *dst, const void *src, size_t bytes) {
    const int nt = bytes < ((size_t)8 << 20) ? 1 : copy_threads();
    if (nt == 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    const size_t part = (bytes + nt - 1) / nt;
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([=] {
            const size_t off = (size_t)t * part;
            if (off < bytes)
                std::memcpy(static_cast<char *>(dst) + off, static_cast<const char *>(src) + off,
                            std::min(part, bytes - off));
        });
    for (std::thread &th : pool) th.join();
}

static int ensure_pinned(fx_context *ctx, void **buf, size_t *have, size_t need) {
    if (*have >= need) return FX_OK;
    if (*buf) cudaFreeHost(*buf);
    *buf = nullptr;
    *have = 0;
    FX_CUDA(ctx, cudaMallocHost(buf, need));
    *have = need;
    return FX_OK;
}

static int staged_upload(fx_context *ctx, Slot &s, void *d_dst, const void *h_src, size_t bytes) {
    int rc = ensure_pinned(ctx, &s.h_in, &s.h_in_bytes, bytes);
    if (rc) return rc;
    const size_t chunk = (bytes + kCopyChunks - 1) / kCopyChunks;
    const int nt = copy_threads();
    std::vector<cudaError_t> errs(nt, cudaSuccess);
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&, t] {
            for (int k = t; k < kCopyChunks; k += nt) {
                const size_t off = (size_t)k * chunk;
                if (off >= bytes) break;
                const size_t len = std::min(chunk, bytes - off);
                std::memcpy(static_cast<char *>(s.h_in) + off,
                            static_cast<const char *>(h_src) + off, len);
                const cudaError_t e = cudaMemcpyAsync(static_cast<char *>(d_dst) + off,
                                                      static_cast<char *>(s.h_in) + off, len,
                                                      cudaMemcpyHostToDevice, s.stream);
                if (e != cudaSuccess) errs[t] = e;
            }
        });
    for (std::thread &th : pool) th.join();
    for (cudaError_t e : errs)
        if (e != cudaSuccess) return fail(ctx, FX_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
    return FX_OK;
}

// SHA-256 of `bytes` of pinned memory, fed chunk by chunk as each chunk's
// device-to-host copy completes (chunk k's event), so hashing overlaps the
// remaining copies.  Returns false when a copy or the digest failed.
static bool hash_chunks(Slot &s, const char *pinned, size_t bytes, size_t chunk,
                        unsigned char *digest) {
    EVP_MD_CTX *md = EVP_MD_CTX_new();
    if (!md) return false;
    bool ok = EVP_DigestInit_ex(md, EVP_sha256(), nullptr) == 1;
    for (int k = 0; ok && k < kCopyChunks; ++k) {
        const size_t off = (size_t)k * chunk;
        if (off >= bytes) break;
        ok = cudaEventSynchronize(s.chunk_done[k]) == cudaSuccess &&
             EVP_DigestUpdate(md, pinned + off, std::min(chunk, bytes - off)) == 1;
    }
    unsigned int len = 0;
    ok = ok && EVP_DigestFinal_ex(md, digest, &len) == 1 && len == 32;
    EVP_MD_CTX_free(md);
    return ok;
}

static int staged_download(fx_context *ctx, Slot &s, void *h_dst, const void *d_src,
                           size_t bytes, unsigned char *digest = nullptr) {
    int rc = ensure_pinned(ctx, &s.h_out, &s.h_out_bytes, bytes);
    if (rc) return rc;
    const size_t chunk = (bytes + kCopyChunks - 1) / kCopyChunks;
    for (int k = 0; k < kCopyChunks; ++k) {
        const size_t off = (size_t)k * chunk;
        if (off >= bytes) break;
        if (!s.chunk_done[k])
            FX_CUDA(ctx, cudaEventCreateWithFlags(&s.chunk_done[k], cudaEventDisableTiming));
        FX_CUDA(ctx, cudaMemcpyAsync(static_cast<char *>(s.h_out) + off,
                                     static_cast<const char *>(d_src) + off,
                                     std::min(chunk, bytes - off), cudaMemcpyDeviceToHost,
                                     s.stream));
        FX_CUDA(ctx, cudaEventRecord(s.chunk_done[k], s.stream));
    }
    const int nt = copy_threads();
    std::vector<cudaError_t> errs(nt, cudaSuccess);
    std::vector<std::thread> pool;
    bool hashed = true;
    if (digest)
        pool.emplace_back([&] {
            hashed = hash_chunks(s, static_cast<const char *>(s.h_out), bytes, chunk, digest);
        });
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&, t] {
            for (int k = t; k < kCopyChunks; k += nt) {
                const size_t off = (size_t)k * chunk;
                if (off >= bytes) break;
                const cudaError_t e = cudaEventSynchronize(s.chunk_done[k]);
                if (e != cudaSuccess) {
                    errs[t] = e;
                    continue;
                }
                std::memcpy(static_cast<char *>(h_dst) + off,
                            static_cast<const char *>(s.h_out) + off, std::min(chunk, bytes - off));
            }
        });
    for (std::thread &th : pool) th.join();
    for (cudaError_t e : errs)
        if (e != cudaSuccess) return fail(ctx, FX_ERR_CUDA, "download: %s", cudaGetErrorString(e));
    if (!hashed) return fail(ctx, FX_ERR_INTERNAL, "output SHA-256 failed");
    return FX_OK;
}

FX_API int fx_process(fx_context *ctx, const fx_frame *f, fx_counters *counters) {
    if (!ctx || !f || !f->main_rgbi || !f->rgb_out) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    int rc = check_frame(ctx, f->params, f->height, f->width);
    if (rc) return rc;
    if (!f->stages && f->width < 8)
        return fail(ctx, FX_ERR_GEOMETRY, "main RGBI frame has no complete producer cell");
    rc = check_slot0_free(ctx);
    if (rc) return rc;
    Slot &s = slot0(ctx);
    const Geometry g = make_geometry(f->height, f->width);
    const size_t px = (size_t)g.h * g.w;
    int64_t cap = pass_capacity(ctx, g);
    for (int attempt = 0; attempt < 2; ++attempt) {
        rc = ensure_arena(ctx, s, g, cap);
        if (rc) return rc;
        rc = staged_upload(ctx, s, s.arena.rgbi, f->main_rgbi, px * 8);
        if (rc) return rc;
        rc = enqueue_pass(ctx, s, g, *f->params, f->stages, f->rng_state, s.arena.rgbi,
                          s.arena.out, s.arena.changed, false);
        if (rc) return rc;
        char *hc = reinterpret_cast<char *>(s.h_ctr);
        FX_CUDA(ctx, cudaMemcpyAsync(hc, s.arena.counters, dev_counters_bytes(),
                                     cudaMemcpyDeviceToHost, s.stream));
        FX_CUDA(ctx, cudaMemcpyAsync(hc + dev_counters_bytes(), s.arena.err, 4,
                                     cudaMemcpyDeviceToHost, s.stream));
        FX_CUDA(ctx, cudaStreamSynchronize(s.stream));
        uint32_t err;
        std::memcpy(&err, hc + dev_counters_bytes(), 4);
        bool overflow;
        rc = finish_counters(ctx, s, hc, err, counters, &overflow);
        if (rc) return rc;
        if (overflow) {
            cap = (int64_t)counters_n_amb(hc) + 1024;
            note_capacity(ctx, g, cap);
            continue;
        }
        if (counters) counters->capacity_reruns = attempt;
        ctx->digest_valid = false;
        rc = staged_download(ctx, s, f->rgb_out, s.arena.out, px * 6,
                             ctx->hash_output ? ctx->digest : nullptr);
        if (rc) return rc;
        ctx->digest_valid = ctx->hash_output;
        if (f->score_out)
            FX_CUDA(ctx, cudaMemcpy2D(f->score_out, (size_t)g.w * 4,
                                      s.arena.hs + g.padded_index(0, 0), (size_t)g.pitch * 4,
                                      (size_t)g.w * 4, g.h, cudaMemcpyDeviceToHost));
        if (f->changed_out)
            FX_CUDA(ctx, cudaMemcpy(f->changed_out, s.arena.changed, px, cudaMemcpyDeviceToHost));
        return FX_OK;
    }
    return fail(ctx, FX_ERR_INTERNAL, "amb capacity retry failed");
}

FX_API int fx_process_device(fx_context *ctx, const uint16_t *d_rgbi, int32_t h, int32_t w,
                             const fx_params *params, const fx_stage *stages, uint32_t rng,
                             uint16_t *d_out, float *d_score, uint8_t *d_changed, void *stream,
                             fx_counters *counters) {
    if (!ctx || !d_rgbi || !d_out) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    int rc = check_frame(ctx, params, h, w);
    if (rc) return rc;
    if (!stages && w < 8)
        return fail(ctx, FX_ERR_GEOMETRY, "main RGBI frame has no complete producer cell");
    rc = check_slot0_free(ctx);
    if (rc) return rc;
    Slot &s = slot0(ctx);
    cudaStream_t user = reinterpret_cast<cudaStream_t>(stream);
    cudaStream_t saved = s.stream;
    if (user) s.stream = user;
    const Geometry g = make_geometry(h, w);
    if (counters) {
        rc = run_device(ctx, s, g, *params, stages, rng, d_rgbi, d_out, d_changed, counters, false);
    } else {
        rc = ensure_arena(ctx, s, g, pass_capacity(ctx, g));
        if (!rc) rc = enqueue_pass(ctx, s, g, *params, stages, rng, d_rgbi, d_out, d_changed, false);
    }
    s.last_stream = s.stream;
    if (!rc && d_score)
        rc = cudaMemcpy2DAsync(d_score, (size_t)w * 4, s.arena.hs + g.padded_index(0, 0),
                               (size_t)g.pitch * 4, (size_t)w * 4, h, cudaMemcpyDeviceToDevice,
                               s.stream) == cudaSuccess
                 ? FX_OK
                 : fail(ctx, FX_ERR_CUDA, "score copy failed");
    s.stream = saved;
    return rc;
}

FX_API int fx_sync_counters(fx_context *ctx, fx_counters *counters) {
    if (!ctx || !counters) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    Slot &s = slot0(ctx);
    cudaStream_t st = s.last_stream ? s.last_stream : s.stream;
    char *hc = reinterpret_cast<char *>(s.h_ctr);
    FX_CUDA(ctx, cudaMemcpyAsync(hc, s.arena.counters, dev_counters_bytes(),
                                 cudaMemcpyDeviceToHost, st));
    FX_CUDA(ctx, cudaMemcpyAsync(hc + dev_counters_bytes(), s.arena.err, 4,
                                 cudaMemcpyDeviceToHost, st));
    FX_CUDA(ctx, cudaStreamSynchronize(st));
    uint32_t err;
    std::memcpy(&err, hc + dev_counters_bytes(), 4);
    bool overflow;
    const int rc = finish_counters(ctx, s, hc, err, counters, &overflow);
    if (rc) return rc;
    if (overflow) return fail(ctx, FX_ERR_INTERNAL, "amb capacity exceeded; rerun with counters");
    return FX_OK;
}

FX_API int fx_set_parallel_walk(fx_context *ctx, int enable) {
    if (!ctx) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->parallel_walk = enable != 0;
    return FX_OK;
}

FX_API int fx_set_output_digest(fx_context *ctx, int enable) {
    if (!ctx) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->hash_output = enable != 0;
    ctx->digest_valid = false;
    return FX_OK;
}

FX_API int fx_output_digest(fx_context *ctx, uint8_t *digest) {
    if (!ctx || !digest) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (!ctx->digest_valid)
        return fail(ctx, FX_ERR_INVALID_ARGUMENT, "no output digest: enable it before fx_process");
    std::memcpy(digest, ctx->digest, 32);
    return FX_OK;
}

FX_API int fx_set_launch_priority(fx_context *ctx, int enable) {
    if (!ctx) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->use_priority = enable != 0;
    return FX_OK;
}

FX_API int fx_set_walk_wave(fx_context *ctx, int32_t segments) {
    if (!ctx || segments < 0) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->walk_wave = segments;
    return FX_OK;
}

FX_API int fx_reserve_frames(fx_context *ctx, int32_t max_height, int32_t max_width) {
    if (!ctx || max_height < 1 || max_width < 1) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    if ((int64_t)max_height * max_width > (int64_t)1 << 30)
        return fail(ctx, FX_ERR_INVALID_ARGUMENT, "frame too large");
    // every buffer of the layout grows with the height and the width, so the
    // arena of the largest frame holds any frame within both bounds
    const Geometry g = make_geometry(max_height, max_width);
    for (Slot &s : ctx->slots) {
        if (s.busy) return fail(ctx, FX_ERR_INVALID_ARGUMENT, "a slot is busy: reserve first");
        const int64_t cap = pass_capacity(ctx, g);
        const int rc = ensure_arena(ctx, s, g, cap);
        if (rc) return rc;
    }
    return FX_OK;
}

FX_API int fx_reserve_slots(fx_context *ctx, int32_t count, int32_t max_height,
                            int32_t max_width) {
    if (!ctx || count < 1 || count > 64 || max_height < 1 || max_width < 1)
        return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    if ((int64_t)max_height * max_width > (int64_t)1 << 30)
        return fail(ctx, FX_ERR_INVALID_ARGUMENT, "frame too large");
    int rc = ensure_slots(ctx, count);
    if (rc) return rc;
    const Geometry g = make_geometry(max_height, max_width);
    for (int k = 0; k < count; ++k) {
        Slot &s = ctx->slots[k];
        if (s.busy) return fail(ctx, FX_ERR_INVALID_ARGUMENT, "a slot is busy: reserve first");
        const int64_t cap = pass_capacity(ctx, g);
        rc = ensure_arena(ctx, s, g, cap);
        if (rc) return rc;
    }
    return FX_OK;
}

FX_API int fx_release_idle_slots(fx_context *ctx, int64_t *released_bytes) {
    if (!ctx) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    int64_t freed = 0;
    for (Slot &s : ctx->slots) {
        if (s.busy || !s.arena.base) continue;
        FX_CUDA(ctx, cudaStreamSynchronize(s.stream));
        FX_CUDA(ctx, cudaFree(s.arena.base));
        freed += (int64_t)s.arena.bytes;
        s.arena = Arena();
    }
    if (released_bytes) *released_bytes = freed;
    return FX_OK;
}

FX_API int fx_set_slots(fx_context *ctx, int32_t slots) {
    if (!ctx || slots < 1 || slots > 64) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    return ensure_slots(ctx, slots);
}

// Device-to-host copies of a host-buffer request's results into the slot's
// pinned staging (h_out: RGB16 at 0, score at 6 px, changed at 10 px), then
// its counters and error word.
static int stage_host_results(fx_context *ctx, Slot &s) {
    const Geometry &g = s.g;
    const size_t px = (size_t)g.h * g.w;
    char *ho = reinterpret_cast<char *>(s.h_out);
    FX_CUDA(ctx, cudaMemcpyAsync(ho, s.arena.out, px * 6, cudaMemcpyDeviceToHost, s.stream));
    if (s.stage_score)
        FX_CUDA(ctx, cudaMemcpy2DAsync(ho + px * 6, (size_t)g.w * 4,
                                       s.arena.hs + g.padded_index(0, 0), (size_t)g.pitch * 4,
                                       (size_t)g.w * 4, g.h, cudaMemcpyDeviceToHost, s.stream));
    if (s.stage_changed)
        FX_CUDA(ctx, cudaMemcpyAsync(ho + px * 10, s.arena.changed, px, cudaMemcpyDeviceToHost,
                                     s.stream));
    char *hc = reinterpret_cast<char *>(s.h_ctr);
    FX_CUDA(ctx, cudaMemcpyAsync(hc, s.arena.counters, dev_counters_bytes(),
                                 cudaMemcpyDeviceToHost, s.stream));
    FX_CUDA(ctx, cudaMemcpyAsync(hc + dev_counters_bytes(), s.arena.err, 4,
                                 cudaMemcpyDeviceToHost, s.stream));
    return FX_OK;
}

// A free slot for a frame of geometry g: the one with the smallest arena
// that already holds the frame, else one without an arena, else the free
// slot with the largest arena (which then grows: a cudaFree, which waits
// for the whole device).
static Slot *free_slot(fx_context *ctx, const Geometry &g) {
    Slot *fit = nullptr, *empty = nullptr, *largest = nullptr;
    for (Slot &s : ctx->slots) {
        if (s.busy) continue;
        if (!s.arena.base) {
            if (!empty) empty = &s;
            continue;
        }
        const size_t need = arena_layout(g, pass_capacity(ctx, g), nullptr);
        if (s.arena.bytes >= need && (!fit || s.arena.bytes < fit->arena.bytes)) fit = &s;
        if (!largest || s.arena.bytes > largest->arena.bytes) largest = &s;
    }
    return fit ? fit : (empty ? empty : largest);
}

FX_API int fx_submit(fx_context *ctx, const fx_frame *f, int64_t *ticket) {
    if (!ctx || !f || !f->main_rgbi || !ticket) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    int rc = check_frame(ctx, f->params, f->height, f->width);
    if (rc) return rc;
    if (!f->stages && f->width < 8)
        return fail(ctx, FX_ERR_GEOMETRY, "main RGBI frame has no complete producer cell");
    const Geometry g = make_geometry(f->height, f->width);
    Slot *slot = free_slot(ctx, g);
    if (!slot) return fail(ctx, FX_PENDING, "no free slot");
    Slot &s = *slot;
    const size_t px = (size_t)g.h * g.w;
    rc = ensure_arena(ctx, s, g, pass_capacity(ctx, g));
    if (rc) return rc;
    const size_t in_bytes = px * 8;
    const size_t out_bytes = px * 6 + px * 4 + px;
    if (s.h_in_bytes < in_bytes) {
        if (s.h_in) cudaFreeHost(s.h_in);
        s.h_in = nullptr;
        s.h_in_bytes = 0;
        FX_CUDA(ctx, cudaMallocHost(&s.h_in, in_bytes));
        s.h_in_bytes = in_bytes;
    }
    if (s.h_out_bytes < out_bytes) {
        if (s.h_out) cudaFreeHost(s.h_out);
        s.h_out = nullptr;
        s.h_out_bytes = 0;
        FX_CUDA(ctx, cudaMallocHost(&s.h_out, out_bytes));
        s.h_out_bytes = out_bytes;
    }
    parallel_memcpy(s.h_in, f->main_rgbi, in_bytes);
    s.device = false;
    s.frame = *f;
    s.params = *f->params;
    s.frame.params = &s.params;
    s.has_stages = f->stages != nullptr;
    if (s.has_stages) s.stages.assign(f->stages, f->stages + (g.h + 6));
    s.g = g;
    // no output buffer now: every result stays staged for fx_fetch
    const bool deferred = f->rgb_out == nullptr;
    s.stage_score = deferred || f->score_out;
    s.stage_changed = deferred || f->changed_out;
    *s.cancel_host = 0u;
    FX_CUDA(ctx, cudaMemcpyAsync(s.arena.rgbi, s.h_in, in_bytes, cudaMemcpyHostToDevice, s.stream));
    rc = enqueue_pass(ctx, s, g, s.params, s.has_stages ? s.stages.data() : nullptr,
                      f->rng_state, s.arena.rgbi, s.arena.out, s.arena.changed, false, true);
    if (rc) return rc;
    rc = stage_host_results(ctx, s);
    if (rc) return rc;
    FX_CUDA(ctx, cudaEventRecord(s.done, s.stream));
    s.busy = true;
    s.ticket = ctx->next_ticket++;
    *ticket = s.ticket;
    return FX_OK;
}

// Score plane and counters of a device-buffer request, enqueued on the
// slot's stream after its pass.
static int copy_device_results(fx_context *ctx, Slot &s) {
    const Geometry &g = s.g;
    if (s.d_score)
        FX_CUDA(ctx, cudaMemcpy2DAsync(s.d_score, (size_t)g.w * 4, s.arena.hs + g.padded_index(0, 0),
                                       (size_t)g.pitch * 4, (size_t)g.w * 4, g.h,
                                       cudaMemcpyDeviceToDevice, s.stream));
    char *hc = reinterpret_cast<char *>(s.h_ctr);
    FX_CUDA(ctx, cudaMemcpyAsync(hc, s.arena.counters, dev_counters_bytes(),
                                 cudaMemcpyDeviceToHost, s.stream));
    FX_CUDA(ctx, cudaMemcpyAsync(hc + dev_counters_bytes(), s.arena.err, 4,
                                 cudaMemcpyDeviceToHost, s.stream));
    return FX_OK;
}

FX_API int fx_submit_device(fx_context *ctx, const uint16_t *d_rgbi, int32_t h, int32_t w,
                            const fx_params *params, const fx_stage *stages, uint32_t rng,
                            uint16_t *d_out, float *d_score, uint8_t *d_changed,
                            int64_t *ticket) {
    if (!ctx || !d_rgbi || !d_out || !ticket) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    int rc = check_frame(ctx, params, h, w);
    if (rc) return rc;
    if (!stages && w < 8)
        return fail(ctx, FX_ERR_GEOMETRY, "main RGBI frame has no complete producer cell");
    const Geometry g = make_geometry(h, w);
    Slot *slot = free_slot(ctx, g);
    if (!slot) return fail(ctx, FX_PENDING, "no free slot");
    Slot &s = *slot;
    rc = ensure_arena(ctx, s, g, pass_capacity(ctx, g));
    if (rc) return rc;
    s.frame = fx_frame{};
    s.frame.height = h;
    s.frame.width = w;
    s.frame.rng_state = rng;
    s.params = *params;
    s.frame.params = &s.params;
    s.has_stages = stages != nullptr;
    if (s.has_stages) s.stages.assign(stages, stages + (g.h + 6));
    s.g = g;
    s.device = true;
    s.d_in = d_rgbi;
    s.d_out = d_out;
    s.d_score = d_score;
    s.d_changed = d_changed;
    *s.cancel_host = 0u;
    rc = enqueue_pass(ctx, s, g, s.params, s.has_stages ? s.stages.data() : nullptr, rng, d_rgbi,
                      d_out, d_changed, false, true);
    if (rc) return rc;
    rc = copy_device_results(ctx, s);
    if (rc) return rc;
    FX_CUDA(ctx, cudaEventRecord(s.done, s.stream));
    s.busy = true;
    s.ticket = ctx->next_ticket++;
    *ticket = s.ticket;
    return FX_OK;
}

static Slot *find_ticket(fx_context *ctx, int64_t ticket) {
    for (Slot &s : ctx->slots)
        if (s.busy && s.ticket == ticket) return &s;
    return nullptr;
}

FX_API int fx_poll(fx_context *ctx, int64_t ticket) {
    if (!ctx) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    Slot *s = find_ticket(ctx, ticket);
    if (!s) return fail(ctx, FX_ERR_INVALID_ARGUMENT, "unknown ticket");
    const cudaError_t e = cudaEventQuery(s->done);
    if (e == cudaErrorNotReady) return FX_PENDING;
    if (e != cudaSuccess) return fail(ctx, FX_ERR_CUDA, "%s", cudaGetErrorString(e));
    return FX_OK;
}

FX_API int fx_cancel(fx_context *ctx, int64_t ticket) {
    if (!ctx) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    Slot *s = find_ticket(ctx, ticket);
    if (!s) return fail(ctx, FX_ERR_INVALID_ARGUMENT, "unknown ticket");
    *s->cancel_host = 1u;  // read by the pass's next stage gate
    return FX_OK;
}

// Where fx_fetch puts a host request's results (NULL: not wanted).
struct FetchTargets {
    uint16_t *rgb;
    float *score;
    uint8_t *at_floor;
    uint8_t *changed;
};

// The pass of slot s completed with more RNG-dependent channels than its
// list held (rare): rerun it synchronously with room for all of them.
static int rerun_with_capacity(fx_context *ctx, Slot &s, fx_counters *counters) {
    char *hc = reinterpret_cast<char *>(s.h_ctr);
    const int64_t cap = (int64_t)counters_n_amb(hc) + 1024;
    note_capacity(ctx, s.g, cap);
    int rc = ensure_arena(ctx, s, s.g, cap);
    if (rc) return rc;
    if (s.device) {
        rc = enqueue_pass(ctx, s, s.g, s.params, s.has_stages ? s.stages.data() : nullptr,
                          s.frame.rng_state, s.d_in, s.d_out, s.d_changed, false, true);
        if (!rc) rc = copy_device_results(ctx, s);
    } else {
        const size_t px = (size_t)s.g.h * s.g.w;
        FX_CUDA(ctx, cudaMemcpyAsync(s.arena.rgbi, s.h_in, px * 8, cudaMemcpyHostToDevice,
                                     s.stream));
        rc = enqueue_pass(ctx, s, s.g, s.params, s.has_stages ? s.stages.data() : nullptr,
                          s.frame.rng_state, s.arena.rgbi, s.arena.out, s.arena.changed, false,
                          true);
        if (!rc) rc = stage_host_results(ctx, s);
    }
    if (rc) return rc;
    if (cudaStreamSynchronize(s.stream) != cudaSuccess)
        return fail(ctx, FX_ERR_CUDA, "capacity rerun failed");
    uint32_t err;
    std::memcpy(&err, hc + dev_counters_bytes(), 4);
    bool overflow;
    rc = finish_counters(ctx, s, hc, err, counters, &overflow);
    if (!rc && overflow) rc = fail(ctx, FX_ERR_INTERNAL, "capacity rerun overflowed");
    if (!rc && counters) counters->capacity_reruns = 1;
    return rc;
}

// Copy a completed host request's staged results to the caller.
static void deliver_host_results(Slot &s, const FetchTargets *fetch) {
    const size_t px = (size_t)s.g.h * s.g.w;
    const char *ho = reinterpret_cast<const char *>(s.h_out);
    uint16_t *rgb = fetch ? fetch->rgb : s.frame.rgb_out;
    float *score = fetch ? fetch->score : s.frame.score_out;
    uint8_t *changed = fetch ? fetch->changed : s.frame.changed_out;
    if (rgb) parallel_memcpy(rgb, ho, px * 6);
    if (score) parallel_memcpy(score, ho + px * 6, px * 4);
    if (changed) parallel_memcpy(changed, ho + px * 10, px);
    if (fetch && fetch->at_floor) {
        // engine.py:175-199: at-floor = score plane == the score floor
        const float *sp = reinterpret_cast<const float *>(ho + px * 6);
        const float floor = s.params.score_floor;
        for (size_t i = 0; i < px; ++i) fetch->at_floor[i] = sp[i] == floor ? 1u : 0u;
    }
}

static int wait_ticket(fx_context *ctx, int64_t ticket, int64_t timeout_ns, fx_counters *counters,
                       const FetchTargets *fetch) {
    const auto start = std::chrono::steady_clock::now();
    for (;;) {
        {
            std::lock_guard<std::mutex> lock(ctx->mu);
            cudaSetDevice(ctx->device);
            Slot *sp = find_ticket(ctx, ticket);
            if (!sp) return fail(ctx, FX_ERR_INVALID_ARGUMENT, "unknown ticket");
            Slot &s = *sp;
            if (fetch && (s.device || ((fetch->score || fetch->at_floor) && !s.stage_score) ||
                          (fetch->changed && !s.stage_changed)))
                return fail(ctx, FX_ERR_INVALID_ARGUMENT,
                            "fx_fetch: the request did not stage what was asked for");
            const cudaError_t e = cudaEventQuery(s.done);
            if (e == cudaSuccess) {
                char *hc = reinterpret_cast<char *>(s.h_ctr);
                uint32_t err;
                std::memcpy(&err, hc + dev_counters_bytes(), 4);
                bool overflow;
                int rc = finish_counters(ctx, s, hc, err, counters, &overflow);
                if (!rc && overflow) rc = rerun_with_capacity(ctx, s, counters);
                if (!rc && !s.device) deliver_host_results(s, fetch);
                s.busy = false;
                s.ticket = -1;
                return rc;
            }
            if (e != cudaErrorNotReady) {
                s.busy = false;
                return fail(ctx, FX_ERR_CUDA, "%s", cudaGetErrorString(e));
            }
        }
        if (timeout_ns >= 0) {
            const auto el = std::chrono::steady_clock::now() - start;
            if (std::chrono::duration_cast<std::chrono::nanoseconds>(el).count() > timeout_ns)
                return FX_ERR_TIMEOUT;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

FX_API int fx_wait(fx_context *ctx, int64_t ticket, int64_t timeout_ns, fx_counters *counters) {
    if (!ctx) return FX_ERR_INVALID_ARGUMENT;
    return wait_ticket(ctx, ticket, timeout_ns, counters, nullptr);
}

FX_API int fx_fetch(fx_context *ctx, int64_t ticket, int64_t timeout_ns, uint16_t *rgb_out,
                    fx_counters *counters, float *score_out, uint8_t *at_floor_out,
                    uint8_t *changed_out) {
    if (!ctx) return FX_ERR_INVALID_ARGUMENT;
    const FetchTargets fetch{rgb_out, score_out, at_floor_out, changed_out};
    return wait_ticket(ctx, ticket, timeout_ns, counters, &fetch);
}

FX_API int fx_set_walk_window(fx_context *ctx, double sigmas) {
    if (!ctx || !(sigmas >= 0.0) || sigmas > 64.0) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->walk_sigmas = sigmas;
    return FX_OK;
}

FX_API int fx_set_stencil_tile(fx_context *ctx, int32_t rows) {
    if (!ctx || (rows != 0 && rows != 8 && rows != 16)) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->stencil_rows = rows == 0 ? 8 : rows;
    return FX_OK;
}

FX_API int fx_set_list_capacity(fx_context *ctx, int64_t channels) {
    if (!ctx || channels < 0 || channels > ((int64_t)1 << 31)) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->list_capacity = channels;
    return FX_OK;
}

FX_API int fx_profile_enable(fx_context *ctx, int enable) {
    if (!ctx) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->profile = enable != 0;
    return FX_OK;
}

FX_API int fx_profile_read(fx_context *ctx, double *ms, int64_t *passes, int reset) {
    if (!ctx) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    for (auto &ev : ctx->pending) {
        FX_CUDA(ctx, cudaEventSynchronize(ev[kProfileStages]));
        for (int i = 0; i < kProfileStages; ++i) {
            float t = 0.0f;
            FX_CUDA(ctx, cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
            ctx->profile_ms[i] += t;
        }
        ctx->profile_passes += 1;
        ctx->spare.push_back(std::move(ev));
    }
    ctx->pending.clear();
    if (ms)
        for (int i = 0; i < kProfileStages; ++i) ms[i] = ctx->profile_ms[i];
    if (passes) *passes = ctx->profile_passes;
    if (reset) {
        for (int i = 0; i < kProfileStages; ++i) ctx->profile_ms[i] = 0.0;
        ctx->profile_passes = 0;
    }
    return FX_OK;
}

FX_API int fx_mem_info(fx_context *ctx, size_t *free_bytes, size_t *total_bytes) {
    if (!ctx || !free_bytes || !total_bytes) return FX_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    FX_CUDA(ctx, cudaMemGetInfo(free_bytes, total_bytes));
    return FX_OK;
}

FX_API int64_t fx_frame_bytes(int32_t h, int32_t w) {
    if (h < 1 || w < 1) return -1;
    const Geometry g = make_geometry(h, w);
    return (int64_t)arena_layout(g, default_amb_capacity(g), nullptr);
}

FX_API int fx_pass_bytes(fx_context *ctx, int32_t h, int32_t w, int64_t *bytes) {
    if (!ctx || !bytes || h < 1 || w < 1) return FX_ERR_INVALID_ARGUMENT;
    if ((int64_t)h * w > (int64_t)1 << 30) return FX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    const Geometry g = make_geometry(h, w);
    *bytes = (int64_t)arena_layout(g, pass_capacity(ctx, g), nullptr);
    return FX_OK;
}

}  // extern "C"
