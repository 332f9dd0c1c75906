// fx_internal.cuh -- shared device definitions of the B200 Digital ICE core.
//
// Numerics: every kernel is compiled with --fmad=false and without fast
// math, so each binary64 / binary32 add, multiply and divide rounds once,
// in the order written, exactly like the reference's scalar NumPy path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#include "../../include/fauxice_b200.h"

namespace fx {

constexpr uint32_t kLcgMask = 0x00FFFFFFu;
// rng.py:135: float32 bits 0x337fffff widened = (2^24 - 1) * 2^-48.
constexpr double kNormalization = 0x1.fffffep-25;
constexpr int kPad = 5;          // history-plane border (rows/cols)
constexpr int kTileH = 16;       // padded planes cover whole 16-row tiles (the
                                 // stencil runs 8- or 16-row tiles)
constexpr int kTileW = 32;       // stencil tile cols
constexpr int kSegment = 1024;   // chain sites per scan segment
constexpr int kSegThreads = 256; // threads per segment block

// Device error word: the first failing status wins.
__device__ __forceinline__ void raise_error(uint32_t *err, uint32_t code) {
    if (*reinterpret_cast<volatile uint32_t *>(err) == 0) atomicCAS(err, 0u, code);
}

// A pass's error block is four words: err[0] the status, err[1] the stop
// word.  Only the stage gates (k_gate, between kernel groups on the pass's
// stream) write the stop word, so it is constant while any other kernel of
// the pass runs and every thread of a kernel sees the same value: a kernel
// that finds it set returns before its first barrier, all its blocks alike.
__device__ __forceinline__ bool pass_stopped(const uint32_t *err) {
    return err[1] != 0u;
}

// ---------------------------------------------------------------------------
// Frame geometry and buffers
// ---------------------------------------------------------------------------

struct Geometry {
    int h, w;              // logical frame
    int th, tw;            // kTileH x kTileW blocks covering the frame
    int hp, wp;            // rows/cols rounded up to whole tiles
    int prow;              // padded rows = hp + 2*kPad
    int pitch;             // floats per padded row (>= wp + 2*kPad, multiple of 32)
    int64_t sites;         // chain sites = 6*w (startup) + h*w (public)
    int64_t segments;      // ceil(sites / kSegment)
    __host__ __device__ int64_t padded_index(int y, int x) const {
        return (int64_t)(y + kPad) * pitch + (x + kPad);
    }
};

// Per-site meta byte: bit 7 attempted, bits 2c..2c+1 draw code of channel c
// (0: no draw, 1: one draw, 2: two draws, 3: RNG-dependent: one or two).
__host__ __device__ __forceinline__ int meta_code(uint8_t m, int c) { return (m >> (2 * c)) & 3; }
__host__ __device__ __forceinline__ int meta_base(uint8_t m) {
    int b = 0;
    for (int c = 0; c < 3; ++c) {
        const int k = meta_code(m, c);
        b += (k == 3) ? 1 : k;
    }
    return b;
}
__host__ __device__ __forceinline__ int meta_amb(uint8_t m) {
    int a = 0;
    for (int c = 0; c < 3; ++c) a += meta_code(m, c) == 3;
    return a;
}

// One RNG-dependent channel for the serial walk.  In "T space" the 24-bit
// state s is held as T = s << 8, so the LCG s -> 125 s + 1 (mod 2^24)
// becomes T -> 125 T + 256 (mod 2^32) and interval tests need no masking.
struct __align__(16) AmbEntry {
    uint32_t l1, w1, l2, w2; // copy iff (T - l1) <= w1 || (T - l2) <= w2
    uint32_t a0, c0;         // T_first_draw = a0 * T_prev + c0 (previous channel drew once)
    uint32_t a1, c1;         // T_first_draw = a1 * T_prev + c1 (previous channel drew twice)
};

// ---------------------------------------------------------------------------
// LCG jump-ahead: g^n as an affine map, composed by binary powering.
// ---------------------------------------------------------------------------

struct Affine {
    uint32_t a, c;
};

__host__ __device__ __forceinline__ Affine affine_compose(Affine f, Affine g) {
    // (f o g)(x) = f.a * (g.a x + g.c) + f.c
    return Affine{f.a * g.a, f.a * g.c + f.c};
}

// g^n in T space (mod 2^32): a = 125^n, c = 256 * (125^n - 1) / 124.
__host__ __device__ __forceinline__ Affine lcg_power_t(uint64_t n) {
    Affine result{1u, 0u};
    Affine base{125u, 256u};
    while (n) {
        if (n & 1u) result = affine_compose(base, result);
        base = affine_compose(base, base);
        n >>= 1;
    }
    return result;
}

// g^n applied to a 24-bit state.
__host__ __device__ __forceinline__ uint32_t lcg_jump(uint32_t s, uint64_t n) {
    const Affine f = lcg_power_t(n);
    return ((f.a * (s << 8) + f.c) >> 8) & kLcgMask;
}

// ---------------------------------------------------------------------------
// Exact scalar pieces of the writer (dither.py:59-104, reconstruction.py:916-982)
// ---------------------------------------------------------------------------

struct DitherConst {
    double low, high;      // widened float32 bounds
    double coefficient;    // 4 / (width * width)
    int low_lt_high;
};

__device__ __forceinline__ DitherConst dither_const(const fx_params &p) {
    DitherConst d;
    d.low = (double)p.dither_low;
    d.high = (double)p.dither_high;
    d.low_lt_high = d.low < d.high;
    const double width = d.high - d.low;
    d.coefficient = 4.0 / (width * width);
    return d;
}

// Raw delta for a first-draw state s1 (before the accept test).
__device__ __forceinline__ double dither_raw_delta(double cand, double envelope, float span,
                                                   uint32_t s1) {
    const double unit = (double)(s1 + 1u) * kNormalization - 0.5;
    const double random_value = 0.0 + unit * (double)span;
    return envelope * random_value;
}

// conditional_dither_delta split in two: the state-free part of one
// channel (whether it draws, the float32-rounded candidate, the binary64
// envelope and the float32 span), computed once for both draws a channel
// may take, and one draw with the state advanced in place.
struct DitherChannel {
    double cand, envelope;
    float span;
    bool draws;
};

__device__ __forceinline__ DitherChannel dither_channel(double value, float scale32,
                                                        const DitherConst &dc) {
    DitherChannel ch;
    const float cand32 = (float)value;
    ch.cand = (double)cand32;
    ch.draws = dc.low_lt_high && dc.low < ch.cand && ch.cand < dc.high;
    ch.envelope = ((dc.high - ch.cand) * (ch.cand - dc.low)) * dc.coefficient;
    ch.span = (float)((double)scale32 * ch.cand);
    return ch;
}

// One draw: the accepted delta (or 0).  `drew` reports whether the LCG
// advanced.
__device__ __forceinline__ double dither_draw(const DitherChannel &ch, const DitherConst &dc,
                                              uint32_t &state, int &drew) {
    drew = 0;
    if (!ch.draws) return 0.0;
    state = (125u * state + 1u) & kLcgMask;
    drew = 1;
    const double d = dither_raw_delta(ch.cand, ch.envelope, ch.span, state);
    const double changed = ch.cand + d;
    return (dc.low < changed && changed < dc.high) ? d : 0.0;
}

// ---------------------------------------------------------------------------
// Host-visible launch helpers (defined in the .cu files)
// ---------------------------------------------------------------------------

// Writer scratch of one frame.  `capacity` bounds the RNG-dependent channel
// list; when a frame has more, the counters report it and the host reruns
// the writer with a larger list (every access below is clamped to it).
// Words of the chain prefix's partial sums: per segment (fixed << 16 |
// RNG-dependent, 1024 sites), then per group of kSegGroup segments the
// exclusive prefixes of fixed draws and of RNG-dependent channels.
constexpr int kSegGroup = 8;
__host__ __device__ inline int64_t seg_raw_words(int64_t segments) {
    const int64_t groups = (segments + kSegGroup - 1) / kSegGroup;
    return ((segments + 63) / 64) * 64 + 2 * (((groups + 63) / 64) * 64);
}

struct WriterBuffers {
    uint32_t *seg_base, *seg_amb;  // segments + 1 each
    uint32_t *seg_raw;             // seg_raw_words(segments): the prefix's partial sums
    AmbEntry *entries;             // capacity (+64 bytes slack)
    uint32_t *pos;                 // capacity
    uint32_t *extra_after;         // capacity
    void *counters;                // DevCounters
    int64_t capacity;
    void *walk_scratch;            // walk_scratch_bytes(capacity, per_wave)
    int per_wave;                  // window blocks per wave (walk_per_wave of the SM count)
    bool parallel_walk;
    double window_sigmas;          // walk window half-width in standard deviations
    const uint32_t *cancel;        // host-mapped cancel word read by the stage gates, or null
    uint8_t *chunk_two;            // walk_chunks(capacity): 1 when a chunk holds a
                                   // two-interval entry
    int priority;                  // launch priority of the chain and the walk (0: default)
};

// A kernel launch with an execution priority (cudaLaunchAttributePriority;
// numerically lower is higher, 0 is the default).  When several streams
// have work pending, the block scheduler dispatches the blocks of the
// higher-priority launch first; results do not depend on it.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_prio(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                               cudaStream_t stream, int priority, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = priority;
    cfg.attrs = attr;
    cfg.numAttrs = priority ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Optional CUDA events between kernel groups (measurement only).
// mark(i) records boundary i: 0 before the producer, then after each stage.
struct Marks {
    cudaEvent_t *events = nullptr;  // kProfileStages + 1 events, or null
    __host__ void mark(int i, cudaStream_t s) const {
        if (events) cudaEventRecord(events[i], s);
    }
};
constexpr int kProfileStages = 7;

cudaError_t analysis_init();
cudaError_t launch_analysis(const uint16_t *rgbi, const Geometry &g, const float *lut,
                            const fx_stage *stages, const fx_params &p, float *aux, float *hs,
                            float *hwa, float *hwr, int64_t plane, double *cand, uint8_t *meta,
                            uint32_t *err, cudaStream_t stream, const Marks &marks,
                            int tile_rows, cudaStream_t side, cudaEvent_t fork,
                            cudaEvent_t join);
cudaError_t writer_identity_table(const float *lut, const uint32_t *hi, const uint32_t *lo,
                                  uint16_t *ident, uint32_t *bad, cudaStream_t stream);
cudaError_t launch_writer(const Geometry &g, const uint8_t *meta, const double *cand,
                          const uint16_t *rgbi, const float *lut, const uint32_t *high,
                          const uint32_t *low, const uint16_t *ident, const fx_stage *stages,
                          const fx_params &p,
                          uint32_t s0, const WriterBuffers &b, uint16_t *rgb_out,
                          uint8_t *changed_out, uint32_t *err, cudaStream_t stream,
                          const Marks &marks);
size_t dev_counters_bytes();
cudaError_t walk_init();
size_t walk_scratch_bytes(int64_t capacity, int per_wave);
int walk_per_wave(int sms);
constexpr double kDefaultWindowSigmas = 4.5;
// Channels per staged chunk of the window walk; chunks start at multiples
// of it in list order (segments are whole chunks).
constexpr int kWalkChunk = 256;
constexpr uint32_t kWalkSegLen = 4096;  // channels per walk segment (whole chunks)
__host__ __device__ inline size_t walk_chunks(int64_t capacity) {
    return (size_t)((capacity + kWalkChunk - 1) / kWalkChunk) + 1;
}
void walk_segment_stats(void *scratch, int64_t capacity, unsigned long long **copy,
                        unsigned long long **spread, size_t *bytes_each);
cudaError_t launch_walk(const AmbEntry *entries, const uint32_t *pos, const uint32_t *n_ptr,
                        int64_t capacity, uint32_t s0, void *scratch, int per_wave,
                        bool parallel, double window_sigmas, const uint8_t *chunk_two,
                        uint32_t *extra_after, uint32_t *fallbacks_out,
                        unsigned long long *stats_out, const uint32_t *err,
                        cudaStream_t stream, int priority);
// Stage gate: when *cancel (host-mapped) is set, stop the pass: err[1] = 1
// and err[0] = FX_ERR_CANCELLED unless an error came first.  No launch when
// `cancel` is null.
cudaError_t launch_gate(const uint32_t *cancel, uint32_t *err, cudaStream_t stream);
void counters_to_host(const void *dev_copy, fx_counters *out);
uint32_t counters_n_amb(const void *dev_copy);
size_t producer_bytes(int h, int w);
cudaError_t launch_producer(const uint16_t *rgbi, int h, int w, const float *lut, void *scratch,
                            fx_stage *stages, float *rows_out, uint32_t *err,
                            cudaStream_t stream, int priority = 0);
int host_reduce_prepass(const uint16_t *px, int h, int w, const float *lut, uint8_t payload[64],
                        int64_t *valid_pixels, int64_t *fully_valid_tiles);
int host_stage_table(int h, const float *p1, const float *p2, const float *mv, const float *mi,
                     float factor_b, fx_stage *stages);

// fx_api.cu: context accessors for entry points defined in other files
int context_device(const fx_context *ctx);
const float *context_lut(const fx_context *ctx);
int context_fail(fx_context *ctx, int code, const char *fmt, ...);
int context_device_error(fx_context *ctx, uint32_t code);
void context_lock(fx_context *ctx);  // the context's call lock (fx_set_tables holds it)
void context_unlock(fx_context *ctx);

}  // namespace fx
