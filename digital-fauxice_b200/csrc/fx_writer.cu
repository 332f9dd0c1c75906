// fx_writer.cu -- the sequential dither writer, restructured for the GPU.
//
// The reference writes attempted sites in strict row-major order, threading
// one 24-bit LCG through every conditional draw (reconstruction.py:916-982,
// dither.py:59-104, rng.py:159-172).  The number of draws a channel takes is
// a function of the state only when its first draw happens, the floor gate
// is on and the floor comparison is not settled by the largest possible
// |delta|.  So:
//   1. k_stencil / k_startup classify every channel: 0, 1 or 2 fixed draws,
//      or "RNG-dependent" (one or two).
//   2. k_seg_sums + k_seg_scan: exclusive prefix of fixed draws and of
//      RNG-dependent channels along the chain (startup sites, then public
//      sites in row-major order).
//   3. k_amb: for each RNG-dependent channel, the set of first-draw states
//      that copy the original, as at most two state intervals (found by
//      binary search on the exact binary64 expressions, which are monotone
//      in the state).
//   4. k_coef: the affine LCG jump g^gap between consecutive such channels.
//   5. the walk (fx_walk.cu) visits only the RNG-dependent channels: a jump,
//      an interval test, a select per channel, parallelised over segments by
//      speculation.  Output: the running count of extra draws.
//   6. k_apply: every public site recomputes its exact draws and values from
//      its own start state g^(fixed + extra before it)(s0), in parallel, and
//      emits public RGB16 with the counters.
#include <algorithm>

#include "fx_internal.cuh"

namespace fx {

struct DevCounters {
    unsigned long long attempted, written, public_advances, changed;
    unsigned long long su_attempted[6], su_advances[6];
    unsigned long long public_base, public_amb;
    uint32_t final_state, su_final_state;
    uint32_t startup_base, startup_amb, startup_extra;
    uint32_t n_amb;
    uint32_t walk_fallbacks;
    uint32_t walk_packed;              // written together with walk_fallbacks
    unsigned long long walk_stats[3];  // candidate steps, window sum, survivor sum
    uint32_t su_base[6], su_amb[6];    // per startup row, for the last block's prefix
    uint32_t su_done;                  // startup rows summed
    unsigned long long apply_next;     // k_apply's next segment
};

// ---------------------------------------------------------------------------
// Block scan helpers (256 threads)
// ---------------------------------------------------------------------------

// Exclusive scan of 64-bit values (packed counters) over a block of NT threads.
template <int NT>
__device__ __forceinline__ unsigned long long block_exclusive_scan64(unsigned long long v,
                                                                    unsigned long long &total,
                                                                    unsigned long long *warp_sums) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned long long w = (lane < NT / 32) ? warp_sums[lane] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < NT / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    const unsigned long long prefix = warp ? warp_sums[warp - 1] : 0ull;
    total = warp_sums[NT / 32 - 1];
    __syncthreads();
    return prefix + x - v;
}

template <int NT, typename T>
__device__ __forceinline__ T block_sum(T v, T *scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    T total = 0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < NT / 32; ++i) total += scratch[i];
        scratch[0] = total;
    }
    __syncthreads();
    total = scratch[0];
    __syncthreads();
    return total;
}

constexpr int kPer = kSegment / kSegThreads;  // sites per thread

// Running extra-draw count after `count` RNG-dependent channels (clamped to
// the list capacity; an overflowing frame is rerun by the host).
__device__ __forceinline__ uint32_t extra_before(const uint32_t *extra_after, uint32_t count,
                                                 int64_t capacity) {
    if (count == 0) return 0u;
    const int64_t i = (int64_t)count - 1;
    return extra_after[i < capacity ? i : capacity - 1];
}

// Packed local (base << 16 | amb) of one thread's sites.
__device__ __forceinline__ void load_meta(const uint8_t *meta, int64_t first, int64_t sites,
                                          uint8_t m[kPer]) {
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int64_t s = first + i;
        m[i] = (s < sites) ? meta[s] : 0;
    }
}

// (fixed draws << 16) | RNG-dependent channels of the four sites of one
// meta word.  Per channel code k (bits 2c, 2c+1): fixed draws k, except 1
// for k = 3, and one RNG-dependent channel when k = 3; so over the lows
// (k & 1), highs (k >> 1) and both: fixed = lows + 2 highs - 2 both.
__device__ __forceinline__ uint32_t packed_word(uint32_t w) {
    const uint32_t lo = w & 0x15151515u, hi = (w >> 1) & 0x15151515u;
    const uint32_t amb = (uint32_t)__popc(lo & hi);
    const uint32_t base = (uint32_t)__popc(lo) + 2u * (uint32_t)__popc(hi) - 2u * amb;
    return (base << 16) | amb;
}

__device__ __forceinline__ uint32_t packed_site(uint8_t m) {
    return ((uint32_t)meta_base(m) << 16) | (uint32_t)meta_amb(m);
}

constexpr int kSegWarps = 8;  // segments per block of the chain kernels (one per warp)

static_assert(kSegWarps == kSegGroup, "a k_seg_sums block sums one group of segments");

// The chain prefix's partial sums (seg_raw_words): per-segment sums, then
// the groups' exclusive prefixes of fixed draws and RNG-dependent channels.
struct SegRaw {
    uint32_t *seg, *grp_base, *grp_amb;
};
__device__ __forceinline__ SegRaw seg_raw_view(uint32_t *raw, int64_t segs) {
    const int64_t groups = (segs + kSegGroup - 1) / kSegGroup;
    SegRaw v;
    v.seg = raw;
    v.grp_base = raw + ((segs + 63) / 64) * 64;
    v.grp_amb = v.grp_base + ((groups + 63) / 64) * 64;
    return v;
}

// Fixed draws and RNG-dependent channels of every segment (packed as
// fixed << 16 | RNG-dependent), and of every group of eight segments: one
// warp per segment, 32 sites per lane in two 16-byte loads (the meta array
// starts on a 256-byte boundary and segments on multiples of 1024 sites),
// one block per group.  The group sums go where k_seg_scan writes the
// groups' prefixes.
__global__ void __launch_bounds__(kSegWarps * 32)
    k_seg_sums(const uint8_t *__restrict__ meta, int64_t sites, int64_t segs,
               uint32_t *__restrict__ raw, const uint32_t *__restrict__ err) {
    __shared__ uint32_t s_warp[kSegWarps];
    if (pass_stopped(err)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t seg = (int64_t)blockIdx.x * kSegWarps + warp;
    const SegRaw v = seg_raw_view(raw, segs);
    uint32_t packed = 0;
    const int64_t first = seg * kSegment + lane * 32;
    if (seg < segs) {
        if (first + 32 <= sites) {
            const uint4 *q = reinterpret_cast<const uint4 *>(meta + first);
            const uint4 u = q[0], w = q[1];
            packed = packed_word(u.x) + packed_word(u.y) + packed_word(u.z) + packed_word(u.w) +
                     packed_word(w.x) + packed_word(w.y) + packed_word(w.z) + packed_word(w.w);
        } else {
            for (int i = 0; i < 32; ++i)
                if (first + i < sites) packed += packed_site(meta[first + i]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) packed += __shfl_xor_sync(0xFFFFFFFFu, packed, o);
    if (lane == 0) {
        if (seg < segs) v.seg[seg] = packed;
        s_warp[warp] = packed;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t g = 0;  // at most 8 x 6144 fixed draws and 8 x 3072 channels
#pragma unroll
        for (int k = 0; k < kSegWarps; ++k) g += s_warp[k];
        v.grp_base[blockIdx.x] = g;
    }
}

// Exclusive scan of the groups' sums into the groups' prefixes; seg_base[n]
// and seg_amb[n] get the totals (n segments).  One block of 1024 threads,
// over tiles of 4096 groups (a native frame has 2.8 k): a tile is loaded
// coalesced into shared memory, each thread scans four neighbouring groups,
// and one block scan of (fixed << 32 | RNG-dependent) pairs gives the
// threads' offsets (the RNG-dependent total stays below 2^32: at most three
// per site).  k_amb adds a segment's offset inside its group.
__global__ void __launch_bounds__(1024)
    k_seg_scan(uint32_t *__restrict__ raw, int64_t n, uint32_t *__restrict__ seg_base,
               uint32_t *__restrict__ seg_amb, const uint32_t *__restrict__ err) {
    constexpr int kPerThread = 4, kTile = 1024 * kPerThread;
    __shared__ uint32_t tb[kTile], ta[kTile];
    __shared__ unsigned long long ws[32];
    if (pass_stopped(err)) return;
    const SegRaw v = seg_raw_view(raw, n);
    const int64_t groups = (n + kSegGroup - 1) / kSegGroup;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned long long carry = 0;
    for (int64_t t0 = 0; t0 < groups; t0 += kTile) {
        for (int j = tid; j < kTile; j += 1024) {
            const int64_t i = t0 + j;
            const uint32_t g = i < groups ? v.grp_base[i] : 0u;
            tb[j] = g >> 16;
            ta[j] = g & 0xFFFFu;
        }
        __syncthreads();
        unsigned long long mine = 0;
#pragma unroll
        for (int k = 0; k < kPerThread; ++k)
            mine += ((unsigned long long)tb[kPerThread * tid + k] << 32) | ta[kPerThread * tid + k];
        unsigned long long x = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) ws[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned long long w = ws[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, w, o);
                if (lane >= o) w += y;
            }
            ws[lane] = w;
        }
        __syncthreads();
        unsigned long long run = carry + (warp ? ws[warp - 1] : 0ull) + x - mine;
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
            const int j = kPerThread * tid + k;
            const unsigned long long val = ((unsigned long long)tb[j] << 32) | ta[j];
            tb[j] = (uint32_t)(run >> 32);
            ta[j] = (uint32_t)run;
            run += val;
        }
        carry += ws[31];
        __syncthreads();
        for (int j = tid; j < kTile; j += 1024) {
            const int64_t i = t0 + j;
            if (i < groups) {
                v.grp_base[i] = tb[j];
                v.grp_amb[i] = ta[j];
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        seg_base[n] = (uint32_t)(carry >> 32);
        seg_amb[n] = (uint32_t)carry;
    }
}

struct SiteInfo {
    float orig[3];
    bool floor_enabled;
};

__device__ __forceinline__ SiteInfo site_info(int64_t site, int w, const uint16_t *rgbi,
                                              const float *lut, const fx_stage *stages,
                                              const fx_params &p) {
    SiteInfo si;
    const int64_t su = 6 * (int64_t)w;
    int64_t pixel;
    int stage_index;
    if (site < su) {
        pixel = site % w;  // startup originals are row 0 (startup.py:327-336)
        stage_index = (int)(site / w);
    } else {
        pixel = site - su;
        stage_index = (int)(pixel / w) + 6;
    }
    const uint2 raw = reinterpret_cast<const uint2 *>(rgbi)[pixel];
    si.orig[0] = __ldg(lut + (raw.x & 0xFFFFu));
    si.orig[1] = __ldg(lut + (raw.x >> 16));
    si.orig[2] = __ldg(lut + (raw.y & 0xFFFFu));
    si.floor_enabled = p.driver_gate_primary || stages[stage_index].gate_secondary;
    return si;
}

// ---------------------------------------------------------------------------
// Copy intervals of one RNG-dependent channel
// ---------------------------------------------------------------------------

struct ChannelView {
    double cand, cd, env, od;
    float span;
    DitherConst dc;
    __device__ double raw(uint32_t s1) const { return dither_raw_delta(cd, env, span, s1); }
    __device__ bool low_ok(uint32_t s1) const { return dc.low < cd + raw(s1); }
    __device__ bool high_ok(uint32_t s1) const { return cd + raw(s1) < dc.high; }
    __device__ bool floor_test(uint32_t s1) const { return cand + raw(s1) <= od; }
    __device__ bool copies(uint32_t s1) const {
        const double d = raw(s1);
        const double changed = cd + d;
        const double eff = (dc.low < changed && changed < dc.high) ? d : 0.0;
        return cand + eff <= od;
    }
};

// First state where a monotone predicate differs from its value at 0
// (2^24 when it never does).  `guess` estimates that state; the search
// gallops from it to a bracket checked on the exact predicate and bisects
// inside, so the estimate changes only the cost, never the result.
template <class F>
__device__ __forceinline__ uint32_t switch_point(F pred, double guess) {
    const bool p0 = pred(0u);
    if (pred(kLcgMask) == p0) return kLcgMask + 1u;
    // invariant: pred(lo) == p0, pred(hi) != p0, lo < hi
    uint32_t lo = 0u, hi = kLcgMask;
    uint32_t x = kLcgMask / 2u;
    if (guess == guess) {  // not NaN
        const double top = (double)(kLcgMask - 1u);
        x = (uint32_t)(guess < 1.0 ? 1.0 : (guess > top ? top : guess));
    }
    uint32_t step = 1u;
    if (pred(x) == p0) {
        lo = x;
        while (hi - lo > 1u) {
            if (hi - lo <= step) break;
            const uint32_t y = lo + step;
            if (pred(y) == p0) {
                lo = y;
                step <<= 1;
            } else {
                hi = y;
                break;
            }
        }
    } else {
        hi = x;
        while (hi - lo > 1u) {
            if (hi - lo <= step) break;
            const uint32_t y = hi - step;
            if (pred(y) != p0) {
                hi = y;
                step <<= 1;
            } else {
                lo = y;
                break;
            }
        }
    }
    while (hi - lo > 1u) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (pred(mid) == p0) lo = mid;
        else hi = mid;
    }
    return hi;
}

// The state s1 at which base + raw(s1) would reach `target` if the delta
// were computed exactly (it is affine in s1): a starting point for
// switch_point.
__device__ __forceinline__ double crossing(const ChannelView &cv, double base, double target) {
    const double scale = cv.env * (double)cv.span;
    return ((target - base) / scale + 0.5) / kNormalization - 1.0;
}

__device__ void copy_intervals(const ChannelView &cv, AmbEntry &e, uint32_t *err) {
    uint32_t b[3] = {
        switch_point([&](uint32_t s) { return cv.low_ok(s); }, crossing(cv, cv.cd, cv.dc.low)),
        switch_point([&](uint32_t s) { return cv.high_ok(s); }, crossing(cv, cv.cd, cv.dc.high)),
        switch_point([&](uint32_t s) { return cv.floor_test(s); }, crossing(cv, cv.cand, cv.od))};
    // sort the three breakpoints
    if (b[0] > b[1]) { const uint32_t t = b[0]; b[0] = b[1]; b[1] = t; }
    if (b[1] > b[2]) { const uint32_t t = b[1]; b[1] = b[2]; b[2] = t; }
    if (b[0] > b[1]) { const uint32_t t = b[0]; b[0] = b[1]; b[1] = t; }
    uint32_t starts[4];
    int n = 0;
    starts[n++] = 0u;
    for (int i = 0; i < 3; ++i)
        if (b[i] <= kLcgMask && b[i] != starts[n - 1]) starts[n++] = b[i];
    uint32_t lo[2], hi[2];
    int intervals = 0;
    bool open = false;
    for (int i = 0; i < n; ++i) {
        const uint32_t first = starts[i];
        const uint32_t last = (i + 1 < n) ? starts[i + 1] - 1u : kLcgMask;
        const bool c = cv.copies(first);
        if (c) {
            if (open) {
                hi[intervals - 1] = last;
            } else {
                if (intervals == 2) { raise_error(err, FX_ERR_INTERNAL); return; }
                lo[intervals] = first;
                hi[intervals] = last;
                ++intervals;
                open = true;
            }
        } else {
            open = false;
        }
    }
    // empty interval: l = 0x80 can never match a T value (low byte zero)
    e.l1 = 0x80u; e.w1 = 0u; e.l2 = 0x80u; e.w2 = 0u;
    if (intervals == 2 && lo[0] == 0u && hi[1] == kLcgMask) {
        // [0, hi0] and [lo1, 2^24 - 1] meet across the wrap: one cyclic
        // interval from lo1 (the test (T - l) <= w wraps modulo 2^32)
        e.l1 = lo[1] << 8;
        e.w1 = (hi[0] - lo[1]) << 8;
        return;
    }
    if (intervals >= 1) { e.l1 = lo[0] << 8; e.w1 = (hi[0] - lo[0]) << 8; }
    if (intervals == 2) { e.l2 = lo[1] << 8; e.w2 = (hi[1] - lo[1]) << 8; }
}

// Lists every RNG-dependent channel in chain order: entry a gets its site
// (site_of[a], a compact array so the writes coalesce) and its draw
// position; k_coef fills in the intervals and jumps.  One warp per segment,
// in 16 rounds of 64 consecutive sites, two neighbouring sites per lane (all
// the segment's meta loads issued first); a round's offsets come from one
// warp scan, so a round's entries are written by consecutive lanes to
// consecutive list positions.
__global__ void __launch_bounds__(kSegWarps * 32)
    k_amb(const uint8_t *__restrict__ meta, int64_t sites, int64_t segs,
          uint32_t *__restrict__ raw, uint32_t *__restrict__ seg_base,
          uint32_t *__restrict__ seg_amb, uint32_t *__restrict__ site_of,
          uint32_t *__restrict__ pos_out, int64_t capacity, const uint32_t *__restrict__ err) {
    if (pass_stopped(err)) return;
    const int lane = threadIdx.x & 31;
    const int64_t seg = (int64_t)blockIdx.x * kSegWarps + (threadIdx.x >> 5);
    if (seg >= segs) return;
    const int64_t first = seg * kSegment + 2 * lane;  // sites first + 64 r, + 1
    uint32_t m2[16];  // the two meta bytes of round r
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        const int64_t s0 = first + 64 * r;
        if (s0 + 1 < sites)
            m2[r] = *reinterpret_cast<const uint16_t *>(meta + s0);  // even offset
        else
            m2[r] = s0 < sites ? meta[s0] : 0u;
    }
    // the segment's prefix: its group's, plus the segments before it in the
    // group (fewer than eight, so the packed halves cannot carry); written
    // for the kernels after the walk
    const SegRaw v = seg_raw_view(raw, segs);
    const int64_t grp = seg / kSegGroup, k0 = grp * kSegGroup;
    uint32_t before = (k0 + lane < seg) ? v.seg[k0 + lane] : 0u;
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) before += __shfl_xor_sync(0xFFFFFFFFu, before, o);
    before = __shfl_sync(0xFFFFFFFFu, before, 0);
    uint32_t P = v.grp_base[grp] + (before >> 16), A = v.grp_amb[grp] + (before & 0xFFFFu);
    if (lane == 0) {
        seg_base[seg] = P;
        seg_amb[seg] = A;
    }
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        const uint8_t mb[2] = {(uint8_t)(m2[r] & 0xFFu), (uint8_t)(m2[r] >> 8)};
        const uint32_t x0 = packed_site(mb[0]), x = x0 + packed_site(mb[1]);
        uint32_t inc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if (lane >= o) inc += y;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, inc, 31);
        if (x & 0xFFFFu) {
            const uint32_t ex = inc - x;
            uint32_t pos = P + (ex >> 16), a = A + (ex & 0xFFFFu);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint8_t mi = mb[h];
                pos = P + ((ex + (h ? x0 : 0u)) >> 16);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int code = meta_code(mi, c);
                    if (code == 3) {
                        if ((int64_t)a < capacity) {
                            site_of[a] = (uint32_t)(first + 64 * r + h);
                            pos_out[a] = pos;
                        }
                        ++a;
                        pos += 1u;
                    } else {
                        pos += (uint32_t)code;
                    }
                }
            }
        }
        P += total >> 16;
        A += total & 0xFFFFu;
    }
}

// k_coef's inputs of one entry, gathered in two dependent steps: the list
// (coalesced) gives the site, the site gives its meta, pixel and candidates.
struct CoefList {
    uint32_t site, gap_lo, gap_hi;  // gap_lo/hi: pos[i-1] (0 for the first) and pos[i]
    int k;                          // this entry is the k-th of its site
};
struct CoefSite {
    uint8_t meta;
    uint2 raw;
    double cand[3];
};

__device__ __forceinline__ CoefList coef_list(const uint32_t *__restrict__ site_of,
                                              const uint32_t *__restrict__ pos, uint32_t i,
                                              uint32_t n) {
    CoefList l{0u, 0u, 0u, 0};
    if (i >= n) return l;
    l.site = site_of[i];
    // a site's RNG-dependent channels are listed in channel order
    l.k = (i >= 1 && site_of[i - 1] == l.site) ? ((i >= 2 && site_of[i - 2] == l.site) ? 2 : 1)
                                                : 0;
    l.gap_hi = pos[i];
    l.gap_lo = i ? pos[i - 1] : 0u;
    return l;
}

__device__ __forceinline__ CoefSite coef_site(const CoefList &l, bool live, int64_t su, int w,
                                              const uint8_t *__restrict__ meta,
                                              const double *__restrict__ cand,
                                              const uint16_t *__restrict__ rgbi) {
    CoefSite c{};
    if (!live) return c;
    const int64_t site = l.site;
    const int64_t pixel = site < su ? site % w : site - su;
    c.meta = meta[site];
    c.raw = reinterpret_cast<const uint2 *>(rgbi)[pixel];
    c.cand[0] = cand[3 * site];
    c.cand[1] = cand[3 * site + 1];
    c.cand[2] = cand[3 * site + 2];
    return c;
}

// Copy intervals and jumps of every RNG-dependent channel.  A thread's
// entries i, i + stride, ... run through a three-stage software pipeline:
// while entry i's interval search computes, the site of entry i + 2 stride
// and the meta, pixel and candidates of entry i + stride are in flight, so
// the dependent gathers overlap the arithmetic instead of stalling it.
__global__ void __launch_bounds__(256, 4) k_coef(AmbEntry *__restrict__ entries, const uint32_t *__restrict__ pos,
                       const uint32_t *__restrict__ n_amb_ptr, int64_t capacity,
                       const uint32_t *__restrict__ site_of, const uint8_t *__restrict__ meta,
                       const double *__restrict__ cand, int w, const uint16_t *__restrict__ rgbi,
                       const float *__restrict__ lut, fx_params p, uint32_t *err,
                       uint8_t *__restrict__ chunk_two, unsigned long long *__restrict__ seg_copy,
                       unsigned long long *__restrict__ seg_spread) {
    if (pass_stopped(err)) return;
    const uint32_t n = (uint32_t)min((int64_t)*n_amb_ptr, capacity);
    const DitherConst dc = dither_const(p);
    const int64_t su = 6 * (int64_t)w;
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    CoefList l0 = coef_list(site_of, pos, i, n);
    CoefSite s0 = coef_site(l0, i < n, su, w, meta, cand, rgbi);
    CoefList l1 = coef_list(site_of, pos, i + stride, n);
    for (; i < n; i += stride) {
        const uint32_t i1 = i + stride, i2 = i1 + stride;
        const CoefSite s1 = coef_site(l1, i1 < n && i1 > i, su, w, meta, cand, rgbi);
        const CoefList l2 = coef_list(site_of, pos, i2 > i1 ? i2 : n, n);
        const uint8_t mi = s0.meta;
        int c = 0;
        for (int seen = 0; c < 3; ++c)
            if (meta_code(mi, c) == 3 && seen++ == l0.k) break;
        const uint2 raw = s0.raw;
        const uint32_t lane = c == 0 ? (raw.x & 0xFFFFu) : (c == 1 ? (raw.x >> 16) : (raw.y & 0xFFFFu));
        ChannelView cv;
        cv.cand = c == 0 ? s0.cand[0] : (c == 1 ? s0.cand[1] : s0.cand[2]);
        cv.cd = (double)(float)cv.cand;
        cv.dc = dc;
        cv.env = ((dc.high - cv.cd) * (cv.cd - dc.low)) * dc.coefficient;
        cv.span = (float)((double)p.dither_scales[c] * cv.cd);
        cv.od = (double)__ldg(lut + lane);
        AmbEntry e;
        copy_intervals(cv, e, err);
        // a chunk of walk channels with a two-interval entry steps with both
        // interval tests (every other chunk with one)
        if (e.l2 != 0x80u) chunk_two[i / kWalkChunk] = 1;
        // the walk's prediction for this segment: m copying states of 2^24
        // (an extra draw with probability p = 1 - m / 2^24), summed exactly
        // per segment, with the spread m (2^24 - m) >> 22 (p (1 - p) in
        // units of 2^-26).  A warp holds 32 consecutive entries of one
        // segment; the lanes past the chain's end have left the loop.
        {
            uint32_t m = 0;
            if (e.l1 != 0x80u) m += (e.w1 >> 8) + 1u;
            if (e.l2 != 0x80u) m += (e.w2 >> 8) + 1u;
            const uint32_t q = (uint32_t)(((unsigned long long)m * ((1u << 24) - m)) >> 22);
            const uint32_t lane = threadIdx.x & 31, live = n - (i - lane);
            const uint32_t mask = live >= 32u ? 0xFFFFFFFFu : ((1u << live) - 1u);
            const uint32_t ms = __reduce_add_sync(mask, m), qs = __reduce_add_sync(mask, q);
            if (lane == 0) {
                atomicAdd(&seg_copy[i / kWalkSegLen], (unsigned long long)ms);
                atomicAdd(&seg_spread[i / kWalkSegLen], (unsigned long long)qs);
            }
        }
        const uint64_t gap = (i == 0) ? (uint64_t)l0.gap_hi + 1u
                                      : (uint64_t)(uint32_t)(l0.gap_hi - l0.gap_lo);
        const Affine f = lcg_power_t(gap);
        const Affine f1 = affine_compose(Affine{125u, 256u}, f);  // one more draw
        e.a0 = f.a;
        e.c0 = f.c;
        e.a1 = (i == 0) ? f.a : f1.a;  // no previous channel before the first
        e.c1 = (i == 0) ? f.c : f1.c;
        entries[i] = e;
        l0 = l1;
        s0 = s1;
        l1 = l2;
    }
}

// ---------------------------------------------------------------------------
// The serial walk (one resident warp per frame; lane 0 walks)
// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// Startup counters, apply + emit, final state
// ---------------------------------------------------------------------------

// Startup counters: one block per startup row sums its attempted sites,
// fixed draws and RNG-dependent channels; the last block to finish chains
// the six rows (the extra draws of a row come from the walk's running count
// at the row's ends).
__global__ void k_startup_counts(const uint8_t *__restrict__ meta, int w,
                                 const uint32_t *__restrict__ extra_after, uint32_t s0,
                                 DevCounters *ctr, int64_t capacity,
                                 const uint32_t *__restrict__ err) {
    __shared__ unsigned long long scratch[8];
    __shared__ bool last;
    if (pass_stopped(err)) return;
    const int k = blockIdx.x;  // startup row 0..5
    unsigned long long att = 0, base = 0, amb = 0;
    for (int x = threadIdx.x; x < w; x += blockDim.x) {
        const uint8_t m = meta[(int64_t)k * w + x];
        att += (m >> 7) & 1u;
        base += meta_base(m);
        amb += meta_amb(m);
    }
    att = block_sum<256, unsigned long long>(att, scratch);
    base = block_sum<256, unsigned long long>(base, scratch);
    amb = block_sum<256, unsigned long long>(amb, scratch);
    if (threadIdx.x == 0) {
        ctr->su_attempted[k] = att;
        ctr->su_base[k] = (uint32_t)base;
        ctr->su_amb[k] = (uint32_t)amb;
        __threadfence();
        last = atomicAdd(&ctr->su_done, 1u) == 5u;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    const volatile DevCounters *vc = ctr;
    uint32_t a_run = 0, p_run = 0;
    for (int r = 0; r < 6; ++r) {
        const uint32_t rb = vc->su_base[r], ra = vc->su_amb[r];
        const uint32_t e_start = extra_before(extra_after, a_run, capacity);
        const uint32_t a_end = a_run + ra;
        const uint32_t e_end = extra_before(extra_after, a_end, capacity);
        ctr->su_advances[r] = (unsigned long long)rb + (e_end - e_start);
        a_run = a_end;
        p_run += rb;
    }
    const uint32_t e = extra_before(extra_after, a_run, capacity);
    ctr->startup_base = p_run;
    ctr->startup_amb = a_run;
    ctr->startup_extra = e;
    ctr->su_final_state = lcg_jump(s0, (uint64_t)p_run + e);
}

__device__ __forceinline__ bool emit_one(float v, const uint32_t *hi, const uint32_t *lo,
                                         uint16_t &out) {
    if (!isfinite(v)) return false;
    double wv = (double)v + 0.5;
    wv = (wv < 0.0) ? 0.0 : wv;
    wv = (wv > 65535.0) ? 65535.0 : wv;
    const uint32_t idx = (uint32_t)wv;  // truncation (output.py:61-73)
    const unsigned long long prod = (unsigned long long)hi[idx >> 8] * lo[idx & 0xFFu];
    out = (uint16_t)((prod >> 20) - 1ull);
    return true;
}

// Identity emits: ident[v] = emit(lut[v]), the output of a channel whose
// value is its original (every unattempted pixel, and the comparison emit of
// an attempted one).  *bad is set when a LUT value is not finite.
__global__ void k_identity(const float *__restrict__ lut, const uint32_t *__restrict__ hi,
                           const uint32_t *__restrict__ lo, uint16_t *__restrict__ ident,
                           uint32_t *bad) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= 65536) return;
    uint16_t e = 0;
    if (!emit_one(lut[v], hi, lo, e)) {
        atomicOr(bad, 1u);
        e = 0;
    }
    ident[v] = e;
}

cudaError_t writer_identity_table(const float *lut, const uint32_t *hi, const uint32_t *lo,
                                  uint16_t *ident, uint32_t *bad, cudaStream_t stream) {
    cudaMemsetAsync(bad, 0, sizeof(uint32_t), stream);
    k_identity<<<256, 256, 0, stream>>>(lut, hi, lo, ident, bad);
    return cudaGetLastError();
}

// Affine jump tables: g_jump[j][d] = g^(d * 64^j) in T space, so any jump
// below 2^36 draws is six table lookups and compositions.
constexpr int kJumpDigits = 6;
__device__ Affine g_jump[kJumpDigits][64];
constexpr int kApplyBlocksPerSM = 5;  // k_apply's resident blocks per SM
static int g_apply_blocks = kApplyBlocksPerSM * 148;

cudaError_t writer_init() {
    int device = 0, sms = 0;
    if (cudaGetDevice(&device) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess &&
        sms > 0)
        g_apply_blocks = kApplyBlocksPerSM * sms;
    Affine tab[kJumpDigits][64];
    Affine step{125u, 256u};  // g^(64^j)
    for (int j = 0; j < kJumpDigits; ++j) {
        Affine acc{1u, 0u};
        for (int d = 0; d < 64; ++d) {
            tab[j][d] = acc;
            acc = affine_compose(step, acc);
        }
        step = acc;
    }
    return cudaMemcpyToSymbol(g_jump, tab, sizeof(tab));
}

__device__ __forceinline__ uint32_t jump_by_table(const Affine (*tab)[64], uint32_t s,
                                                  uint64_t n) {
    Affine r{1u, 0u};
#pragma unroll
    for (int j = 0; j < kJumpDigits; ++j) r = affine_compose(tab[j][(n >> (6 * j)) & 63u], r);
    return ((r.a * (s << 8) + r.c) >> 8) & kLcgMask;
}

// Public sites: exact draws and values, emit, counters.  A block takes
// 1024-site segments by ticket until none is left (one resident wave of
// blocks; the LCG jump and emit tables are loaded once per block).  Phase 1
// emits every site that was not attempted (its output is the identity emit)
// and lists the attempted ones in shared memory; phase 2 processes that list
// densely, each entry from its own start state g^(fixed + extra before
// it)(s0), and checks the draws it makes against the classification and the
// walk.
__global__ void __launch_bounds__(kSegThreads, kApplyBlocksPerSM)
    k_apply(const uint8_t *__restrict__ meta, const double *__restrict__ cand, int64_t sites,
            int w, const uint16_t *__restrict__ rgbi, const float *__restrict__ lut,
            const uint32_t *__restrict__ g_high, const uint32_t *__restrict__ g_low,
            const uint16_t *__restrict__ ident, const fx_stage *__restrict__ stages, fx_params p,
            const uint32_t *__restrict__ seg_base, const uint32_t *__restrict__ seg_amb,
            const uint32_t *__restrict__ extra_after, uint32_t s0, uint16_t *__restrict__ rgb_out,
            uint8_t *__restrict__ changed_out, DevCounters *ctr, uint32_t *err,
            int64_t capacity) {
    __shared__ uint32_t hi[256], lo[256];
    __shared__ unsigned long long s_sums[kSegThreads / 32][4];
    __shared__ Affine s_jump[kJumpDigits][64];
    __shared__ uint32_t s_ref[kSegment], s_p[kSegment], s_a[kSegment];
    __shared__ unsigned long long s_seg;
    __shared__ unsigned long long ws64[kSegThreads / 32];
    if (pass_stopped(err)) return;  // cancelled: the output stays untouched
    for (int i = threadIdx.x; i < 256; i += kSegThreads) {
        hi[i] = g_high[i];
        lo[i] = g_low[i];
    }
    for (int i = threadIdx.x; i < kJumpDigits * 64; i += kSegThreads)
        s_jump[i / 64][i % 64] = g_jump[i / 64][i % 64];
    const int64_t su = 6 * (int64_t)w;
    const int64_t segs = (sites + kSegment - 1) / kSegment;
    const DitherConst dc = dither_const(p);
    unsigned long long att = 0, written = 0, changed = 0, draws_total = 0;
    bool ok = true;
    // segments by ticket: the tables above are loaded once per block
    for (;;) {
        __syncthreads();  // the previous segment's list and ticket are consumed
        if (threadIdx.x == 0) s_seg = atomicAdd(&ctr->apply_next, 1ull);
        __syncthreads();
        const int64_t seg = (int64_t)s_seg;
        if (seg >= segs) break;
        const int64_t seg0 = seg * kSegment;
        const int64_t first = seg0 + threadIdx.x * kPer;
        uint8_t m[kPer];
        load_meta(meta, first, sites, m);
        // one block scan gives each thread its sites' chain offsets (fixed
        // draws, RNG-dependent channels) and its first slot in the list of
        // attempted public sites: (fixed << 40 | channels << 20 | attempted)
        unsigned long long mine = 0;
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
            const int64_t site = first + i;
            const bool listed = site >= su && site < sites && (m[i] & 0x80u);
            mine += ((unsigned long long)meta_base(m[i]) << 40) |
                    ((unsigned long long)meta_amb(m[i]) << 20) | (listed ? 1ull : 0ull);
        }
        unsigned long long total;
        const unsigned long long ex = block_exclusive_scan64<kSegThreads>(mine, total, ws64);
        uint32_t P = seg_base[seg] + (uint32_t)(ex >> 40);
        uint32_t A = seg_amb[seg] + (uint32_t)((ex >> 20) & 0xFFFFFu);
        const uint32_t listed = (uint32_t)(total & 0xFFFFFu);

        // ---- phase 1: identity emits; list the attempted sites ---------------
        {
            uint32_t slot = (uint32_t)(ex & 0xFFFFFu);
#pragma unroll
            for (int i = 0; i < kPer; ++i) {
                const int64_t site = first + i;
                const uint8_t mi = m[i];
                if (site >= su && site < sites) {
                    if (mi & 0x80u) {
                        s_ref[slot] = ((uint32_t)mi << 16) | (uint32_t)(threadIdx.x * kPer + i);
                        s_p[slot] = P;
                        s_a[slot] = A;
                        ++slot;
                    } else {
                        const int64_t pixel = site - su;
                        const uint2 raw = reinterpret_cast<const uint2 *>(rgbi)[pixel];
                        uint16_t *o = rgb_out + 3 * pixel;
                        o[0] = __ldg(ident + (raw.x & 0xFFFFu));
                        o[1] = __ldg(ident + (raw.x >> 16));
                        o[2] = __ldg(ident + (raw.y & 0xFFFFu));
                        if (changed_out) changed_out[pixel] = 0;
                    }
                }
                P += meta_base(mi);
                A += meta_amb(mi);
            }
        }
        __syncthreads();

        // ---- phase 2: attempted sites, densely ----------------------------------
        for (uint32_t k = threadIdx.x; k < listed; k += kSegThreads) {
            const uint32_t r = s_ref[k];
            const uint8_t mi = (uint8_t)(r >> 16);
            const int64_t site = seg0 + (r & 0xFFFFu);
            const uint32_t pixel = (uint32_t)(site - su);  // H*W < 2^31
            const uint32_t y = pixel / (uint32_t)w;
            const uint2 raw = reinterpret_cast<const uint2 *>(rgbi)[pixel];
            const float orig[3] = {__ldg(lut + (raw.x & 0xFFFFu)), __ldg(lut + (raw.x >> 16)),
                                   __ldg(lut + (raw.y & 0xFFFFu))};
            const bool floor_enabled = p.driver_gate_primary || stages[y + 6].gate_secondary;
            float values[3] = {orig[0], orig[1], orig[2]};
            const uint32_t Ak = s_a[k];
            const int amb = meta_amb(mi);
            const uint32_t e_before = extra_before(extra_after, Ak, capacity);
            const uint32_t extra = extra_before(extra_after, Ak + amb, capacity) - e_before;
            uint32_t state = jump_by_table(s_jump, s0, (uint64_t)s_p[k] + e_before);
            const double *cd = cand + 3 * site;
            const double c3[3] = {cd[0], cd[1], cd[2]};
            bool valid = true;
#pragma unroll
            for (int c = 0; c < 3; ++c) valid &= isfinite(c3[c]) && c3[c] > 0.0;
            uint32_t draws = 0;
            if (valid) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    int drew;
                    const DitherChannel ch = dither_channel(c3[c], p.dither_scales[c], dc);
                    const double firstd = dither_draw(ch, dc, state, drew);
                    draws += drew;
                    if (floor_enabled && c3[c] + firstd <= (double)orig[c]) {
                        values[c] = orig[c];
                    } else {
                        double d = firstd;
                        if (floor_enabled) {
                            d = dither_draw(ch, dc, state, drew);
                            draws += drew;
                        }
                        values[c] = (float)(c3[c] + d);
                    }
                }
            }
            if ((int64_t)(Ak + amb) <= capacity && draws != (uint32_t)meta_base(mi) + extra)
                raise_error(err, FX_ERR_INTERNAL);
            att += 1;
            draws_total += draws;
            written += (values[0] != orig[0] || values[1] != orig[1] || values[2] != orig[2]);
            const uint16_t e0[3] = {__ldg(ident + (raw.x & 0xFFFFu)), __ldg(ident + (raw.x >> 16)),
                                    __ldg(ident + (raw.y & 0xFFFFu))};
            uint16_t e[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                e[c] = e0[c];
                if (!(values[c] == orig[c])) ok &= emit_one(values[c], hi, lo, e[c]);
            }
            const bool ch = (e[0] != e0[0]) || (e[1] != e0[1]) || (e[2] != e0[2]);
            changed += ch;
            uint16_t *o = rgb_out + 3 * (int64_t)pixel;
            o[0] = e[0];
            o[1] = e[1];
            o[2] = e[2];
            if (changed_out) changed_out[pixel] = ch ? 1 : 0;
        }
    }
    if (!ok) raise_error(err, FX_ERR_NONFINITE_WORK);
    // the four counters in one reduction: warps, then thread 0
    unsigned long long v4[4] = {att, written, changed, draws_total};
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v4[q] += __shfl_down_sync(0xFFFFFFFFu, v4[q], o);
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q) s_sums[threadIdx.x >> 5][q] = v4[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t4[4] = {0, 0, 0, 0};
        for (int wq = 0; wq < kSegThreads / 32; ++wq)
#pragma unroll
            for (int q = 0; q < 4; ++q) t4[q] += s_sums[wq][q];
        if (t4[0]) atomicAdd(&ctr->attempted, t4[0]);
        if (t4[1]) atomicAdd(&ctr->written, t4[1]);
        if (t4[2]) atomicAdd(&ctr->changed, t4[2]);
        if (t4[3]) atomicAdd(&ctr->public_advances, t4[3]);
    }
}

__global__ void k_final(const uint32_t *__restrict__ seg_base, const uint32_t *__restrict__ seg_amb,
                        int64_t segments, const uint32_t *__restrict__ extra_after, uint32_t s0,
                        DevCounters *ctr, uint32_t *err, int64_t capacity) {
    if (pass_stopped(err)) return;
    const uint32_t p_total = seg_base[segments];
    const uint32_t a_total = seg_amb[segments];
    const uint32_t e_total = extra_before(extra_after, a_total, capacity);
    ctr->n_amb = a_total;
    ctr->final_state = lcg_jump(s0, (uint64_t)p_total + e_total);
    const unsigned long long expect =
        (unsigned long long)(p_total - ctr->startup_base) + (e_total - ctr->startup_extra);
    if ((int64_t)a_total <= capacity && expect != ctr->public_advances)
        raise_error(err, FX_ERR_INTERNAL);
}

// ---------------------------------------------------------------------------
// Launcher
// ---------------------------------------------------------------------------

cudaError_t launch_writer(const Geometry &g, const uint8_t *meta, const double *cand,
                          const uint16_t *rgbi, const float *lut, const uint32_t *high,
                          const uint32_t *low, const uint16_t *ident, const fx_stage *stages,
                          const fx_params &p,
                          uint32_t s0, const WriterBuffers &b, uint16_t *rgb_out,
                          uint8_t *changed_out, uint32_t *err, cudaStream_t stream,
                          const Marks &marks) {
    const int64_t segs = g.segments;
    DevCounters *ctr = reinterpret_cast<DevCounters *>(b.counters);
    cudaMemsetAsync(ctr, 0, sizeof(DevCounters), stream);
    cudaError_t e = launch_gate(b.cancel, err, stream);
    if (e != cudaSuccess) return e;
    // the chain and the walk are latency-bound: launched with b.priority, so
    // that with several frames in flight their blocks are dispatched ahead
    // of other frames' stencil and apply blocks, which fill the SMs they
    // leave idle
    const int pr = b.priority;
    const unsigned seg_blocks = (unsigned)((segs + kSegWarps - 1) / kSegWarps);
    e = launch_prio(k_seg_sums, dim3(seg_blocks), dim3(kSegWarps * 32), 0, stream, pr, meta,
                    g.sites, segs, b.seg_raw, err);
    if (e != cudaSuccess) return e;
    e = launch_prio(k_seg_scan, dim3(1), dim3(1024), 0, stream, pr, b.seg_raw, segs, b.seg_base,
                    b.seg_amb, err);
    if (e != cudaSuccess) return e;
    // the site list lives in extra_after until the walk writes the counts
    e = launch_prio(k_amb, dim3(seg_blocks), dim3(kSegWarps * 32), 0, stream, pr, meta, g.sites,
                    segs, b.seg_raw, b.seg_base, b.seg_amb, b.extra_after, b.pos, b.capacity,
                    err);
    if (e != cudaSuccess) return e;
    const uint32_t *n_amb = b.seg_amb + segs;
    cudaMemsetAsync(b.chunk_two, 0, walk_chunks(b.capacity), stream);
    unsigned long long *seg_copy, *seg_spread;
    size_t stat_bytes;
    walk_segment_stats(b.walk_scratch, b.capacity, &seg_copy, &seg_spread, &stat_bytes);
    cudaMemsetAsync(seg_copy, 0, stat_bytes, stream);
    cudaMemsetAsync(seg_spread, 0, stat_bytes, stream);
    e = launch_prio(k_coef, dim3(1184), dim3(256), 0, stream, pr, b.entries, b.pos, n_amb,
                    b.capacity, b.extra_after, meta, cand, g.w, rgbi, lut, p, err, b.chunk_two,
                    seg_copy, seg_spread);
    if (e != cudaSuccess) return e;
    marks.mark(5, stream);
    e = launch_gate(b.cancel, err, stream);
    if (e != cudaSuccess) return e;
    e = launch_walk(b.entries, b.pos, n_amb, b.capacity, s0, b.walk_scratch, b.per_wave,
                    b.parallel_walk, b.window_sigmas, b.chunk_two, b.extra_after,
                    &ctr->walk_fallbacks, ctr->walk_stats, err, stream, pr);
    if (e != cudaSuccess) return e;
    marks.mark(6, stream);
    e = launch_gate(b.cancel, err, stream);
    if (e != cudaSuccess) return e;
    k_startup_counts<<<6, 256, 0, stream>>>(meta, g.w, b.extra_after, s0 & kLcgMask, ctr,
                                            b.capacity, err);
    k_apply<<<(unsigned)std::min<int64_t>(segs, g_apply_blocks), kSegThreads, 0, stream>>>(
        meta, cand, g.sites, g.w, rgbi, lut, high, low, ident, stages, p, b.seg_base, b.seg_amb,
        b.extra_after, s0 & kLcgMask, rgb_out, changed_out, ctr, err, b.capacity);
    k_final<<<1, 1, 0, stream>>>(b.seg_base, b.seg_amb, segs, b.extra_after, s0 & kLcgMask,
                                 ctr, err, b.capacity);
    marks.mark(7, stream);
    return cudaGetLastError();
}

// One thread: a cancel request seen here stops every later kernel of the pass.
__global__ void k_gate(const volatile uint32_t *cancel, uint32_t *err) {
    if (*cancel && err[1] == 0u) {
        err[1] = 1u;
        atomicCAS(err, 0u, (uint32_t)FX_ERR_CANCELLED);
    }
}

cudaError_t launch_gate(const uint32_t *cancel, uint32_t *err, cudaStream_t stream) {
    if (!cancel) return cudaSuccess;
    k_gate<<<1, 1, 0, stream>>>(cancel, err);
    return cudaGetLastError();
}

size_t dev_counters_bytes() { return sizeof(DevCounters); }

void counters_to_host(const void *dev_copy, fx_counters *out) {
    const DevCounters &c = *reinterpret_cast<const DevCounters *>(dev_copy);
    out->attempted = (int64_t)c.attempted;
    out->written = (int64_t)c.written;
    out->public_advances = (int64_t)c.public_advances;
    out->changed = (int64_t)c.changed;
    out->final_state = c.final_state;
    out->startup_final_state = c.su_final_state;
    for (int k = 0; k < 6; ++k) {
        out->startup_attempted[k] = (int64_t)c.su_attempted[k];
        out->startup_advances[k] = (int64_t)c.su_advances[k];
    }
    out->rng_dependent = (int64_t)c.n_amb;
    out->walk_fallbacks = (int64_t)c.walk_fallbacks;
    out->walk_candidate_steps = (int64_t)c.walk_stats[0];
    out->walk_candidates = (int64_t)c.walk_stats[1];
    out->walk_survivors = (int64_t)c.walk_stats[2];
    out->walk_packed_segments = (int64_t)c.walk_packed;
    out->capacity_reruns = 0;  // set by the host when the pass runs again
}

uint32_t counters_n_amb(const void *dev_copy) {
    return reinterpret_cast<const DevCounters *>(dev_copy)->n_amb;
}

}  // namespace fx
