// fx_walk.cu -- the serial RNG walk, parallelised by speculation.
//
// The chain of RNG-dependent channels (see fx_writer.cu) is a function of
// one integer: E_i, the number of extra draws before channel i.  The state
// at channel i's first draw is T_i = G^(pos_i + 1 + E_i)(T0) (G = one LCG step
// in T space), the channel draws an extra time iff T_i misses its copy
// intervals, and E_{i+1} = E_i + extra_i.  So a segment of channels maps an
// entry count E_in to an exit count E_out, and:
//   * two candidates E < E' keep their order and merge for good once equal
//     (E'_k - E_k moves by -1, 0 or +1 per channel), so merges only ever
//     happen between neighbours in E order;
//   * candidates merge quickly (the gap is a lazy random walk absorbed at 0).
//
// A wave of segments is one launch of k_wave.  Its window blocks each walk
// one segment for a window of candidate E_in values around the predicted
// value (expected extras from the exact state-space measure of every copy
// set, summed per segment by k_coef), merging candidates as they meet and
// compacting the survivors, and
// write a dense E_in -> E_out table and a compact survivor list.  Block 0
// chains the exact E through the wave with one list read per segment, each
// segment as soon as its window block has finished (per-segment completion
// flags); when E falls outside a window it walks that segment exactly, so
// correctness never depends on the prediction.  k_rewalk then walks every
// segment in parallel from its exact E_in and writes the running extra
// count per channel.  With one segment covering the whole chain, k_rewalk
// alone is the plain serial walk.
#include "fx_internal.cuh"

namespace fx {

constexpr int kWinThreads = 256;
constexpr int kWinBlocksPerSM = 3;                  // three segments resident per SM
constexpr int kWinSlots = 16;                       // candidates per thread
constexpr int kWinMax = kWinThreads * kWinSlots;    // 4096 candidates
constexpr uint32_t kSegLen = kWalkSegLen;           // channels per walk segment
constexpr int kWinChunk = kWalkChunk;               // channels staged per chunk
constexpr int kWinRing = 3;                         // staged chunks in flight
constexpr uint32_t kCompactEvery = 512;             // block compaction period (steady state)
constexpr uint32_t kSettledCompactEvery = 512;      // the same once at most 256 are left
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint32_t kSerialBelow = 4 * kSegLen;      // short chains: one serial walk
// The window half-width is kDefaultWindowSigmas (4.5) standard deviations of
// the predicted entry count, plus 16.  A count outside its window costs one
// exact serial walk of that segment (about 40 us) and never changes a
// result; at 4.5 sigma that happens for about 7e-6 of the segments.
// fx_set_walk_window narrows it, so tests can force such misses.

struct WalkState {
    uint32_t e_wave;     // exact E at the start of the current wave
    uint32_t waves;
    uint32_t fallbacks;  // segments resolved by an exact serial walk
    uint32_t packed;     // segments whose settled phase ran two candidates per lane
    unsigned long long candidate_steps;  // window-walk work, for diagnostics
    unsigned long long window_sum;       // candidates started
    unsigned long long survivor_sum;     // candidates left at segment ends
};

struct SegWindow {
    uint32_t lo, hi;  // candidate E_in range, inclusive
};

__device__ __forceinline__ uint32_t jump_t(uint32_t t0, uint64_t n) {
    const Affine f = lcg_power_t(n);
    return f.a * t0 + f.c;
}

// Steps n with G^n(from) = to (T space, 24-bit state in the high bits), by
// matching one bit per round: G^(2^j) leaves the bits below j unchanged and
// flips bit j (full-period LCG: multiplier 1 mod 4, odd increment).
__device__ __forceinline__ uint32_t lcg_distance_t(uint32_t from_t, uint32_t to_t) {
    uint32_t cur = from_t >> 8, target = to_t >> 8, a = 125u, c = 1u, d = 0u;
#pragma unroll
    for (int j = 0; j < 24; ++j) {
        const uint32_t bit = 1u << j;
        if ((cur ^ target) & bit) {
            cur = (a * cur + c) & 0xFFFFFFu;
            d |= bit;
        }
        c = (a + 1u) * c;
        a = a * a;
    }
    return d;
}

__device__ __forceinline__ bool copies(const uint4 &lw, uint32_t T) {
    return ((T - lw.x) <= lw.y) | ((T - lw.z) <= lw.w);
}

// The copy test of an entry whose copy set is one (cyclic) interval: the
// second interval is the empty marker, so its test is always false.
template <bool TWO>
__device__ __forceinline__ bool copies_of(const uint4 &lw, uint32_t T) {
    return TWO ? copies(lw, T) : ((T - lw.x) <= lw.y);
}

__device__ __forceinline__ uint4 intervals(const AmbEntry &e) {
    return make_uint4(e.l1, e.w1, e.l2, e.w2);
}

// ---------------------------------------------------------------------------
// Block scans over 1024 threads
// ---------------------------------------------------------------------------

// Exclusive "last valid value" scan in thread order (kNone = no value);
// `total` receives the inclusive result of the whole block.
__device__ __forceinline__ uint32_t last_valid_exclusive(uint32_t v, uint32_t *buf,
                                                         uint32_t &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o && x == kNone) x = y;
    }
    constexpr int kWarps = kWinThreads / 32;
    if (lane == 31) buf[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < kWarps ? buf[lane] : kNone;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o && s == kNone) s = y;
        }
        if (lane < kWarps) buf[lane] = s;
    }
    __syncthreads();
    uint32_t before = __shfl_up_sync(0xFFFFFFFFu, x, 1);
    if (lane == 0) before = kNone;
    if (before == kNone && warp > 0) before = buf[warp - 1];
    total = buf[kWarps - 1];
    __syncthreads();
    return before;
}

__device__ __forceinline__ uint32_t add_exclusive(uint32_t v, uint32_t *buf, uint32_t &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    constexpr int kWarps = kWinThreads / 32;
    if (lane == 31) buf[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < kWarps ? buf[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kWarps) buf[lane] = s;
    }
    __syncthreads();
    const uint32_t prefix = warp ? buf[warp - 1] : 0u;
    total = buf[kWarps - 1];
    __syncthreads();
    return prefix + x - v;
}

// ---------------------------------------------------------------------------
// Window walk
// ---------------------------------------------------------------------------

constexpr int kListMax = 256;  // survivors kept in the compact per-segment list

// Compact result of one window: survivors in E_in order as 16-bit offsets
// (E_in - lo, E_out - lo); count == 0xFFFF means "use the dense table".
struct __align__(16) SegList {
    uint32_t count;
    uint32_t pad[3];
    uint16_t ein[kListMax];
    uint16_t eout[kListMax];
};
static_assert(sizeof(SegList) % 16 == 0, "SegList is staged with 16-byte copies");

struct WindowSmem {
    AmbEntry ring[kWinRing][kWinChunk + 1];
    uint32_t ein[kWinMax], e[kWinMax], t[kWinMax];  // survivors in E_in order
    uint32_t buf[32];
    uint32_t wlast[kWinSlots * (kWinThreads / 32)];   // per warp-slot, list order
    uint32_t wcount[kWinSlots * (kWinThreads / 32)];
    double pred[2];
};
static_assert(kWinSlots * (kWinThreads / 32) <= 256, "prefix covers 8 entries per lane");
static_assert(kWinSlots <= 32, "live mask is 32 bits");

// One warp steps its candidates over LEN staged channels.  The entries do
// not depend on the candidates, so all LEN are loaded first and the
// dependent chain per channel is compare -> select -> multiply-add.  Dead
// candidates (merged into a neighbour) keep stepping: their values are
// never read again, and skipping them would put a divergent branch on every
// step.
template <int SLOTS, int LEN, bool TWO>
__device__ __forceinline__ void walk_group(const uint4 *r4, uint32_t r, bool tail_next,
                                           uint32_t (&rT)[kWinSlots], uint32_t live_mask,
                                           uint32_t &steps) {
    uint4 lw[LEN], ac[LEN];
#pragma unroll
    for (int k = 0; k < LEN; ++k) {
        lw[k] = r4[2 * (r + k)];
        const bool next = (k + 1 < LEN) || tail_next;
        ac[k] = r4[2 * (r + k + (next ? 1 : 0)) + 1];
    }
    steps += (uint32_t)__popc(live_mask & ((1u << SLOTS) - 1u)) * LEN;
#pragma unroll
    for (int k = 0; k < LEN; ++k) {
#pragma unroll
        for (int s = 0; s < SLOTS; ++s)
            rT[s] = copies_of<TWO>(lw[k], rT[s]) ? ac[k].x * rT[s] + ac[k].y
                                                 : ac[k].z * rT[s] + ac[k].w;
    }
}

// Single channels (segment and compaction boundaries).
template <int SLOTS, bool TWO>
__device__ __forceinline__ void walk_one(const uint4 *r4, uint32_t r, bool has_next,
                                         uint32_t (&rT)[kWinSlots], uint32_t live_mask,
                                         uint32_t &steps) {
    const uint4 lw = r4[2 * r];
    const uint4 ac = r4[2 * (r + (has_next ? 1u : 0u)) + 1];
    steps += (uint32_t)__popc(live_mask & ((1u << SLOTS) - 1u));
#pragma unroll
    for (int s = 0; s < SLOTS; ++s)
        rT[s] = copies_of<TWO>(lw, rT[s]) ? ac.x * rT[s] + ac.y : ac.z * rT[s] + ac.w;
}

// Warp-local merge: lanes of one slot hold consecutive candidates; equal
// states mean equal counts.
template <int SLOTS>
__device__ __forceinline__ void warp_merge(const uint32_t (&rT)[kWinSlots], uint32_t &live_mask) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) {
        const bool alive = live_mask & (1u << s);
        uint32_t x = alive ? rT[s] : kNone;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o && x == kNone) x = y;
        }
        uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, x, 1);
        if (lane == 0) prev = kNone;
        if (alive && rT[s] == prev) live_mask &= ~(1u << s);
    }
}

// Walk channels [r, stop) of the staged ring for one warp.  TWO: some entry
// of the staged chunk has two copy intervals.
template <int SLOTS, bool TWO>
__device__ __forceinline__ void walk_span(const uint4 *r4, uint32_t r, uint32_t stop,
                                          bool end_next, uint32_t merge_len,
                                          uint32_t (&rT)[kWinSlots], uint32_t &live_mask,
                                          uint32_t &steps) {
    // many slots give their own parallelism: stage fewer channels at once
    constexpr int kLen = SLOTS == 1 ? 16 : (SLOTS <= 2 ? 8 : (SLOTS <= 8 ? 4 : 2));
    uint32_t since = 0;
    while (r < stop) {
        if (r + kLen <= stop) {
            const bool tail_next = (r + kLen < stop) || end_next;
            walk_group<SLOTS, kLen, TWO>(r4, r, tail_next, rT, live_mask, steps);
            r += kLen;
            since += kLen;
        } else {
            const bool has_next = (r + 1 < stop) || end_next;
            walk_one<SLOTS, TWO>(r4, r, has_next, rT, live_mask, steps);
            r += 1;
            since += 1;
        }
        if (since >= merge_len || r == stop) {
            warp_merge<SLOTS>(rT, live_mask);
            since = 0;
        }
    }
}

// Slots per lane for `live` candidates.  Warp w holds list positions
// [w * slots * 32, (w + 1) * slots * 32).  Above kWinThreads candidates every
// warp walks; at most kWinThreads left (the settled phase), more than 32 of
// them are packed two per lane into the fewest warps: two slots in four
// warps measured 1.48x the candidate-step rate of one slot in eight (three
// blocks per SM, 4096 channels), and warps with no candidate left do not
// step.
__device__ __forceinline__ int window_slots(uint32_t live) {
    if (live <= (uint32_t)kWinThreads) return live > 32u ? 2 : 1;
    const uint32_t s = (live + kWinThreads - 1u) / kWinThreads;
    return s > (uint32_t)kWinSlots ? kWinSlots : (int)s;
}

// Release / acquire of the per-segment completion flags (gpu scope).
__device__ __forceinline__ void flag_release(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t flag_acquire(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// One segment's window walk: block blk of the wave (segment seg0 + blk).
// When its table, list and window are written it releases flags[blk] = tag,
// which the wave's resolve block waits for.
__device__ __forceinline__ void window_block(
    const AmbEntry *__restrict__ entries, const uint32_t *__restrict__ pos, uint32_t n,
    const unsigned long long *__restrict__ seg_copy,
    const unsigned long long *__restrict__ seg_spread, const WalkState *st, uint32_t wave, uint32_t per_wave, uint32_t t0,
    SegWindow *__restrict__ windows, uint32_t *__restrict__ table, SegList *__restrict__ lists,
    WalkState *stats, double sigmas, const uint8_t *__restrict__ chunk_two, uint32_t blk,
    uint32_t *flags, uint32_t tag) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WindowSmem &S = *reinterpret_cast<WindowSmem *>(smem_raw);
    const uint32_t seg0 = wave * per_wave;
    const uint32_t j = seg0 + blk;
    const uint32_t i0 = j * kSegLen;
    if (i0 >= n) return;
    const uint32_t i1 = min(n, i0 + kSegLen);
    const uint32_t tid = threadIdx.x;

    // window of candidate entry counts around the prediction
    if (tid < 32) {  // the prediction only centres the window: any summation order
        // every segment before j is full: kSegLen channels, each drawing an
        // extra with probability p = 1 - copying states / 2^24
        double mu = 0.0, var = 0.0;
        for (uint32_t k = seg0 + tid; k < j; k += 32) {
            mu += (double)kSegLen - (double)seg_copy[k] * 0x1p-24;
            var += (double)seg_spread[k] * 0x1p-26;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mu += __shfl_down_sync(0xFFFFFFFFu, mu, o);
            var += __shfl_down_sync(0xFFFFFFFFu, var, o);
        }
        if (tid == 0) {
            S.pred[0] = mu;
            S.pred[1] = var;
        }
    }
    __syncthreads();
    const uint32_t e0 = st->e_wave;
    const uint32_t before = i0 - seg0 * kSegLen;  // channels since the wave start
    const double half = sigmas * sqrt(S.pred[1]) + 16.0;
    const double center = S.pred[0];
    int64_t lo = (int64_t)floor(center - half), hi = (int64_t)ceil(center + half);
    lo = lo < 0 ? 0 : lo;
    hi = hi > (int64_t)before ? (int64_t)before : hi;
    if (hi < lo) hi = lo;
    if (hi - lo + 1 > kWinMax) {
        lo = (int64_t)center - kWinMax / 2;
        lo = lo < 0 ? 0 : lo;
        hi = lo + kWinMax - 1;
        if (hi > (int64_t)before) {
            hi = before;
            lo = hi - kWinMax + 1;
        }
    }
    const uint32_t wlo = e0 + (uint32_t)lo;
    const uint32_t count = (uint32_t)(hi - lo + 1);

    // candidates in list order k = (warp * slots + slot) * 32 + lane; E_in of
    // the candidate at list position k is S.ein[k] (kept in shared memory)
    uint32_t rT[kWinSlots];
    uint32_t live_mask = 0;
    uint32_t live = count;
    int slots = window_slots(live);
    {
        const uint32_t k0 = (tid >> 5) * (uint32_t)slots * 32u + (tid & 31u);
        uint32_t t = jump_t(t0, (uint64_t)pos[i0] + 1u + wlo + k0);
        const Affine stride = lcg_power_t(32);
#pragma unroll
        for (int s = 0; s < kWinSlots; ++s) {
            rT[s] = 0;
            if (s < slots) {
                const uint32_t k = k0 + (uint32_t)s * 32u;
                rT[s] = t;
                if (k < live) live_mask |= 1u << s;
                S.ein[k] = wlo + k;
                t = stride.a * t + stride.c;
            }
        }
    }

    auto stage = [&](uint32_t first, int b) {
        const uint32_t avail = min((uint32_t)kWinChunk + 1u, n - first);
        const uint4 *src = reinterpret_cast<const uint4 *>(entries + first);
        uint4 *dst = reinterpret_cast<uint4 *>(S.ring[b]);
        for (uint32_t v = tid; v < 2 * avail; v += kWinThreads) {
            const uint32_t sa = (uint32_t)__cvta_generic_to_shared(dst + v);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(src + v));
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };

    // Block-wide merge and compaction.  List order is warp-major
    // (k = (warp * slots + slot) * 32 + lane) and E is non-decreasing along it.  The
    // candidates carry only their state T: at one channel, equal T means
    // equal E (distinct counts of one window are far closer than the LCG's
    // 2^24 period).  After warp_merge the live values of one warp-slot are
    // distinct, so only its first live lane can equal the last live value
    // before it.
    auto merge_and_compact = [&](int slots) {
        const int lane = tid & 31, warp = tid >> 5;
        constexpr int kW = kWinThreads / 32;
        uint32_t ein[kWinSlots];
        // 1. last live value of every warp-slot
#pragma unroll
        for (int s = 0; s < kWinSlots; ++s) {
            if (s < slots) {  // block-uniform
                const bool alive = live_mask & (1u << s);
                const uint32_t bal = __ballot_sync(0xFFFFFFFFu, alive);
                const uint32_t last = bal ? __shfl_sync(0xFFFFFFFFu, rT[s], 31 - __clz(bal)) : kNone;
                if (lane == 0) S.wlast[warp * slots + s] = last;
                if (alive) ein[s] = S.ein[(warp * slots + s) * 32 + lane];
            }
        }
        __syncthreads();
        // 2. drop a first live lane that repeats the previous warp-slots' last
        //    value; publish the live counts
#pragma unroll
        for (int s = 0; s < kWinSlots; ++s) {
            if (s < slots) {
                const bool alive = live_mask & (1u << s);
                const uint32_t bal = __ballot_sync(0xFFFFFFFFu, alive);
                if (bal && lane == __ffs(bal) - 1) {
                    uint32_t prev = kNone;
                    for (int q = warp * slots + s - 1; q >= 0; --q) {
                        const uint32_t v = S.wlast[q];
                        if (v != kNone) {
                            prev = v;
                            break;
                        }
                    }
                    if (prev == rT[s]) live_mask &= ~(1u << s);
                }
                const uint32_t cnt = __popc(__ballot_sync(0xFFFFFFFFu, live_mask & (1u << s)));
                if (lane == 0) S.wcount[warp * slots + s] = cnt;
            }
        }
        __syncthreads();
        // 3. exclusive prefix of the counts in list order (every warp computes
        //    it; lane l covers entries 8l..8l+7), then scatter
        const int entries = slots * kW;
        uint32_t lsum = 0;
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int q = lane * 8 + m;
            lsum += (q < entries) ? S.wcount[q] : 0u;
        }
        uint32_t incl = lsum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t excl = incl - lsum;
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
#pragma unroll
        for (int s = 0; s < kWinSlots; ++s) {
            if (s < slots) {
                const int q = warp * slots + s;
                uint32_t base = __shfl_sync(0xFFFFFFFFu, excl, q >> 3);
#pragma unroll
                for (int m = 0; m < 7; ++m)
                    if (m < (q & 7)) base += S.wcount[(q & ~7) + m];
                const bool alive = live_mask & (1u << s);
                const uint32_t bal = __ballot_sync(0xFFFFFFFFu, alive);
                if (alive) {
                    const uint32_t at = base + __popc(bal & ((1u << lane) - 1u));
                    S.ein[at] = ein[s];
                    S.t[at] = rT[s];
                }
            }
        }
        __syncthreads();
        // reload in the layout of the new slot count (the caller's next
        // window_slots(live) is the same value)
        live = total;
        live_mask = 0;
        const int next_slots = window_slots(total);
#pragma unroll
        for (int s = 0; s < kWinSlots; ++s) {
            if (s < next_slots) {
                const uint32_t k = (uint32_t)((warp * next_slots + s) * 32 + lane);
                if (k < live) {
                    live_mask |= 1u << s;
                    rT[s] = S.t[k];
                }
            }
        }
    };

    uint32_t steps = 0;
    bool packed = false;  // the settled phase ran two candidates per lane
    // Three staged chunks: chunk c+2 is fetched into the buffer of chunk c-1
    // right after the barrier that ends every warp's work on chunk c-1.
    stage(i0, 0);
    if (i0 + kWinChunk < i1) stage(i0 + kWinChunk, 1);
    else asm volatile("cp.async.commit_group;\n" ::);
    int b = 0;
    uint32_t next_compact = 8;  // then 16, 32, ..., every kCompactEvery channels
    // Walk channels [i0, iw): every candidate ends at the state of the last
    // channel iw, whose extra draw is added when the counts are recovered.
    const uint32_t iw = i1 - 1;
    for (uint32_t c0 = i0; c0 < iw; c0 += kWinChunk) {
        const uint32_t c1 = min(iw, c0 + (uint32_t)kWinChunk);
        asm volatile("cp.async.wait_group 1;\n" ::);
        __syncthreads();
        const uint32_t c2 = c0 + 2 * kWinChunk;
        if (c2 < i1) stage(c2, (b + 2) % kWinRing);
        else asm volatile("cp.async.commit_group;\n" ::);
        const uint4 *r4 = reinterpret_cast<const uint4 *>(S.ring[b]);
        uint32_t r = 0;
        const uint32_t len = c1 - c0;
        const bool two = chunk_two[c0 / kWinChunk] != 0;  // block-uniform
        while (r < len) {
            const uint32_t done0 = (c0 - i0) + r;
            const uint32_t stop =
                min(len, r + (next_compact > done0 ? next_compact - done0 : len));
            const bool end_next = (c0 + stop) < i1;
            // at most one candidate per thread: only the span ends merge
            // (duplicates step in lanes that run anyway); otherwise warps
            // merge every 16 channels, then every 32
            const bool settled = live <= (uint32_t)kWinThreads;
            const uint32_t merge_len = settled ? kSegLen : ((done0 < 256u) ? 16u : 32u);
            if (__any_sync(0xFFFFFFFFu, live_mask != 0)) {
                switch (slots) {
#define FX_WALK_CASE(K)                                                                         \
    case K:                                                                                     \
        if (two) walk_span<K, true>(r4, r, stop, end_next, merge_len, rT, live_mask, steps);    \
        else walk_span<K, false>(r4, r, stop, end_next, merge_len, rT, live_mask, steps);       \
        break;
                    FX_WALK_CASE(1) FX_WALK_CASE(2) FX_WALK_CASE(3) FX_WALK_CASE(4)
                    FX_WALK_CASE(5) FX_WALK_CASE(6) FX_WALK_CASE(7) FX_WALK_CASE(8)
                    FX_WALK_CASE(9) FX_WALK_CASE(10) FX_WALK_CASE(11) FX_WALK_CASE(12)
                    FX_WALK_CASE(13) FX_WALK_CASE(14) FX_WALK_CASE(15)
                default:
                    if (two) walk_span<16, true>(r4, r, stop, end_next, merge_len, rT, live_mask, steps);
                    else walk_span<16, false>(r4, r, stop, end_next, merge_len, rT, live_mask, steps);
                    break;
#undef FX_WALK_CASE
                }
            }
            r = stop;
            const uint32_t done = (c0 - i0) + r;
            if (done >= next_compact || c0 + r == iw) {
                merge_and_compact(slots);
                slots = window_slots(live);
                packed |= live <= (uint32_t)kWinThreads && slots == 2;
                // settled: compact every kSettledCompactEvery channels, so
                // warps drop out as duplicates merge
                next_compact = live <= (uint32_t)kWinThreads
                                   ? min(iw - i0, done + kSettledCompactEvery)
                                   : min(2 * next_compact, done + kCompactEvery);
            }
        }
        b = (b + 1) % kWinRing;
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncthreads();
    if (iw == i0) merge_and_compact(slots);  // one-channel segment: nothing walked

    // Exit counts: a survivor's state at channel iw is G^(pos_iw + 1 + E)(t0),
    // so E - wlo is its LCG distance from the state of count wlo (exact: the
    // difference is below count + kSegLen, far under the 2^24 period); the
    // last channel adds its extra draw.  Channel iw's entry is still staged
    // (chunk q of the ring, whose buffer no later staging reused).
    {
        const uint32_t q = (iw - i0) / kWinChunk;
        const uint4 lw_last = reinterpret_cast<const uint4 *>(S.ring[q % kWinRing])
            [2 * ((iw - i0) % kWinChunk)];
        const uint32_t t_ref = jump_t(t0, (uint64_t)pos[iw] + 1u + wlo);
        for (uint32_t k = tid; k < live; k += kWinThreads) {
            const uint32_t t = S.t[k];
            S.e[k] = wlo + lcg_distance_t(t_ref, t) + (copies(lw_last, t) ? 0u : 1u);
        }
    }

    // Outputs.  Survivors sit compacted in S.* in E_in order.
    uint32_t *out = table + (size_t)blk * kWinMax;
    for (uint32_t k = tid; k < live; k += kWinThreads) {
        const uint32_t from = S.ein[k] - wlo;
        const uint32_t to = (k + 1 < live) ? S.ein[k + 1] - wlo : count;
        const uint32_t value = S.e[k];
        for (uint32_t m = from; m < to; ++m) out[m] = value;
    }
    SegList *list = lists + blk;
    if (live <= (uint32_t)kListMax) {
        for (uint32_t k = tid; k < live; k += kWinThreads) {
            list->ein[k] = (uint16_t)(S.ein[k] - wlo);
            list->eout[k] = (uint16_t)(S.e[k] - wlo);
        }
    }
    if (tid == 0) {
        windows[blk] = SegWindow{wlo, wlo + count - 1};
        list->count = (live <= (uint32_t)kListMax) ? live : 0xFFFFu;
        atomicAdd(&stats->window_sum, (unsigned long long)count);
        atomicAdd(&stats->survivor_sum, (unsigned long long)live);
        if (packed) atomicAdd(&stats->packed, 1u);
    }
    for (int o = 16; o > 0; o >>= 1) steps += __shfl_down_sync(0xFFFFFFFFu, steps, o);
    if ((tid & 31) == 0 && steps) atomicAdd(&stats->candidate_steps, (unsigned long long)steps);
    __syncthreads();  // every output of the segment is written
    if (tid == 0) {
        __threadfence();
        flag_release(flags + blk, tag);
    }
}

// Exact serial walk of one segment from a known entry count (the fallback).
__device__ uint32_t walk_segment_exact(const AmbEntry *entries, const uint32_t *pos, uint32_t i0,
                                       uint32_t i1, uint32_t e_in, uint32_t t0) {
    uint32_t T = jump_t(t0, (uint64_t)pos[i0] + 1u + e_in);
    uint32_t E = e_in;
    for (uint32_t i = i0; i < i1; ++i) {
        const uint32_t x = copies(intervals(entries[i]), T) ? 0u : 1u;
        E += x;
        if (i + 1 < i1) {
            const AmbEntry nx = entries[i + 1];
            T = x ? nx.a1 * T + nx.c1 : nx.a0 * T + nx.c0;
        }
    }
    return E;
}

// Resolve one wave: chain the exact E through its segments.  The compact
// survivor lists stream through shared memory in chunks (warps 1.. stage
// chunk c+1 while warp 0 chains chunk c), so each hop is a warp-reduced count
// of survivors at or below E, from registers loaded ahead; a segment whose list overflowed uses its dense table, and
// E outside a window walks the segment exactly.
// A hop the survivor list cannot answer: a list that overflowed (dense
// table) or E outside the window (exact walk of the segment).  Kept out of
// line so the resolve loop stays short.
__device__ __noinline__ uint32_t resolve_off_list(const AmbEntry *entries, const uint32_t *pos,
                                                  uint32_t n, uint32_t t0, const uint32_t *table,
                                                  SegWindow win, uint32_t E, uint32_t j,
                                                  uint32_t b, uint32_t &fallbacks) {
    if (E >= win.lo && E <= win.hi) return __ldcg(table + (size_t)b * kWinMax + (E - win.lo));
    const uint32_t i0 = j * kSegLen, i1 = min(n, i0 + kSegLen);
    fallbacks += 1;
    return walk_segment_exact(entries, pos, i0, i1, E, t0);
}

// The resolve block of a wave stages the segments' lists in chunks of
// kResolveChunk (two chunks in flight within the window kernel's shared
// memory): warps 1..7 wait for a chunk's window blocks and copy it while
// warp 0 chains the previous chunk.
constexpr int kResolveChunk = 32;
constexpr int kStageWarps = kWinThreads / 32 - 1;
// A wait for a window block gives up after kFlagSpins polls about 128 ns
// apart (about half a second), sets an error and stops the wave.
constexpr uint32_t kFlagSpins = 1u << 22;

struct ResolveSmem {
    SegList list[2][kResolveChunk];
    SegWindow win[2][kResolveChunk];
    uint32_t e_in[2][kResolveChunk];  // exact entry counts found by warp 0
    int abort;                        // a wait for a window block gave up
};
static_assert(sizeof(ResolveSmem) <= sizeof(WindowSmem),
              "the resolve block runs in a window block's shared memory");

// Resolve one wave: chain the exact E through its segments.  Hops read the
// window results only through L2 (cp.async.cg, ld.global.cg): the same
// scratch slots are rewritten every wave, and a line this SM cached in an
// earlier wave must not be read.
__device__ void resolve_block(const AmbEntry *__restrict__ entries,
                              const uint32_t *__restrict__ pos, uint32_t n, WalkState *st,
                              uint32_t wave, uint32_t per_wave, uint32_t t0,
                              const SegWindow *__restrict__ windows,
                              const uint32_t *__restrict__ table,
                              const SegList *__restrict__ lists, uint32_t *__restrict__ e_in_exact,
                              const uint32_t *flags, uint32_t tag, uint32_t *err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ResolveSmem &S = *reinterpret_cast<ResolveSmem *>(smem_raw);
    const uint32_t segs = (n + kSegLen - 1) / kSegLen;
    const uint32_t here = min(per_wave, segs > wave * per_wave ? segs - wave * per_wave : 0u);
    const uint32_t chunks = (here + kResolveChunk - 1) / kResolveChunk;
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid == 0) S.abort = 0;
    __syncthreads();
    // threads 32..255: wait (warp 1, one lane per segment) until the chunk's
    // window blocks are done, then copy the chunk
    auto stage = [&](uint32_t c) {
        const uint32_t first = c * kResolveChunk;
        const uint32_t cnt = min((uint32_t)kResolveChunk, here - first);
        if (tid < 64 && (uint32_t)lane < cnt) {
            uint32_t spins = 0;
            while (flag_acquire(flags + first + lane) != tag) {
                if (++spins > kFlagSpins) {
                    S.abort = 1;
                    raise_error(err, FX_ERR_INTERNAL);
                    break;
                }
                __nanosleep(128);
            }
        }
        asm volatile("bar.sync 1, %0;\n" ::"n"(kStageWarps * 32) : "memory");
        __threadfence();
        if (!S.abort) {
            const uint4 *src = reinterpret_cast<const uint4 *>(lists + first);
            uint4 *dst = reinterpret_cast<uint4 *>(S.list[c & 1]);
            const uint32_t vecs = cnt * (uint32_t)(sizeof(SegList) / 16);
            for (uint32_t v = tid - 32; v < vecs; v += kWinThreads - 32) {
                const uint32_t sa = (uint32_t)__cvta_generic_to_shared(dst + v);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(src + v));
            }
            for (uint32_t bb = tid - 32; bb < cnt; bb += kWinThreads - 32) {
                const uint2 wv = __ldcg(reinterpret_cast<const uint2 *>(windows + first + bb));
                S.win[c & 1][bb] = SegWindow{wv.x, wv.y};
            }
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    if (tid >= 32 && chunks > 0) stage(0);
    uint32_t E = st->e_wave;
    uint32_t fallbacks = 0;
    for (uint32_t c = 0; c < chunks; ++c) {
        if (tid >= 32) asm volatile("cp.async.wait_group 0;\n" ::);
        __syncthreads();  // chunk c visible; warp 0 is done with chunk c-1
        if (S.abort) break;
        if (tid >= 32) {
            if (c + 1 < chunks) stage(c + 1);
            continue;
        }
        // warp 0: one hop per segment; survivor E_in values are increasing
        // and the first is the window's lowest candidate
        const uint32_t first = c * kResolveChunk;
        const uint32_t cnt_c = min((uint32_t)kResolveChunk, here - first);
        // software-pipelined: hop bb+1's window and list (independent of E)
        // are loaded while hop bb resolves
        constexpr int kM = kListMax / 32;
        auto load_hop = [&](uint32_t bb, SegWindow &w, uint32_t &cnt, uint32_t (&e)[kM]) {
            w = S.win[c & 1][bb];
            const SegList *L = &S.list[c & 1][bb];
            cnt = L->count;
            const uint32_t valid = cnt != 0xFFFFu ? cnt : 0u;
#pragma unroll
            for (int m = 0; m < kM; ++m) {  // in bounds for any count: no branch
                const uint32_t k = m * 32 + lane;
                const uint32_t v = L->ein[k];
                e[m] = k < valid ? v : 0xFFFFFFFFu;
            }
        };
        SegWindow win{};
        uint32_t cnt = 0, ein[kM];
        if (cnt_c) load_hop(0, win, cnt, ein);
        for (uint32_t bb = 0; bb < cnt_c; ++bb) {
            SegWindow nwin{};
            uint32_t ncnt = 0, nein[kM];
            if (bb + 1 < cnt_c) load_hop(bb + 1, nwin, ncnt, nein);
            S.e_in[c & 1][bb] = E;  // every lane writes the same value
            // the list lookup runs unconditionally (an E outside the window
            // reads an in-bounds but meaningless entry, discarded below), so
            // the rare-case test is off the dependent path
            const uint32_t q = E - win.lo;
            uint32_t mine = 0;  // this lane's entries at or below q
#pragma unroll
            for (int m = 0; m < kM; ++m) mine += ein[m] <= q;
            const uint32_t below = __reduce_add_sync(0xFFFFFFFFu, mine);
            const uint32_t fast = win.lo + S.list[c & 1][bb].eout[(below - 1) & (kListMax - 1)];
            const bool listed = E >= win.lo && E <= win.hi && cnt != 0xFFFFu && cnt > 0;
            if (!listed)  // rare: every lane computes the same value, out of line
                E = resolve_off_list(entries, pos, n, t0, table, win, E,
                                     wave * per_wave + first + bb, first + bb, fallbacks);
            else
                E = fast;
            win = nwin;
            cnt = ncnt;
#pragma unroll
            for (int m = 0; m < kM; ++m) ein[m] = nein[m];
        }
        __syncwarp();
        for (uint32_t bb = lane; bb < cnt_c; bb += 32)
            e_in_exact[wave * per_wave + first + bb] = S.e_in[c & 1][bb];
    }
    if (tid == 0 && !S.abort) {
        st->e_wave = E;
        st->waves += 1;
        st->fallbacks += fallbacks;
    }
}

// One wave of the speculative walk in one launch: block 0 resolves the wave
// (chaining the exact entry count through its segments as their window
// blocks finish, segment by segment), blocks 1.. walk one segment's window
// each.  Only block 0 waits, and only for window blocks, which wait for
// nothing: they always finish, whichever blocks are resident.
__global__ void __launch_bounds__(kWinThreads, kWinBlocksPerSM)
    k_wave(const AmbEntry *__restrict__ entries, const uint32_t *__restrict__ pos,
           const uint32_t *__restrict__ n_ptr, int64_t capacity,
           const unsigned long long *__restrict__ seg_copy,
           const unsigned long long *__restrict__ seg_spread, WalkState *st, uint32_t wave, uint32_t per_wave, uint32_t t0, SegWindow *__restrict__ windows,
           uint32_t *__restrict__ table, SegList *__restrict__ lists,
           uint32_t *__restrict__ e_in_exact, uint32_t serial_below, double sigmas,
           const uint8_t *__restrict__ chunk_two, uint32_t *flags, uint32_t *err) {
    if (pass_stopped(err)) return;
    const uint32_t n = (uint32_t)min((int64_t)*n_ptr, capacity);
    if (n < serial_below) return;  // the chain is walked serially instead
    const uint32_t tag = wave + 1;  // flags are cleared once per pass
    if (blockIdx.x == 0) {
        resolve_block(entries, pos, n, st, wave, per_wave, t0, windows, table, lists, e_in_exact,
                      flags, tag, err);
        return;
    }
    const uint32_t b = blockIdx.x - 1;
    if ((wave * per_wave + b) * (uint64_t)kSegLen >= n) return;  // past the chain: no flag
    window_block(entries, pos, n, seg_copy, seg_spread, st, wave, per_wave, t0, windows, table, lists,
                 st, sigmas, chunk_two, b, flags, tag);
}

// ---------------------------------------------------------------------------
// Per-channel running counts: one warp per segment; lane 0 walks from the
// exact entry count while the warp stages the entries with cp.async.
// ---------------------------------------------------------------------------

constexpr int kRewalkWarps = 4;
constexpr int kRewalkLanes = 4;    // segments per warp: lane l < 4 walks one
constexpr int kRewalkChunk = 128;  // channels per staged chunk and segment
constexpr int kRewalkRing = 3;
constexpr int kGroup = 8;

// A warp walks kRewalkLanes segments at once, one per lane, so resident
// warps no longer each issue a full instruction stream for a single chain
// (with one walking lane, lane 0 measured 61 cycles per channel against 30
// for the bare step).  217 KB: one block of 16 segments per SM.  Two
// segments per walking lane, stepped alternately in 64-channel chunks,
// measured 301 us against 125 us: no overlap of the two chains' steps, and
// half the SMs.
// A segment's ring and output rows are padded (32 bytes and one word), so
// that the four walking lanes of a warp, which read and write the same
// offset of four different segments, fall into different shared-memory
// banks (unpadded, the segments' strides are multiples of 128 bytes and
// every entry load was a four-way conflict).
struct RewalkRing {
    AmbEntry e[kRewalkRing][kRewalkChunk];
    uint4 pad[2];
};
struct RewalkOut {
    uint32_t v[kRewalkRing][kRewalkChunk];
    uint32_t pad;
};
struct RewalkSmem {
    RewalkRing ring[kRewalkWarps][kRewalkLanes];
    RewalkOut out[kRewalkWarps][kRewalkLanes];
};
static_assert(sizeof(RewalkRing) % 128 == 32 && sizeof(RewalkOut) / 4 % 32 == 1,
              "the walking lanes' segments start in different banks");
static_assert(sizeof(RewalkSmem) <= 232448, "one rewalk block fits an SM's shared memory");

__device__ __forceinline__ void step(const uint4 &lw, const uint4 &ac, uint32_t &T, uint32_t &extra,
                                     uint32_t &E) {
    const uint32_t u0 = ac.x * T + ac.y;
    const uint32_t u1 = ac.z * T + ac.w;
    T = extra ? u1 : u0;
    extra = copies(lw, T) ? 0u : 1u;
    E += extra;
}

__global__ void __launch_bounds__(kRewalkWarps * 32)
    k_rewalk(const AmbEntry *__restrict__ entries, const uint32_t *__restrict__ pos,
             const uint32_t *__restrict__ n_ptr, int64_t capacity, uint32_t parallel_seg_len,
             const uint32_t *__restrict__ e_in_exact, uint32_t t0,
             uint32_t *__restrict__ extra_after, uint32_t serial_below,
             const uint32_t *__restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RewalkSmem &S = *reinterpret_cast<RewalkSmem *>(smem_raw);
    if (pass_stopped(err)) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t n = (uint32_t)min((int64_t)*n_ptr, capacity);
    // a short chain (or the serial mode) is one segment walked from E = 0
    const bool serial = n < serial_below;
    const uint32_t seg_len = serial ? (n > 0 ? n : 1u) : parallel_seg_len;
    const uint32_t jbase = (blockIdx.x * kRewalkWarps + warp) * kRewalkLanes;
    if ((uint64_t)jbase * seg_len >= n) return;  // the whole warp is past the chain
    // bounds of the warp's segments (every lane computes all of them)
    uint32_t s_i0[kRewalkLanes], s_i1[kRewalkLanes];
#pragma unroll
    for (int q = 0; q < kRewalkLanes; ++q) {
        const uint64_t a = (uint64_t)(jbase + q) * seg_len;
        s_i0[q] = a < n ? (uint32_t)a : n;
        s_i1[q] = a < n ? (uint32_t)min((uint64_t)n, a + seg_len) : n;
    }
    const uint32_t chunks = (s_i1[0] - s_i0[0] + kRewalkChunk - 1) / kRewalkChunk;  // longest
    auto issue = [&](uint32_t k) {
        if (k < chunks) {
#pragma unroll
            for (int q = 0; q < kRewalkLanes; ++q) {
                const uint32_t first = s_i0[q] + k * kRewalkChunk;
                if (first >= s_i1[q]) continue;  // warp-uniform
                const uint32_t count = min((uint32_t)kRewalkChunk, s_i1[q] - first);
                const uint4 *src = reinterpret_cast<const uint4 *>(entries + first);
                uint4 *dst = reinterpret_cast<uint4 *>(S.ring[warp][q].e[k % kRewalkRing]);
                for (uint32_t v = lane; v < 2 * count; v += 32) {
                    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(dst + v);
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa),
                                 "l"(src + v));
                }
            }
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
#pragma unroll
    for (int k = 0; k < kRewalkRing - 1; ++k) issue(k);
    // this lane's own segment (lanes 0..kRewalkLanes-1)
    const uint64_t my_a = (uint64_t)(jbase + (lane < kRewalkLanes ? lane : 0)) * seg_len;
    const bool walker = lane < kRewalkLanes && my_a < n;
    const int me = walker ? lane : 0;
    const uint32_t i0 = walker ? (uint32_t)my_a : 0u;
    const uint32_t i1 = walker ? (uint32_t)min((uint64_t)n, my_a + seg_len) : 0u;
    uint32_t T = 0, E = 0, extra = 0u;
    if (walker) {
        const uint32_t e_in = serial ? 0u : e_in_exact[jbase + me];
        T = jump_t(t0, (uint64_t)pos[i0] + 1u + e_in);  // state at channel i0's first draw
        E = e_in;
    }
    for (uint32_t k = 0; k < chunks; ++k) {
        issue(k + kRewalkRing - 1);
        asm volatile("cp.async.wait_group %0;\n" ::"n"(kRewalkRing - 1));
        __syncwarp();
        const uint32_t first = i0 + k * kRewalkChunk;
        if (walker && first < i1) {
            const uint32_t count = min((uint32_t)kRewalkChunk, i1 - first);
            const uint4 *__restrict__ e4 =
                reinterpret_cast<const uint4 *>(S.ring[warp][me].e[k % kRewalkRing]);
            uint32_t *__restrict__ o = S.out[warp][me].v[k % kRewalkRing];
            uint32_t i = 0;
            if (k == 0) {
                // the first channel needs no transition: its state is the jump
                extra = copies(e4[0], T) ? 0u : 1u;
                E += extra;
                o[0] = E;
                i = 1;
            }
            const uint32_t groups = (count - i) / kGroup;
            for (uint32_t g = 0; g < groups; ++g) {
                const uint32_t base = i + g * kGroup;
                uint4 lw[kGroup], ac[kGroup];
#pragma unroll
                for (int q = 0; q < kGroup; ++q) {
                    lw[q] = e4[2 * (base + q)];
                    ac[q] = e4[2 * (base + q) + 1];
                }
#pragma unroll
                for (int q = 0; q < kGroup; ++q) {
                    step(lw[q], ac[q], T, extra, E);
                    o[base + q] = E;
                }
            }
            for (uint32_t r = i + groups * kGroup; r < count; ++r) {
                step(e4[2 * r], e4[2 * r + 1], T, extra, E);
                o[r] = E;
            }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < kRewalkLanes; ++q) {
            const uint32_t f = s_i0[q] + k * kRewalkChunk;
            if (f >= s_i1[q]) continue;  // warp-uniform
            const uint32_t count = min((uint32_t)kRewalkChunk, s_i1[q] - f);
            const uint32_t *o = S.out[warp][q].v[k % kRewalkRing];
            for (uint32_t r = lane; r < count; r += 32) extra_after[f + r] = o[r];
        }
        __syncwarp();
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

int64_t walk_max_segments(int64_t capacity) { return (capacity + kSegLen - 1) / kSegLen + 1; }

// The first two arrays of the walk scratch: per segment, the copying states
// summed over its channels and the spread (sum of m (2^24 - m) >> 22); k_coef
// accumulates them, so they are cleared before it.
void walk_segment_stats(void *scratch, int64_t capacity, unsigned long long **copy,
                        unsigned long long **spread, size_t *bytes_each) {
    const size_t each = (size_t)walk_max_segments(capacity) * sizeof(unsigned long long);
    char *p = reinterpret_cast<char *>(scratch);
    *copy = reinterpret_cast<unsigned long long *>(p);
    *spread = reinterpret_cast<unsigned long long *>(p + ((each + 255) & ~(size_t)255));
    *bytes_each = each;
}

size_t walk_scratch_bytes(int64_t capacity, int per_wave) {
    const int64_t segs = walk_max_segments(capacity);
    size_t b = 0;
    auto add = [&](size_t n) { b += (n + 255) & ~(size_t)255; };
    add(segs * sizeof(unsigned long long));  // copying states per segment
    add(segs * sizeof(unsigned long long));  // spread per segment
    add(segs * sizeof(uint32_t));  // exact E_in
    add((size_t)per_wave * sizeof(SegWindow));
    add((size_t)per_wave * kWinMax * sizeof(uint32_t));
    add((size_t)per_wave * sizeof(SegList));
    add(sizeof(WalkState));
    add((size_t)per_wave * sizeof(uint32_t));  // completion flags of a wave's windows
    return b;
}


// Segments per wave: three window blocks per SM, less one slot for the
// wave's resolve block, so every block of a wave is resident at once (a
// window block left waiting for a slot would start late, and it would be
// the wave's last, widest window).
int walk_per_wave(int sms) { return kWinBlocksPerSM * sms - 1; }

cudaError_t walk_init() {
    cudaError_t e = cudaFuncSetAttribute(k_wave, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(WindowSmem));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_rewalk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(RewalkSmem));
}

// Enqueue the walk.  The channel count stays on the device (n_ptr): the
// launch shape is sized from the list capacity and every kernel exits early
// beyond the count, so nothing waits for the host.  Chains shorter than
// kSerialBelow (or every chain, when `parallel` is off) are walked by one
// warp instead of the speculative windows.
cudaError_t launch_walk(const AmbEntry *entries, const uint32_t *pos, const uint32_t *n_ptr,
                        int64_t capacity, uint32_t s0, void *scratch, int per_wave,
                        bool parallel, double window_sigmas, const uint8_t *chunk_two,
                        uint32_t *extra_after, uint32_t *fallbacks_out,
                        unsigned long long *stats_out, const uint32_t *err,
                        cudaStream_t stream, int priority) {
    const int64_t segs_max = walk_max_segments(capacity);
    char *p = reinterpret_cast<char *>(scratch);
    auto take = [&](size_t bytes) {
        void *r = p;
        p += (bytes + 255) & ~(size_t)255;
        return r;
    };
    unsigned long long *copy = (unsigned long long *)take(segs_max * sizeof(unsigned long long));
    unsigned long long *spread =
        (unsigned long long *)take(segs_max * sizeof(unsigned long long));
    uint32_t *e_in = (uint32_t *)take(segs_max * sizeof(uint32_t));
    SegWindow *windows = (SegWindow *)take((size_t)per_wave * sizeof(SegWindow));
    uint32_t *table = (uint32_t *)take((size_t)per_wave * kWinMax * sizeof(uint32_t));
    SegList *lists = (SegList *)take((size_t)per_wave * sizeof(SegList));
    WalkState *st = (WalkState *)take(sizeof(WalkState));
    uint32_t *flags = (uint32_t *)take((size_t)per_wave * sizeof(uint32_t));
    const uint32_t t0 = (s0 & kLcgMask) << 8;
    const uint32_t serial_below = parallel ? kSerialBelow : 0xFFFFFFFFu;
    cudaMemsetAsync(st, 0, sizeof(WalkState), stream);
    cudaMemsetAsync(flags, 0, (size_t)per_wave * sizeof(uint32_t), stream);
    const uint32_t segs = (uint32_t)segs_max;
    if (parallel) {
        const uint32_t waves = (segs + per_wave - 1) / per_wave;
        cudaError_t e = cudaSuccess;
        for (uint32_t w = 0; w < waves; ++w) {
            // block 0 resolves the wave, blocks 1.. walk its windows
            const uint32_t blocks = min((uint32_t)per_wave, segs - w * per_wave) + 1u;
            e = launch_prio(k_wave, dim3(blocks), dim3(kWinThreads), sizeof(WindowSmem), stream,
                            priority, entries, pos, n_ptr, capacity, copy, spread, st, w, per_wave,
                            t0,
                            windows, table, lists, e_in, serial_below, window_sigmas, chunk_two,
                            flags, const_cast<uint32_t *>(err));
            if (e != cudaSuccess) return e;
        }
    }
    constexpr uint32_t kRewalkPerBlock = kRewalkWarps * kRewalkLanes;
    cudaError_t e = launch_prio(k_rewalk, dim3((segs + kRewalkPerBlock - 1) / kRewalkPerBlock),
                                dim3(kRewalkWarps * 32), sizeof(RewalkSmem), stream, priority,
                                entries, pos, n_ptr, capacity, (uint32_t)kSegLen, e_in, t0,
                                extra_after, serial_below, err);
    if (e != cudaSuccess) return e;
    // fallbacks_out[0] = segments walked exactly, fallbacks_out[1] = packed segments
    if (fallbacks_out)
        cudaMemcpyAsync(fallbacks_out, &st->fallbacks, 2 * sizeof(uint32_t),
                        cudaMemcpyDeviceToDevice, stream);
    if (stats_out)
        cudaMemcpyAsync(stats_out, &st->candidate_steps, 3 * sizeof(unsigned long long),
                        cudaMemcpyDeviceToDevice, stream);
    return cudaGetLastError();
}

}  // namespace fx
