// fx_analysis.cu -- per-pixel scoring and the 9x9 reconstruction stencil.
//
// Kernels (all exact binary64/binary32 in the reference's order):
//   k_planes      x3a.py:193-221 derive_auxiliary with the stage y+1 alpha,
//                 x3a.py:245-286 continuous_score + streaming.py:139-147
//                 weighted planes, written into zero/pseudo-row/repeat padded
//                 history planes (streaming.py:201-233), and the aux plane
//   k_stencil     streaming.py:454-521: decision gate, five feature records,
//                 RGB candidates, combiner, then the writer classification
//   k_startup     startup.py:186-353 hidden centres -6..-1 (RNG-free part)
#include <cstddef>

#include "fx_internal.cuh"

namespace fx {

// ---------------------------------------------------------------------------
// Planes
// ---------------------------------------------------------------------------

// The auxiliary value of one pixel (x3a.py:193-221): stage y+1's alpha and
// offset, visible lane and IR lane through the LUT, binary64 then float.
__device__ __forceinline__ float aux_value(const uint2 raw, const fx_stage &st, int visible,
                                           const float *__restrict__ lut, uint32_t *err) {
    float a;
    if (st.alpha == 1.0f) {
        if (!st.replacement_valid) raise_error(err, FX_ERR_ALPHA_ONE_UNBOUND);
        a = st.replacement;
    } else {
        const uint32_t lanes[4] = {raw.x & 0xFFFFu, raw.x >> 16, raw.y & 0xFFFFu, raw.y >> 16};
        const double vis = (double)__ldg(lut + lanes[visible]);
        const double ir = (double)__ldg(lut + lanes[3]);
        const double alpha = (double)st.alpha;
        const double offset = (double)st.offset;
        a = (float)((ir - alpha * vis) / (1.0 - alpha) - offset);
    }
    if (!isfinite(a)) raise_error(err, FX_ERR_NONFINITE_AUX);
    return a;
}

// One padded row segment of the history planes (streaming.py:111-147,
// 201-233), with the auxiliary plane computed on the way.  A block of 256
// threads covers kPlaneCols = 254 columns: thread t computes the aux of
// column base + t - 1, so the first and last thread compute only the
// segment's outer neighbours for the horizontal minimum and every thread
// computes one aux value.  History planes: rows above the
// image take the pseudo row, rows below repeat the last row, columns outside
// are zero.  The auxiliary plane is written padded too, but edge-replicated
// (the decision bars clamp their indices, streaming.py:166-198): padded
// (y, x) holds the aux of (clamp(y), clamp(x)).
constexpr int kPlaneCols = 254;  // output columns per 256-thread k_planes block

__global__ void __launch_bounds__(256)
    k_planes(const uint16_t *__restrict__ rgbi, Geometry g, const float *__restrict__ lut,
             const fx_stage *__restrict__ stages, fx_params p, float *__restrict__ auxp,
             float *__restrict__ hs, float *__restrict__ hwa, float *__restrict__ hwr,
             int64_t plane, uint32_t *err) {
    __shared__ float s_aux[256];  // aux of columns base-1 .. base+254 of the segment
    if (pass_stopped(err)) return;
    const int t = threadIdx.x;
    const bool owner = t >= 1 && t <= kPlaneCols;  // threads 0 and 255: neighbours only
    const int px = blockIdx.x * kPlaneCols + t - 1;
    const int py = blockIdx.y;
    const int y = py - kPad, x = px - kPad;
    const bool live = y >= -1;  // rows above the pseudo row are zero
    const int r = y < 0 ? 0 : (y < g.h ? y : g.h - 1);
    const int64_t row0 = (int64_t)r * g.w;
    const fx_stage ast = stages[r];  // stage y+1 (stage_parameters.py:207-212)
    const bool inside = x >= 0 && x < g.w;
    const bool own = live && px >= 0 && px < g.pitch && inside;
    uint2 raw = make_uint2(0u, 0u);
    float a = 0.0f;
    if (px >= 0 && px < g.pitch) {
        // the aux of (clamp(y), clamp(x)), for the edge-replicated plane
        const int xc = x < 0 ? 0 : (x < g.w ? x : g.w - 1);
        const uint2 rc = reinterpret_cast<const uint2 *>(rgbi)[row0 + xc];
        const float ac = aux_value(rc, ast, p.visible_channel, lut, err);
        if (owner) auxp[(int64_t)py * g.pitch + px] = ac;
        if (own) {
            raw = rc;
            a = ac;
        }
    }
    s_aux[t] = a;  // 0 outside the row, as the horizontal minimum's guard needs
    __syncthreads();
    if (!owner || px < 0 || px >= g.pitch) return;
    const float floor = p.score_floor;
    float s = 0.0f, wa = 0.0f, wr[3] = {0.0f, 0.0f, 0.0f};
    if (own) {
        const float rgb[3] = {__ldg(lut + (raw.x & 0xFFFFu)), __ldg(lut + (raw.x >> 16)),
                              __ldg(lut + (raw.y & 0xFFFFu))};
        if (y == -1) {
            // the pseudo row above the image (streaming.py:218-228)
            s = floor;
            wa = a * floor;
            for (int c = 0; c < 3; ++c) wr[c] = rgb[c] * floor;
        } else {
            float sample = a;
            if (p.horizontal_minimum && g.w > 2 && x > 0 && x < g.w - 1) {
                const float l = s_aux[t - 1], rr = s_aux[t + 1];
                const float m = (l < a) ? l : a;
                sample = (m < rr) ? m : rr;
            }
            const double primary = (double)stages[r + 1].score_base;  // stage y+2
            double sc = (((primary + (double)p.score_addend) - (double)sample) *
                         (double)p.score_scale) + (double)p.score_offset;
            sc = (sc > 1.0) ? 1.0 : sc;
            sc = (sc < (double)floor) ? (double)floor : sc;
            s = (float)sc;
            wa = s * a;
            for (int c = 0; c < 3; ++c) wr[c] = s * rgb[c];
        }
    }
    const int64_t o = (int64_t)py * g.pitch + px;
    hs[o] = s;
    hwa[o] = wa;
    hwr[o] = wr[0];
    hwr[o + plane] = wr[1];
    hwr[o + 2 * plane] = wr[2];
}

// ---------------------------------------------------------------------------
// Shared scalar pieces
// ---------------------------------------------------------------------------

// Vertical chain of one column (reconstruction.py:187-237), p = 9 samples.
struct ColumnSums {
    float s3, s5, s7, s9, b16;
};

__device__ __forceinline__ ColumnSums column_sums(const float v[9]) {
    ColumnSums o;
    double acc = (double)v[3] + (double)v[4];
    acc += (double)v[5];
    o.s3 = (float)acc;
    acc += (double)v[2];
    acc += (double)v[6];
    o.s5 = (float)acc;
    acc += (double)v[1];
    acc += (double)v[7];
    o.s7 = (float)acc;
    acc += (double)v[0];
    acc += (double)v[8];
    o.s9 = (float)acc;
    const double center = (double)v[4];
    double b = (double)v[3] + center;
    b += (double)v[5];
    b += center;
    o.b16 = (float)(b * (double)(float)(1.0 / 16.0));
    return o;
}

// column_sums on samples already widened to binary64 (the widening is
// exact, so the chains and roundings are the same).
__device__ __forceinline__ ColumnSums column_sums_wide(const double *v) {
    ColumnSums o;
    double acc = v[3] + v[4];
    acc += v[5];
    o.s3 = (float)acc;
    acc += v[2];
    acc += v[6];
    o.s5 = (float)acc;
    acc += v[1];
    acc += v[7];
    o.s7 = (float)acc;
    acc += v[0];
    acc += v[8];
    o.s9 = (float)acc;
    const double center = v[4];
    double b = v[3] + center;
    b += v[5];
    b += center;
    o.b16 = (float)(b * (double)(float)(1.0 / 16.0));
    return o;
}

// Horizontal combination (reconstruction.py:240-268).  S(k) gives the
// column sums of patch column k (0..8).
template <class S3, class S5, class S7, class S9>
__device__ __forceinline__ void q69_q21(S3 s3, S5 s5, S7 s7, S9 s9, double &q69, double &q21) {
    double t21 = (double)s3(6) + (double)s3(2);
    t21 += (double)s5(3);
    t21 += (double)s5(4);
    t21 += (double)s5(5);
    double t69 = (double)s5(8) + (double)s5(0);
    t69 += (double)s7(1);
    t69 += (double)s7(7);
#pragma unroll
    for (int x = 2; x < 7; ++x) t69 += (double)s9(x);
    q69 = t69 * (double)(float)(1.0 / 69.0);
    q21 = t21 * (double)(float)(1.0 / 21.0);
}

// The two halves of q69_q21, each in the same operation order.
template <class S5, class S7, class S9>
__device__ __forceinline__ double q69_only(S5 s5, S7 s7, S9 s9) {
    double t69 = (double)s5(8) + (double)s5(0);
    t69 += (double)s7(1);
    t69 += (double)s7(7);
#pragma unroll
    for (int x = 2; x < 7; ++x) t69 += (double)s9(x);
    return t69 * (double)(float)(1.0 / 69.0);
}

template <class S3, class S5>
__device__ __forceinline__ double q21_only(S3 s3, S5 s5) {
    double t21 = (double)s3(6) + (double)s3(2);
    t21 += (double)s5(3);
    t21 += (double)s5(4);
    t21 += (double)s5(5);
    return t21 * (double)(float)(1.0 / 21.0);
}

template <class B>
__device__ __forceinline__ double q16_wa(B b16) {
    double t = (double)b16(4) + (double)b16(3);
    t += (double)b16(5);
    t += (double)b16(4);
    return t;
}

// RGB Q16 (reconstruction.py:284-298): at(i, j) is patch row 3+i, col 3+j.
template <class A>
__device__ __forceinline__ double q16_rgb(A at) {
    double rows[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double center = (double)at(i, 1);
        double h = (double)at(i, 0) + (double)at(i, 2);
        h += center;
        h += center;
        rows[i] = h;
    }
    double total = rows[0] + rows[1];
    total += rows[1];
    total += rows[2];
    return total * (double)(float)(1.0 / 16.0);
}

// recovered_rgb_candidates (reconstruction.py:425-462), UNNORMALIZED_SUM:
// C_k = f32(Q_k * (1.0 / f64(W_k))) when W_k > 0, else f32(Q_k).  The
// reciprocal depends only on the weight, so it is computed once per weight
// and shared by the three channels (the same value every time).
struct Reciprocals {
    double r[3];
    bool pos[3];
};

__device__ __forceinline__ Reciprocals weight_reciprocals(const float weights[4]) {
    Reciprocals o;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        o.pos[k] = weights[k] > 0.0f;
        o.r[k] = o.pos[k] ? 1.0 / (double)weights[k] : 0.0;
    }
    return o;
}

__device__ __forceinline__ float rgb_candidate(double avg, const Reciprocals &rc, int k) {
    return rc.pos[k] ? (float)(avg * rc.r[k]) : (float)avg;
}

// The combiner's and writer's float32 profile constants, widened once on the
// host (the widening is exact).
struct CombineConst {
    double band_scale[3], factor_a[9], factor_b[9], coarse_slope[3], strength[3];
    double dither_scale[3];
};

static CombineConst combine_const(const fx_params &p) {
    CombineConst c;
    for (int i = 0; i < 3; ++i) {
        c.band_scale[i] = (double)p.band_scales[i];
        c.coarse_slope[i] = (double)p.coarse_slopes[i];
        c.strength[i] = (double)p.configured_strengths[i];
        c.dither_scale[i] = (double)p.dither_scales[i];
    }
    for (int i = 0; i < 9; ++i) {
        c.factor_a[i] = (double)p.factors_a[i];
        c.factor_b[i] = (double)p.factors_b[i];
    }
    return c;
}

// combine_recovered_candidate (reconstruction.py:807-887).  feats[r][l].
__device__ bool combine(const float cand[3][3], const float source[3], const float weights[4],
                        const float feats[5][4], int records, float coarse_reference,
                        const fx_params &p, const CombineConst &cc, double out[3]) {
    bool finite = true;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) finite &= isfinite(cand[k][c]);
#pragma unroll
    for (int c = 0; c < 3; ++c) finite &= isfinite(source[c]);
#pragma unroll
    for (int l = 0; l < 4; ++l) finite &= isfinite(weights[l]);
    for (int r = 0; r < records; ++r)
#pragma unroll
        for (int l = 0; l < 4; ++l) finite &= isfinite(feats[r][l]);
    if (!finite) return false;

    // band ranges: each record's four values widened once
    double rmin[3], rmax[3];
    double f00;
    {
        const double a0 = (double)feats[0][0], a1 = (double)feats[0][1];
        const double a2 = (double)feats[0][2], a3 = (double)feats[0][3];
        f00 = a0;
        rmin[0] = rmax[0] = a1 - a0;
        rmin[1] = rmax[1] = a2 - a1;
        rmin[2] = rmax[2] = a3 - a2;
    }
    for (int r = 1; r < records; ++r) {
        const double a0 = (double)feats[r][0], a1 = (double)feats[r][1];
        const double a2 = (double)feats[r][2], a3 = (double)feats[r][3];
        const double d[3] = {a1 - a0, a2 - a1, a3 - a2};
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            rmin[t] = (d[t] < rmin[t]) ? d[t] : rmin[t];
            rmax[t] = (d[t] > rmax[t]) ? d[t] : rmax[t];
        }
    }
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        rmin[t] = (double)(float)rmin[t];
        rmax[t] = (double)(float)rmax[t];
    }
    double strengths[3];
    if (p.configured_strengths[0] == 0.0f) {
        const double v = (double)(float)(2.0 * (double)weights[1]);
        const double lower = (v > 0.0) ? v : 0.0;
        const double clamped = (lower < 1.0) ? lower : 1.0;
        strengths[0] = (double)(float)clamped;
    } else {
        strengths[0] = cc.strength[0];
    }
    if (p.configured_strengths[1] == 0.0f) {
        const float m2 = (weights[2] < 0.0f) ? 0.0f : weights[2];
        strengths[1] = (double)m2;
    } else {
        strengths[1] = cc.strength[1];
    }
    if (p.configured_strengths[2] == 0.0f) {
        const double w3 = (double)weights[3];
        strengths[2] = w3 * w3;
    } else {
        strengths[2] = cc.strength[2];
    }

    double candidate[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) candidate[c] = (double)cand[0][c];
    if (p.coarse_enabled) {
        const double delta = (double)coarse_reference - f00;
#pragma unroll
        for (int c = 0; c < 3; ++c) candidate[c] = candidate[c] + cc.coarse_slope[c] * delta;
    }
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        if (!p.band_enabled[b]) continue;
        const double scale = cc.band_scale[b];
        const double emin = rmin[b], emax = rmax[b];
        const bool negative = emin < 0.0 && emax < 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double coarse_v = (double)cand[b][c];
            const double fine_v = (b < 2) ? (double)cand[b + 1][c] : (double)source[c];
            const double diff = scale * (fine_v - coarse_v);
            const double fa = cc.factor_a[b * 3 + c];
            const double fb = cc.factor_b[b * 3 + c];
            const double upper = negative ? fb * emax : fa * emax;
            const double lower = negative ? fa * emin : fb * emin;
            double residual;
            if (diff > upper) residual = diff - upper;
            else if (diff < lower) residual = diff - lower;
            else residual = 0.0;
            candidate[c] = candidate[c] + strengths[b] * residual;
        }
    }
    out[0] = candidate[0];
    out[1] = candidate[1];
    out[2] = candidate[2];
    return true;
}

// Writer draw classification for one attempted site (the RNG-free part of
// reconstruction.py:916-982).  Per channel: 0 = no draw, 1 = one draw,
// 2 = two draws, 3 = one or two draws depending on the state.
__device__ uint8_t classify_site(const double cand[3], const float orig[3], bool floor_enabled,
                                 const CombineConst &cc, const DitherConst &dc, uint32_t *err) {
    uint8_t meta = 0x80;
    bool valid = true;
#pragma unroll
    for (int c = 0; c < 3; ++c) valid &= isfinite(cand[c]) && cand[c] > 0.0;
    if (!valid) return meta;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float c32 = (float)cand[c];
        if (!isfinite(c32)) raise_error(err, FX_ERR_DITHER_INPUT);
        const double cd = (double)c32;
        int code;
        if (!dc.low_lt_high || !(dc.low < cd && cd < dc.high)) {
            code = 0;
        } else if (!floor_enabled) {
            code = 1;
        } else {
            const double env = ((dc.high - cd) * (cd - dc.low)) * dc.coefficient;
            const float span = (float)(cc.dither_scale[c] * cd);
            const double da = dither_raw_delta(cd, env, span, 0u);
            const double db = dither_raw_delta(cd, env, span, kLcgMask);
            double lo = (da < db) ? da : db, hi = (da < db) ? db : da;
            lo = (lo < 0.0) ? lo : 0.0;
            hi = (hi > 0.0) ? hi : 0.0;
            const double od = (double)orig[c];
            if (cand[c] + hi <= od) code = 1;        // always copies the original
            else if (!(cand[c] + lo <= od)) code = 2;  // never copies: redraws
            else code = 3;
        }
        meta |= (uint8_t)(code << (2 * c));
    }
    return meta;
}

// ---------------------------------------------------------------------------
// The stencil
// ---------------------------------------------------------------------------

// Tile geometry for a tile of TH pixel rows by 32 pixel columns.  Every plane
// tile is staged with 16-byte cp.async copies from a 16-byte aligned origin:
// padded column x0 (x0 a multiple of 32, the pitch a multiple of 32 floats),
// 44 floats (11 vectors) per row.
template <int TH>
struct Tile {
    static constexpr int TW = 32;
    static constexpr int THREADS = TH * TW;
    static constexpr int PR = TH + 10;   // history tile rows (y0-5 .. y0+TH+4)
    static constexpr int PC = TW + 10;   // history tile cols used (x0-5 .. x0+TW+4)
    static constexpr int RR = TH + 8;    // rgb / decision tile rows (y0-4 ..)
    static constexpr int RC = TW + 8;    // rgb / decision tile cols used (x0-4 ..)
    static constexpr int CR = TH + 2;    // record rows (y0-1 .. y0+TH)
    static constexpr int CC = TW + 10;   // column-sum cols (x0-5 .. x0+TW+4)
    static constexpr int RECC = TW + 2;  // record cols (x0-1 .. x0+TW)
    static constexpr int SW = 44;        // staged floats per row (11 x 16 bytes)
    static constexpr int RO = 1;         // staged column of rgb / decision col 0
    static constexpr int WA_RUN = TH == 8 ? 5 : 6;  // score / waux column-sum run
    static constexpr int RGB_RUN = 4;               // rgb column-sum run
    static constexpr int BLOCKS_PER_SM = TH == 8 ? 4 : 2;
};

// A feature record of the stencil (streaming.py:236-308): the four feature
// values (one 16-byte vector, read by a consumer pixel in one load) and the
// W of its score patch (the consumer's weights when it is the centre
// record), kept in three separate planes.  A lane that takes the consumer
// row's fallback value holds kFallbackBits, a NaN: the feature values are
// quotients and aux values of finite planes, never NaN, so the marker
// cannot collide with a value.
template <int CR, int RECC>
struct StencilRecords {
    float4 a[CR][RECC];
    float w[3][CR][RECC];
};
constexpr uint32_t kFallbackBits = 0x7FC0FB00u;

// The tiles staged with 16-byte cp.async (hs, hwa, hwr, auxt) start on
// 16-byte boundaries (checked below); the other members follow them.
template <int TH>
struct StencilSmem {
    using T = Tile<TH>;
    __align__(16) float hs[T::PR][T::SW];
    union __align__(16) {
        float hwa[T::PR][T::SW];                // waux tile: dead after the column sums
        StencilRecords<T::CR, T::RECC> rec;     // written by the records phase
    };
    __align__(16) float hwr[3][T::RR][T::SW];   // staged column j: logical col j - RO
    float cs[2][5][T::CR][T::CC];               // [score|waux][S3,S5,S7,S9,B16]
    float rcs[3][4][TH][T::RC];                 // [channel][S3,S5,S7,S9]
    uint16_t reclist[T::CR * T::RECC];          // record positions an attempted pixel reads
    int nrec;
    union __align__(16) {
        // aux at clamped (y0-4+r, x0-5+j): decision masks and point aux,
        // dead once the records are built
        float auxt[T::RR][T::SW];
        struct {  // the attempted-pixel list of the per-pixel phase
            uint32_t wcount[T::THREADS / 32];
            int n_attempted;
            uint16_t attempted[T::THREADS];  // thread index of each attempted pixel
        } dec;
    };
    unsigned long long rowlow[T::RR];  // bit c: aux (row r, col c) below the threshold
    uint32_t collow[T::RC];            // bit r: the same, by column
    uint32_t rowbal[TH];               // bit x: pixel (row, x) of the tile is attempted
};
// four 8-row blocks per SM (228 KB less 1 KB reserved per block); two 16-row
template <int TH>
constexpr bool staged_tiles_aligned() {
    return offsetof(StencilSmem<TH>, hs) % 16 == 0 && offsetof(StencilSmem<TH>, hwa) % 16 == 0 &&
           offsetof(StencilSmem<TH>, hwr) % 16 == 0 && offsetof(StencilSmem<TH>, auxt) % 16 == 0 &&
           (Tile<TH>::SW * sizeof(float)) % 16 == 0;
}
static_assert(staged_tiles_aligned<8>() && staged_tiles_aligned<16>(),
              "cp.async 16-byte destinations must start on 16-byte boundaries");
static_assert(sizeof(StencilSmem<8>) <= 57344, "the 8-row tile keeps four blocks per SM");
static_assert(sizeof(StencilSmem<16>) <= 115712, "the 16-row tile keeps two blocks per SM");
static_assert(Tile<8>::RR <= 32 && Tile<16>::RR <= 32, "column masks are 32 bits");
static_assert(sizeof(float) * Tile<16>::RR * Tile<16>::SW >=
                  4 * (Tile<16>::THREADS / 32 + 1) + 2 * Tile<16>::THREADS,
              "the attempted list fits in the aux tile");
static_assert(sizeof(float) * Tile<8>::RR * Tile<8>::SW >=
                  4 * (Tile<8>::THREADS / 32 + 1) + 2 * Tile<8>::THREADS,
              "the attempted list fits in the aux tile");
static_assert(kTileH % 16 == 0, "padded planes cover whole tiles of either height");

template <int TH>
__global__ void __launch_bounds__(Tile<TH>::THREADS, Tile<TH>::BLOCKS_PER_SM)
    k_stencil(const uint16_t *__restrict__ rgbi, Geometry g, const float *__restrict__ lut,
              const fx_stage *__restrict__ stages, fx_params p, CombineConst cc,
              const float *__restrict__ auxp, const float *__restrict__ hs,
              const float *__restrict__ hwa, const float *__restrict__ hwr, int64_t plane,
              double *__restrict__ cand_out, uint8_t *__restrict__ meta_out, uint32_t *err) {
    using T = Tile<TH>;
    constexpr int PR = T::PR, RR = T::RR, RC = T::RC, CR = T::CR, CC = T::CC;
    constexpr int RECC = T::RECC, RO = T::RO, NT = T::THREADS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    StencilSmem<TH> &S = *reinterpret_cast<StencilSmem<TH> *>(smem_raw);
    if (pass_stopped(err)) return;
    const int tid = threadIdx.x;
    const int y0 = blockIdx.y * TH, x0 = blockIdx.x * T::TW;
    const int h = g.h, w = g.w;
    const int dty = tid / T::TW, dtx = tid % T::TW;
    // the writer stage's gates of this thread's pixel row (stage y+7),
    // loaded while the tile is staged
    int gate_secondary = 0, row_gate = 1;
    if (y0 + dty < h) {
        gate_secondary = stages[y0 + dty + 6].gate_secondary;
        row_gate = stages[y0 + dty + 6].row_gate;
    }
    if (tid == 0) S.nrec = 0;

    // ---- stage the tile ---------------------------------------------------
    // 16-byte copies, 11 per staged row, in two groups: first what the
    // decision reads (PR score rows from padded row y0, RR aux rows from
    // padded row y0+1), then the waux rows and the 3 x RR rgb rows.  The
    // decision runs while the second group is in flight.
    {
        constexpr int kVec = T::SW / 4;
        const int64_t col = x0;
        constexpr int kRowsA = PR + RR, kRowsB = PR + 3 * RR;
        for (int i = tid; i < kRowsA * kVec; i += NT) {
            const int row = i / kVec, v = i % kVec;
            const bool score = row < PR;
            const int r = score ? row : row - PR;
            const float *src = (score ? hs + (int64_t)(y0 + r) * g.pitch
                                      : auxp + (int64_t)(y0 + 1 + r) * g.pitch) + col;
            float *dst = score ? S.hs[r] : S.auxt[r];
            const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst + 4 * v);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + 4 * v));
        }
        asm volatile("cp.async.commit_group;\n" ::);
        for (int i = tid; i < kRowsB * kVec; i += NT) {
            const int row = i / kVec, v = i % kVec;
            const float *src;
            float *dst;
            if (row < PR) {
                src = hwa + (int64_t)(y0 + row) * g.pitch + col;
                dst = S.hwa[row];
            } else {
                const int q = row - PR, k = q / RR, r = q % RR;  // rgb plane k
                src = hwr + k * plane + (int64_t)(y0 + 1 + r) * g.pitch + col;
                dst = S.hwr[k][r];
            }
            const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst + 4 * v);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + 4 * v));
        }
        asm volatile("cp.async.commit_group;\n" ::);
        asm volatile("cp.async.wait_group 1;\n" ::);  // the first group
    }
    const float thr = p.decision_threshold;
    __syncthreads();

    // ---- decision masks -----------------------------------------------------
    // bit c of rowlow[r] / bit r of collow[c]: aux (row r, col c) of the
    // decision tile is below the threshold; rows by warp ballots (columns
    // 0..31, then 32..RC-1), columns transposed from the rows
    {
        const int lane = tid & 31;
        static_assert(T::RC > 32 && T::RC <= 64, "two ballots cover a mask row");
        for (int r = tid >> 5; r < RR; r += NT / 32) {
            const bool lo = S.auxt[r][lane + RO] < thr;
            const bool hi = lane < RC - 32 && S.auxt[r][lane + 32 + RO] < thr;
            const uint32_t b0 = __ballot_sync(0xFFFFFFFFu, lo);
            const uint32_t b1 = __ballot_sync(0xFFFFFFFFu, hi);
            if (lane == 0) S.rowlow[r] = ((unsigned long long)b1 << 32) | b0;
        }
        __syncthreads();
        if (tid < RC) {
            uint32_t m = 0;
            for (int r = 0; r < RR; ++r) m |= (uint32_t)((S.rowlow[r] >> tid) & 1ull) << r;
            S.collow[tid] = m;
        }
        __syncthreads();
    }

    // ---- per output pixel: the decision -------------------------------------
    // It needs only the aux masks, the point score and the stage gates, so it
    // comes first: a tile without an attempted pixel stops here, and the
    // others build only the records their attempted pixels read.
    bool eligible = false;
    {
        const int y = y0 + dty, x = x0 + dtx;
        if (y < h && x < w) {
            const bool floor_enabled = p.driver_gate_primary || gate_secondary;
            // decision bars (streaming.py:157-198), edge-replicated via the
            // tile: rows ty..ty+8 of a column, columns tx..tx+8 of a row
            const int rad = p.radius;
            const int vl = __popc((S.collow[dtx + 4 - rad] >> dty) & 0x1FFu);
            const int vr = __popc((S.collow[dtx + 4 + rad] >> dty) & 0x1FFu);
            const int ha = __popcll((S.rowlow[dty + 4 - rad] >> dtx) & 0x1FFull);
            const int hb = __popcll((S.rowlow[dty + 4 + rad] >> dtx) & 0x1FFull);
            const int lim = p.count_limit;
            eligible = !(vl > lim || ha > lim || vr > lim || hb > lim);
            const float point_score = S.hs[dty + 5][dtx + 5];
            if (row_gate != 0) eligible = false;
            else if (floor_enabled && !(point_score < 1.0f)) eligible = false;
            // driver_forces_fallback (reconstruction.py:890-904)
            if (eligible && (row_gate != 0 || (floor_enabled && point_score >= 1.0f)))
                eligible = false;
            if (!eligible) meta_out[6 * (int64_t)w + (int64_t)y * w + x] = 0;
        }
        // a warp is one pixel row of the tile (32 columns)
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, eligible);
        if (dtx == 0) S.rowbal[dty] = bal;
    }
    if (!__syncthreads_or(eligible)) {  // no attempted pixel in the tile
        asm volatile("cp.async.wait_group 0;\n" ::);  // no copy outlives the block
        return;
    }

    // The record positions an attempted pixel reads, listed densely (any
    // order: each record is computed alone): record row r is the centre row
    // of pixel row r-1 and the cross neighbour of pixel rows r and r-2.
    // (A warp-ordered list, by ballot and one atomic per warp, measured 2%
    // more instructions and no fewer shared-memory bank conflicts.)
    for (int i = tid; i < CR * RECC; i += NT) {
        const int r = i / RECC, c = i % RECC;
        unsigned long long need = 0;
        if (r >= 1 && r <= TH) {
            const unsigned long long b = S.rowbal[r - 1];
            need |= b | (b << 1) | (b << 2);
        }
        if (r < TH) need |= (unsigned long long)S.rowbal[r] << 1;
        if (r >= 2) need |= (unsigned long long)S.rowbal[r - 2] << 1;
        if ((need >> c) & 1ull) S.reclist[atomicAdd(&S.nrec, 1)] = (uint16_t)i;
    }

    asm volatile("cp.async.wait_group 0;\n" ::);  // the waux and rgb rows
    __syncthreads();

    // One work item is a vertical run of column sums in one column: the
    // samples are loaded and widened once and shared by the run's chains.
    // Items below kWaItems: score / waux planes, runs of WA_RUN record rows;
    // the rest: the three RGB planes, runs of RGB_RUN pixel rows.
    constexpr int WR = T::WA_RUN, GR = T::RGB_RUN;
    static_assert(CR % WR == 0 && TH % GR == 0, "runs tile the rows");
    constexpr int kWaItems = 2 * CC * (CR / WR), kRgbItems = 3 * RC * (TH / GR);
    for (int it = tid; it < kWaItems + kRgbItems; it += NT) {
        if (it < kWaItems) {
            const int src = it / (CC * (CR / WR)), rem = it % (CC * (CR / WR));
            const int c = rem % CC, r0 = (rem / CC) * WR;  // lanes on consecutive columns
            const float(*pl)[T::SW] = src ? S.hwa : S.hs;
            double v[WR + 8];
#pragma unroll
            for (int k = 0; k < WR + 8; ++k) v[k] = (double)pl[r0 + k][c];
#pragma unroll
            for (int j = 0; j < WR; ++j) {
                const ColumnSums cs = column_sums_wide(v + j);
                S.cs[src][0][r0 + j][c] = cs.s3;
                S.cs[src][1][r0 + j][c] = cs.s5;
                S.cs[src][2][r0 + j][c] = cs.s7;
                S.cs[src][3][r0 + j][c] = cs.s9;
                S.cs[src][4][r0 + j][c] = cs.b16;
            }
        } else {
            const int q = it - kWaItems;
            const int ch = q / (RC * (TH / GR)), rem = q % (RC * (TH / GR));
            const int c = rem % RC, r0 = (rem / RC) * GR;
            double v[GR + 8];
#pragma unroll
            for (int k = 0; k < GR + 8; ++k) v[k] = (double)S.hwr[ch][r0 + k][c + RO];
#pragma unroll
            for (int j = 0; j < GR; ++j) {
                const ColumnSums cs = column_sums_wide(v + j);
                S.rcs[ch][0][r0 + j][c] = cs.s3;
                S.rcs[ch][1][r0 + j][c] = cs.s5;
                S.rcs[ch][2][r0 + j][c] = cs.s7;
                S.rcs[ch][3][r0 + j][c] = cs.s9;
            }
        }
    }
    __syncthreads();

    // ---- feature records (streaming.py:236-308) ---------------------------
    // (the record array overlays the waux tile, dead after the column sums)
    const int nrec = S.nrec;
    for (int k = tid; k < nrec; k += NT) {
        const int i = S.reclist[k];
        const int r = i / RECC, c = i % RECC;
        const int xx = x0 - 1 + c;
        float ra[4], rw[3];
        if (xx < 0 || xx >= w) {
            // horizontal guard records stay zero (streaming.py:281-282)
            ra[0] = ra[1] = ra[2] = ra[3] = 0.0f;
            rw[0] = rw[1] = rw[2] = 0.0f;
        } else {
            double wq[3], nq[3];
#pragma unroll
            for (int src = 0; src < 2; ++src) {
                const float(*s3)[CC] = S.cs[src][0];
                const float(*s5)[CC] = S.cs[src][1];
                const float(*s7)[CC] = S.cs[src][2];
                const float(*s9)[CC] = S.cs[src][3];
                const float(*bb)[CC] = S.cs[src][4];
                double q69, q21;
                q69_q21([&](int k) { return s3[r][c + k]; }, [&](int k) { return s5[r][c + k]; },
                        [&](int k) { return s7[r][c + k]; }, [&](int k) { return s9[r][c + k]; },
                        q69, q21);
                const double q16 = q16_wa([&](int k) { return bb[r][c + k]; });
                double *dst = src ? nq : wq;
                dst[0] = q69;
                dst[1] = q21;
                dst[2] = q16;
            }
            const float point_score = S.hs[r + 4][c + 4];
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                ra[l] = wq[l] > 0.0 ? (float)(nq[l] / wq[l]) : __uint_as_float(kFallbackBits);
                rw[l] = (float)wq[l];
            }
            ra[3] = point_score > 0.0f ? S.auxt[r + 3][c + 3 + RO]  // xx is inside the row
                                       : __uint_as_float(kFallbackBits);
        }
        S.rec.a[r][c] = make_float4(ra[0], ra[1], ra[2], ra[3]);
        S.rec.w[0][r][c] = rw[0];
        S.rec.w[1][r][c] = rw[1];
        S.rec.w[2][r][c] = rw[2];
    }
    __syncthreads();

    // ---- the attempted pixels, listed ----------------------------------------
    // About half the pixels are attempted, mixed within every warp: they are
    // listed in shared memory (over the aux tile, dead once the records are
    // built) and processed densely.
    {
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, eligible);
        if ((tid & 31) == 0) S.dec.wcount[tid >> 5] = __popc(bal);
        __syncthreads();
        uint32_t base = 0, total = 0;
#pragma unroll
        for (int k = 0; k < NT / 32; ++k) {
            const uint32_t c = S.dec.wcount[k];
            base += k < (tid >> 5) ? c : 0u;
            total += c;
        }
        if (eligible) S.dec.attempted[base + __popc(bal & ((1u << (tid & 31)) - 1u))] = (uint16_t)tid;
        if (tid == 0) S.dec.n_attempted = total;
        __syncthreads();
    }

    // ---- attempted pixels, densely -----------------------------------------
    const int listed = S.dec.n_attempted;
    if (tid >= listed) return;
    const int me = S.dec.attempted[tid];
    const int ty = me / T::TW, tx = me % T::TW;
    const int y = y0 + ty, x = x0 + tx;
    const int64_t site = 6 * (int64_t)w + (int64_t)y * w + x;
    const uint2 raw = reinterpret_cast<const uint2 *>(rgbi)[(int64_t)y * w + x];
    const fx_stage ws = stages[y + 6];  // writer stage y+7
    const bool floor_enabled = p.driver_gate_primary || ws.gate_secondary;
    const float orig[3] = {__ldg(lut + (raw.x & 0xFFFFu)), __ldg(lut + (raw.x >> 16)),
                           __ldg(lut + (raw.y & 0xFFFFu))};

    const float fallback = ws.coarse;
    const int records = p.cross_neighbor ? 5 : 1;
    float feats[5][4];
    const int rr[5] = {ty + 1, ty + 1, ty + 1, ty, ty + 2};
    const int rc[5] = {tx + 1, tx, tx + 2, tx + 1, tx + 1};
    for (int k = 0; k < records; ++k) {
        const float4 q = S.rec.a[rr[k]][rc[k]];
        const float rec_a[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int l = 0; l < 4; ++l)
            feats[k][l] = __float_as_uint(rec_a[l]) == kFallbackBits ? fallback : rec_a[l];
    }
    // W of the centre record (record row ty + 1, column tx + 1): the score
    // patch averages its record phase computed, and the point score
    float weights[4];
    {
        weights[0] = S.rec.w[0][ty + 1][tx + 1];
        weights[1] = S.rec.w[1][ty + 1][tx + 1];
        weights[2] = S.rec.w[2][ty + 1][tx + 1];
        weights[3] = S.hs[ty + 5][tx + 5];
    }

    // RGB candidates (reconstruction.py:425-462), one weight at a time: its
    // reciprocal serves the three channels
    float cand[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const bool pos = weights[k] > 0.0f;
        const double recip = pos ? 1.0 / (double)weights[k] : 0.0;
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            const float(*s3)[RC] = S.rcs[ch][0];
            const float(*s5)[RC] = S.rcs[ch][1];
            const float(*s7)[RC] = S.rcs[ch][2];
            const float(*s9)[RC] = S.rcs[ch][3];
            const float(*pl)[T::SW] = S.hwr[ch];
            double q;
            if (k == 0)
                q = q69_only([&](int j) { return s5[ty][tx + j]; },
                             [&](int j) { return s7[ty][tx + j]; },
                             [&](int j) { return s9[ty][tx + j]; });
            else if (k == 1)
                q = q21_only([&](int j) { return s3[ty][tx + j]; },
                             [&](int j) { return s5[ty][tx + j]; });
            else
                q = q16_rgb([&](int i, int j) { return pl[ty + 3 + i][tx + 3 + j + RO]; });
            cand[k][ch] = pos ? (float)(q * recip) : (float)q;
        }
    }
    double combined[3];
    if (!combine(cand, orig, weights, feats, records, ws.coarse, p, cc, combined)) {
        raise_error(err, FX_ERR_COMBINER_INPUT);
        meta_out[site] = 0;
        return;
    }
    const DitherConst dc = dither_const(p);
    meta_out[site] = classify_site(combined, orig, floor_enabled, cc, dc, err);
    double *dst = cand_out + 3 * site;
    dst[0] = combined[0];
    dst[1] = combined[1];
    dst[2] = combined[2];
}

// ---------------------------------------------------------------------------
// Hidden startup replay, RNG-free part (startup.py:74-353)
// ---------------------------------------------------------------------------

struct StartupView {
    Geometry g;
    const float *aux, *hs, *hwa, *hwr;
    int64_t plane;
    int rows;  // first real rows available (5 cross-neighbour, 4 centre-only)
};

// History rows of startup.py:82-117: x outside -> 0, row -1 pseudo row,
// rows below -1 zero, real rows 0..rows-1 (the public padded planes hold
// exactly these values for rows -5..rows-1).
__device__ __forceinline__ float su_plane(const StartupView &v, const float *pl, int y, int x) {
    if (x < 0 || x >= v.g.w || y < -5) return 0.0f;
    return pl[v.g.padded_index(y, x)];
}

// Raw decision history (startup.py:119-126) at padded column xp = x + 4,
// read from the edge-replicated padded aux plane.
__device__ __forceinline__ float su_raw(const StartupView &v, int y, int xp) {
    const int w = v.g.w;
    const float *src = v.aux + v.g.padded_index(y < 0 ? 0 : y, 0);
    if (xp < 4) return src[0];
    if (xp < 4 + w) return src[xp - 4];
    return y >= 0 ? src[w - 1] : 0.0f;
}

// startup.py:131-183 (weights are only needed for the centre record).
__device__ void su_record(const StartupView &v, int ly, int x, float fallback, float weights[4],
                          float feature[4]) {
    if (ly <= -6 || x < 0 || x >= v.g.w) {
#pragma unroll
        for (int l = 0; l < 4; ++l) weights[l] = feature[l] = 0.0f;
        return;
    }
    ColumnSums sc[9], wc[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) {
        float a[9], b[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            a[i] = su_plane(v, v.hs, ly - 4 + i, x - 4 + j);
            b[i] = su_plane(v, v.hwa, ly - 4 + i, x - 4 + j);
        }
        sc[j] = column_sums(a);
        wc[j] = column_sums(b);
    }
    double wq[3], nq[3];
    q69_q21([&](int k) { return sc[k].s3; }, [&](int k) { return sc[k].s5; },
            [&](int k) { return sc[k].s7; }, [&](int k) { return sc[k].s9; }, wq[0], wq[1]);
    wq[2] = q16_wa([&](int k) { return sc[k].b16; });
    q69_q21([&](int k) { return wc[k].s3; }, [&](int k) { return wc[k].s5; },
            [&](int k) { return wc[k].s7; }, [&](int k) { return wc[k].s9; }, nq[0], nq[1]);
    nq[2] = q16_wa([&](int k) { return wc[k].b16; });
    weights[0] = (float)wq[0];
    weights[1] = (float)wq[1];
    weights[2] = (float)wq[2];
    weights[3] = su_plane(v, v.hs, ly, x);
#pragma unroll
    for (int l = 0; l < 3; ++l) feature[l] = (wq[l] > 0.0) ? (float)(nq[l] / wq[l]) : fallback;
    feature[3] = (weights[3] > 0.0f) ? su_raw(v, ly, x + 4) : fallback;
}

__device__ __forceinline__ int max1(int v) { return v < 1 ? 1 : v; }

__global__ void k_startup(const uint16_t *__restrict__ rgbi, StartupView v,
                          const float *__restrict__ lut, const fx_stage *__restrict__ stages,
                          fx_params p, CombineConst cc, double *__restrict__ cand_out,
                          uint8_t *__restrict__ meta_out, uint32_t *err) {
    if (pass_stopped(err)) return;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;  // stage hit k+1, centre k-6
    const int w = v.g.w;
    if (x >= w) return;
    const int64_t site = (int64_t)k * w + x;
    const int hit = k + 1, center = k - 6;
    const fx_stage act = stages[hit - 1];
    const bool floor_enabled = p.driver_gate_primary || act.gate_secondary;
    const int writer_width = (p.cross_neighbor && hit <= 2) ? w - 4 : w;
    if (x >= writer_width) {
        meta_out[site] = 0;
        return;
    }
    const int r = p.radius;
    bool fallback_hit = false;
    for (int gi = 0; gi < 4 && !fallback_hit; ++gi) {
        int count = 0;
        for (int s = 0; s < 9; ++s) {
            const int axis = s - 4;
            const int dy = (gi == 0 || gi == 2) ? axis : (gi == 1 ? -r : r);
            const int dx = (gi == 0) ? -r : (gi == 2 ? r : axis);
            count += su_raw(v, center + dy, x + 4 + dx) < p.decision_threshold;
        }
        if (count > p.count_limit) fallback_hit = true;
    }
    const float fb_center = stages[max1(center + 6) - 1].coarse;
    float weights[4], feats[5][4];
    su_record(v, center, x, fb_center, weights, feats[0]);
    if (fallback_hit || act.row_gate != 0 || (floor_enabled && weights[3] >= 1.0f)) {
        meta_out[site] = 0;
        return;
    }
    const Reciprocals rcp = weight_reciprocals(weights);
    float cand[3][3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        const float *pl = v.hwr + ch * v.plane;
        ColumnSums cs[9];
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            float a[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) a[i] = su_plane(v, pl, center - 4 + i, x - 4 + j);
            cs[j] = column_sums(a);
        }
        double q69, q21;
        q69_q21([&](int kk) { return cs[kk].s3; }, [&](int kk) { return cs[kk].s5; },
                [&](int kk) { return cs[kk].s7; }, [&](int kk) { return cs[kk].s9; }, q69, q21);
        const double q16 = q16_rgb(
            [&](int i, int j) { return su_plane(v, pl, center - 1 + i, x - 1 + j); });
        cand[0][ch] = rgb_candidate(q69, rcp, 0);
        cand[1][ch] = rgb_candidate(q21, rcp, 1);
        cand[2][ch] = rgb_candidate(q16, rcp, 2);
    }
    const int records = p.cross_neighbor ? 5 : 1;
    if (records == 5) {
        float wn[4];
        const float fb_up = stages[max1(center + 5) - 1].coarse;
        const float fb_down = stages[max1(center + 7) - 1].coarse;
        su_record(v, center, x - 1, fb_center, wn, feats[1]);
        su_record(v, center, x + 1, fb_center, wn, feats[2]);
        su_record(v, center - 1, x, fb_up, wn, feats[3]);
        su_record(v, center + 1, x, fb_down, wn, feats[4]);
    }
    const uint2 raw = reinterpret_cast<const uint2 *>(rgbi)[x];  // row 0
    const float orig[3] = {__ldg(lut + (raw.x & 0xFFFFu)), __ldg(lut + (raw.x >> 16)),
                           __ldg(lut + (raw.y & 0xFFFFu))};
    double combined[3];
    if (!combine(cand, orig, weights, feats, records, act.coarse, p, cc, combined)) {
        raise_error(err, FX_ERR_COMBINER_INPUT);
        meta_out[site] = 0;
        return;
    }
    const DitherConst dc = dither_const(p);
    meta_out[site] = classify_site(combined, orig, floor_enabled, cc, dc, err);
    double *dst = cand_out + 3 * site;
    dst[0] = combined[0];
    dst[1] = combined[1];
    dst[2] = combined[2];
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------

cudaError_t launch_analysis(const uint16_t *rgbi, const Geometry &g, const float *lut,
                            const fx_stage *stages, const fx_params &p, float *aux, float *hs,
                            float *hwa, float *hwr, int64_t plane, double *cand, uint8_t *meta,
                            uint32_t *err, cudaStream_t stream, const Marks &marks,
                            int tile_rows, cudaStream_t side, cudaEvent_t fork,
                            cudaEvent_t join) {
    const CombineConst cc = combine_const(p);
    {
        dim3 block(256), grid((g.pitch + kPlaneCols - 1) / kPlaneCols, g.prow);
        k_planes<<<grid, block, 0, stream>>>(rgbi, g, lut, stages, p, aux, hs, hwa, hwr, plane,
                                             err);
    }
    marks.mark(2, stream);
    // k_startup (the six hidden stages, 6 W sites: too few blocks to fill the
    // GPU) runs on `side` beside the stencil: both only read the planes and
    // they write disjoint sites (startup sites 0 .. 6W-1, public ones after)
    StartupView v{g, aux, hs, hwa, hwr, plane, p.cross_neighbor ? 5 : 4};
    const dim3 su_block(128), su_grid((g.w + 127) / 128, 6);
    if (side) {
        cudaError_t e = cudaEventRecord(fork, stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(side, fork, 0);
        if (e != cudaSuccess) return e;
        k_startup<<<su_grid, su_block, 0, side>>>(rgbi, v, lut, stages, p, cc, cand, meta, err);
        e = cudaEventRecord(join, side);
        if (e != cudaSuccess) return e;
    }
    if (tile_rows == 16) {
        dim3 grid(g.tw, g.hp / 16);
        k_stencil<16><<<grid, Tile<16>::THREADS, sizeof(StencilSmem<16>), stream>>>(
            rgbi, g, lut, stages, p, cc, aux, hs, hwa, hwr, plane, cand, meta, err);
    } else {
        dim3 grid(g.tw, g.hp / 8);
        k_stencil<8><<<grid, Tile<8>::THREADS, sizeof(StencilSmem<8>), stream>>>(
            rgbi, g, lut, stages, p, cc, aux, hs, hwa, hwr, plane, cand, meta, err);
    }
    marks.mark(3, stream);
    if (side) {
        const cudaError_t e = cudaStreamWaitEvent(stream, join, 0);
        if (e != cudaSuccess) return e;
    } else
        k_startup<<<su_grid, su_block, 0, stream>>>(rgbi, v, lut, stages, p, cc, cand, meta, err);
    marks.mark(4, stream);
    return cudaGetLastError();
}


cudaError_t producer_init();
cudaError_t writer_init();

// Opt in to the dynamic shared memory the tiled kernels use (once per
// device, with the device current).
cudaError_t analysis_init() {
    cudaError_t e = cudaFuncSetAttribute(k_stencil<8>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(StencilSmem<8>));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_stencil<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(StencilSmem<16>));
    if (e != cudaSuccess) return e;
    e = walk_init();
    if (e != cudaSuccess) return e;
    e = writer_init();
    if (e != cudaSuccess) return e;
    return producer_init();
}

}  // namespace fx
