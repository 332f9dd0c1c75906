/*
 * fx_oracle.c -- CPU restatement of the Digital ICE processing core.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the B200
 * library: the tests, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py call it; the product never links, imports or executes it.
 *
 * It restates, in plain C with scalar binary64/binary32 arithmetic, the
 * reference package portable_digital_ice (version 0.3.1).  Every function
 * cites the reference file:line it follows (paths are relative to the
 * package directory src/portable_digital_ice/).  Compile with
 * -ffp-contract=off and without fast-math: every add, multiply and divide
 * must round exactly once, in the reference's order.
 *
 * Parallelism: the per-row analysis (decision gate, feature records,
 * candidates, combiner) is a pure function of read-only planes, so it runs
 * over rows with OpenMP, exactly as the reference's numba backend runs it
 * with prange (fast_cpu/kernels.py:1071-1136).  The dither writer is
 * strictly serial (reconstruction.py:916-982).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* status codes ---------------------------------------------------------- */
#define OX_OK 0
#define OX_ERR_ARG 1
#define OX_ERR_NOMEM 2
#define OX_ERR_NONFINITE_AUX 3      /* x3a.py:262-263 */
#define OX_ERR_NONFINITE_WORK 4     /* output.py:69-70 */
#define OX_ERR_COMBINER_INPUT 5     /* reconstruction.py:837-838 */
#define OX_ERR_DITHER_INPUT 6       /* dither.py:79-82 */
#define OX_ERR_SETTER_ONE 7         /* stage_parameters.py:111-112 */
#define OX_ERR_STAGE_NONFINITE 8    /* stage_parameters.py:29-33 */
#define OX_ERR_ALPHA_ONE_UNBOUND 9  /* x3a.py:209-212 */
#define OX_ERR_GEOMETRY 10          /* streaming.py:391-392, startup.py:210-213 */

#define LCG_MASK 0x00FFFFFFu
/* rng.py:135 -- float32 bits 0x337fffff widened: (2^24-1) * 2^-48 */
static const double NIKON_NORMALIZATION = 0x1.fffffep-25;

typedef struct {
    float alpha;              /* auxiliary alpha (stage_parameters.py:173) */
    float offset;             /* calibration offset (+0xf78) */
    float replacement;        /* alpha==1 replacement (x3a.py:208-215) */
    int32_t replacement_valid;
    float score_base;         /* score base primary (streaming.py:130-133) */
    float coarse;             /* writer coarse reference (streaming.py:436-443) */
    int32_t gate_secondary;   /* writer gate secondary */
    int32_t row_gate;         /* row reconstruction gate */
} ox_stage;

typedef struct {
    float score_addend, score_scale, score_offset, score_floor;
    int32_t horizontal_minimum;   /* x3a.py:266-268 */
    int32_t visible_channel;      /* x3a.py:218 */
    float decision_threshold;     /* profile.py:415-420 */
    int32_t count_limit, radius;
    int32_t cross_neighbor;       /* reconstruction.py:561-572 */
    int32_t coarse_enabled;
    float coarse_slopes[3];
    int32_t band_enabled[3];
    float band_scales[3];
    float factors_a[9], factors_b[9];  /* [band][channel] */
    float configured_strengths[3];
    int32_t driver_gate_primary;
    float dither_scales[3];
    float dither_low, dither_high;     /* dither.py:41-56 */
} ox_params;

typedef struct {
    int64_t attempted, written, public_advances, changed;
    uint32_t final_state;
    uint32_t startup_final_state;
    int64_t startup_attempted[6];
    int64_t startup_advances[6];
} ox_counters;

/* ======================================================================
 * L2 math primitives
 * ====================================================================== */

/* reconstruction.py:187-268: _vertical_scratch + _vertical_binomial_16 +
 * _recovered_unscaled_averages for one scalar 9x9 patch p[row][col]. */
static void ox_unscaled_averages(const float p[9][9], double out[3])
{
    float s3[9], s5[9], s7[9], s9[9], b16[9];
    const double c16 = (double)(float)(1.0 / 16.0);
    for (int x = 0; x < 9; ++x) {
        double acc = (double)p[3][x] + (double)p[4][x];
        acc += (double)p[5][x];
        s3[x] = (float)acc;
        acc += (double)p[2][x];
        acc += (double)p[6][x];
        s5[x] = (float)acc;
        acc += (double)p[1][x];
        acc += (double)p[7][x];
        s7[x] = (float)acc;
        acc += (double)p[0][x];
        acc += (double)p[8][x];
        s9[x] = (float)acc;
        const double center = (double)p[4][x];
        double b = (double)p[3][x] + center;
        b += (double)p[5][x];
        b += center;
        b16[x] = (float)(b * c16);
    }
    double t21 = (double)s3[6] + (double)s3[2];
    t21 += (double)s5[3];
    t21 += (double)s5[4];
    t21 += (double)s5[5];
    double t69 = (double)s5[8] + (double)s5[0];
    t69 += (double)s7[1];
    t69 += (double)s7[7];
    for (int x = 2; x < 7; ++x) t69 += (double)s9[x];
    double t16 = (double)b16[4] + (double)b16[3];
    t16 += (double)b16[5];
    t16 += (double)b16[4];
    out[0] = t69 * (double)(float)(1.0 / 69.0);
    out[1] = t21 * (double)(float)(1.0 / 21.0);
    out[2] = t16;
}

/* reconstruction.py:271-299: the RGB Q16 schedule (horizontal [1,2,1]
 * rows kept in binary64, one multiply by float32(1/16)). */
static double ox_rgb_q16(const float p[9][9])
{
    const double c16 = (double)(float)(1.0 / 16.0);
    double rows[3];
    for (int i = 0; i < 3; ++i) {
        const int y = 3 + i;
        const double center = (double)p[y][4];
        double h = (double)p[y][3] + (double)p[y][5];
        h += center;
        h += center;
        rows[i] = h;
    }
    double total = rows[0] + rows[1];
    total += rows[1];
    total += rows[2];
    return total * c16;
}

/* streaming.py:236-256 (_feature_record) / startup.py:166-183. */
static void ox_feature_record(const float sp[9][9], const float wp[9][9],
                              float point_aux, float point_score,
                              float fallback, float weights[4],
                              float feature[4])
{
    double w[3], n[3];
    ox_unscaled_averages(sp, w);
    weights[0] = (float)w[0];
    weights[1] = (float)w[1];
    weights[2] = (float)w[2];
    weights[3] = point_score;
    ox_unscaled_averages(wp, n);
    for (int lane = 0; lane < 3; ++lane)
        feature[lane] = (w[lane] > 0.0) ? (float)(n[lane] / w[lane]) : fallback;
    feature[3] = (weights[3] > 0.0f) ? point_aux : fallback;
}

/* reconstruction.py:425-462 with the UNNORMALIZED_SUM policy. */
static void ox_rgb_candidates(const float rp[3][9][9], const float weights[4],
                              float cand[3][3])
{
    double avg[3][3]; /* [scale][channel] */
    for (int c = 0; c < 3; ++c) {
        double q[3];
        ox_unscaled_averages(rp[c], q);
        avg[0][c] = q[0];
        avg[1][c] = q[1];
        avg[2][c] = ox_rgb_q16(rp[c]);
    }
    for (int k = 0; k < 3; ++k) {
        const float den = weights[k];
        if (den > 0.0f) {
            const double recip = 1.0 / (double)den;
            for (int c = 0; c < 3; ++c) cand[k][c] = (float)(avg[k][c] * recip);
        } else {
            for (int c = 0; c < 3; ++c) cand[k][c] = (float)avg[k][c];
        }
    }
}

static int ox_finite_f(float v) { return isfinite(v) != 0; }

/* reconstruction.py:807-887 (combine_recovered_candidate), including
 * feature_band_ranges :672-705, _automatic_strengths :745-771 and
 * asymmetric_dead_zone_residual :708-742.  Returns OX_ERR_COMBINER_INPUT
 * when the reference would raise "combiner inputs must be finite". */
static int ox_combine(const float cand[3][3], const float source[3],
                      const float weights[4], const float feats[5][4],
                      int record_count, float coarse_reference,
                      const ox_params *prm, double out[3])
{
    for (int k = 0; k < 3; ++k)
        for (int c = 0; c < 3; ++c)
            if (!ox_finite_f(cand[k][c])) return OX_ERR_COMBINER_INPUT;
    for (int c = 0; c < 3; ++c)
        if (!ox_finite_f(source[c])) return OX_ERR_COMBINER_INPUT;
    for (int l = 0; l < 4; ++l)
        if (!ox_finite_f(weights[l])) return OX_ERR_COMBINER_INPUT;
    for (int r = 0; r < record_count; ++r)
        for (int l = 0; l < 4; ++l)
            if (!ox_finite_f(feats[r][l])) return OX_ERR_COMBINER_INPUT;

    /* feature_band_ranges: float32(min/max of binary64 differences) */
    double rmin[3], rmax[3];
    for (int t = 0; t < 3; ++t) {
        double mn = (double)feats[0][t + 1] - (double)feats[0][t];
        double mx = mn;
        for (int r = 1; r < record_count; ++r) {
            const double d = (double)feats[r][t + 1] - (double)feats[r][t];
            if (d < mn) mn = d;
            if (d > mx) mx = d;
        }
        rmin[t] = (double)(float)mn;
        rmax[t] = (double)(float)mx;
    }

    /* _automatic_strengths */
    double strengths[3];
    if (prm->configured_strengths[0] == 0.0f) {
        const float doubled = (float)(2.0 * (double)weights[1]);
        double v = (double)doubled;
        double lower = 0.0; /* max(0.0, v): NaN loses the comparison */
        if (v > 0.0) lower = v;
        double clamped = 1.0; /* min(1.0, lower) */
        if (lower < 1.0) clamped = lower;
        strengths[0] = (double)(float)clamped;
    } else {
        strengths[0] = (double)prm->configured_strengths[0];
    }
    if (prm->configured_strengths[1] == 0.0f) {
        float m2 = weights[2];
        if (m2 < 0.0f) m2 = 0.0f;
        strengths[1] = (double)m2;
    } else {
        strengths[1] = (double)prm->configured_strengths[1];
    }
    if (prm->configured_strengths[2] == 0.0f)
        strengths[2] = (double)weights[3] * (double)weights[3];
    else
        strengths[2] = (double)prm->configured_strengths[2];

    double candidate[3];
    for (int c = 0; c < 3; ++c) candidate[c] = (double)cand[0][c];
    if (prm->coarse_enabled) {
        const double delta = (double)coarse_reference - (double)feats[0][0];
        for (int c = 0; c < 3; ++c)
            candidate[c] = candidate[c] + (double)prm->coarse_slopes[c] * delta;
    }
    for (int b = 0; b < 3; ++b) {
        if (!prm->band_enabled[b]) continue;
        const double scale = (double)prm->band_scales[b];
        const double emin = rmin[b], emax = rmax[b];
        const int negative = (emin < 0.0 && emax < 0.0);
        for (int c = 0; c < 3; ++c) {
            double coarse_v, fine_v;
            if (b == 0) { coarse_v = cand[0][c]; fine_v = cand[1][c]; }
            else if (b == 1) { coarse_v = cand[1][c]; fine_v = cand[2][c]; }
            else { coarse_v = cand[2][c]; fine_v = source[c]; }
            const double diff = scale * (fine_v - coarse_v);
            const double fa = (double)prm->factors_a[b * 3 + c];
            const double fb = (double)prm->factors_b[b * 3 + c];
            double upper, lower;
            if (negative) { upper = fb * emax; lower = fa * emin; }
            else { upper = fa * emax; lower = fb * emin; }
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
    return OX_OK;
}

/* dither.py:59-104 (conditional_dither_delta) with rng.py:159-172.
 * The LCG state is threaded explicitly. */
static int ox_dither_delta(double value, float scale32, float low32,
                           float high32, uint32_t *state, double *delta)
{
    const float cand32 = (float)value;
    if (!ox_finite_f(cand32) || !ox_finite_f(scale32) || !ox_finite_f(low32) ||
        !ox_finite_f(high32))
        return OX_ERR_DITHER_INPUT;
    const double cand = (double)cand32;
    const double low = (double)low32, high = (double)high32;
    *delta = 0.0;
    if (!(low < high)) return OX_OK;
    if (!(low < cand && cand < high)) return OX_OK;
    const double width = high - low;
    const double coefficient = 4.0 / (width * width);
    const double envelope = ((high - cand) * (cand - low)) * coefficient;
    const float span = (float)((double)scale32 * cand);
    *state = (125u * *state + 1u) & LCG_MASK;
    const double unit = (double)(*state + 1u) * NIKON_NORMALIZATION - 0.5;
    const double random_value = 0.0 + unit * (double)span;
    const double d = envelope * random_value;
    const double changed = cand + d;
    if (low < changed && changed < high) *delta = d;
    return OX_OK;
}

/* reconstruction.py:916-982 (write_reconstructed_pixel). */
static int ox_write_pixel(const double cand[3], const float orig[3],
                          int floor_enabled, const ox_params *prm,
                          uint32_t *state, float values[3], int64_t *advances)
{
    int valid = 1;
    for (int c = 0; c < 3; ++c)
        if (!isfinite(cand[c]) || !(cand[c] > 0.0)) valid = 0;
    *advances = 0;
    if (!valid) {
        for (int c = 0; c < 3; ++c) values[c] = orig[c];
        return OX_OK;
    }
    for (int c = 0; c < 3; ++c) {
        const uint32_t before = *state;
        double first;
        int rc = ox_dither_delta(cand[c], prm->dither_scales[c], prm->dither_low,
                                 prm->dither_high, state, &first);
        if (rc) return rc;
        *advances += (*state != before);
        if (floor_enabled && cand[c] + first <= (double)orig[c]) {
            values[c] = orig[c];
        } else {
            double d = first;
            if (floor_enabled) {
                const uint32_t before2 = *state;
                rc = ox_dither_delta(cand[c], prm->dither_scales[c],
                                     prm->dither_low, prm->dither_high, state, &d);
                if (rc) return rc;
                *advances += (*state != before2);
            }
            values[c] = (float)(cand[c] + d);
        }
    }
    return OX_OK;
}

/* output.py:61-94: work value -> public uint16 through the factor tables. */
static int ox_emit(float v, const uint32_t *hi, const uint32_t *lo, uint16_t *out)
{
    if (!ox_finite_f(v)) return OX_ERR_NONFINITE_WORK;
    double w = (double)v + 0.5;
    if (w < 0.0) w = 0.0;
    if (w > 65535.0) w = 65535.0;
    const uint32_t idx = (uint32_t)trunc(w);
    const uint64_t prod = (uint64_t)hi[idx >> 8] * (uint64_t)lo[idx & 0xFFu];
    *out = (uint16_t)((prod >> 20) - 1u);
    return OX_OK;
}

/* ======================================================================
 * Whole-image planes (streaming.py:103-149 _RowCache.get)
 * ====================================================================== */

typedef struct {
    int h, w;
    float *working; /* h*w*4 */
    float *aux;     /* h*w */
    float *score;   /* h*w */
    float *waux;    /* h*w */
    float *wrgb;    /* h*w*3 */
} ox_planes;

static void ox_free_planes(ox_planes *pl)
{
    free(pl->working);
    free(pl->aux);
    free(pl->score);
    free(pl->waux);
    free(pl->wrgb);
    memset(pl, 0, sizeof(*pl));
}

/* x3a.py:193-221 derive_auxiliary, x3a.py:245-286 continuous_score and the
 * weighted planes of streaming.py:139-147, with per-row stage parameters
 * (aux from stage y+1, score base from stage y+2). */
static int ox_build_planes(const uint16_t *px, int h, int w, const float *lut,
                           const ox_params *prm, const ox_stage *stages,
                           ox_planes *pl)
{
    const size_t n = (size_t)h * (size_t)w;
    pl->h = h;
    pl->w = w;
    pl->working = (float *)malloc(n * 4 * sizeof(float));
    pl->aux = (float *)malloc(n * sizeof(float));
    pl->score = (float *)malloc(n * sizeof(float));
    pl->waux = (float *)malloc(n * sizeof(float));
    pl->wrgb = (float *)malloc(n * 3 * sizeof(float));
    if (!pl->working || !pl->aux || !pl->score || !pl->waux || !pl->wrgb) {
        ox_free_planes(pl);
        return OX_ERR_NOMEM;
    }
    int status = OX_OK;
    int first_bad_row = h;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; ++y) {
        const ox_stage *aux_stage = &stages[y];        /* stage y+1 */
        const ox_stage *score_stage = &stages[y + 1];  /* stage y+2 */
        float *work = pl->working + (size_t)y * w * 4;
        float *aux = pl->aux + (size_t)y * w;
        for (int x = 0; x < w * 4; ++x) work[x] = lut[px[(size_t)y * w * 4 + x]];
        const float alpha32 = aux_stage->alpha;
        int bad = 0;
        if (alpha32 == 1.0f) {
            if (!aux_stage->replacement_valid) bad = 2;
            for (int x = 0; x < w; ++x) aux[x] = aux_stage->replacement;
        } else {
            const double alpha = (double)alpha32;
            const double offset = (double)aux_stage->offset;
            for (int x = 0; x < w; ++x) {
                const double vis = (double)work[x * 4 + prm->visible_channel];
                const double ir = (double)work[x * 4 + 3];
                aux[x] = (float)((ir - alpha * vis) / (1.0 - alpha) - offset);
            }
        }
        for (int x = 0; x < w; ++x)
            if (!ox_finite_f(aux[x])) bad = bad ? bad : 1;
        if (bad) {
#pragma omp critical
            {
                if (y < first_bad_row) {
                    first_bad_row = y;
                    status = (bad == 2) ? OX_ERR_ALPHA_ONE_UNBOUND
                                        : OX_ERR_NONFINITE_AUX;
                }
            }
            continue;
        }
        const double primary = (double)score_stage->score_base;
        const double addend = (double)prm->score_addend;
        const double scale = (double)prm->score_scale;
        const double offset = (double)prm->score_offset;
        const double lower = (double)prm->score_floor;
        float *score = pl->score + (size_t)y * w;
        float *waux = pl->waux + (size_t)y * w;
        float *wrgb = pl->wrgb + (size_t)y * w * 3;
        for (int x = 0; x < w; ++x) {
            float sample = aux[x];
            if (prm->horizontal_minimum && w > 2 && x > 0 && x < w - 1) {
                float m = aux[x - 1] < aux[x] ? aux[x - 1] : aux[x];
                sample = m < aux[x + 1] ? m : aux[x + 1];
            }
            double s = ((primary + addend) - (double)sample) * scale + offset;
            if (s > 1.0) s = 1.0;       /* np.minimum(score64, 1.0) */
            if (s < lower) s = lower;   /* np.maximum(score64, lower) */
            score[x] = (float)s;
            waux[x] = score[x] * aux[x];
            for (int c = 0; c < 3; ++c) wrgb[x * 3 + c] = score[x] * work[x * 4 + c];
        }
    }
    if (status != OX_OK) ox_free_planes(pl);
    return status;
}

/* ======================================================================
 * History boundary rules for public rows
 * (streaming.py:201-233 _history_window; reconstruction.py:39-82)
 * ====================================================================== */

static inline float ox_hist_score(const ox_planes *pl, float floor, int y, int x)
{
    if (x < 0 || x >= pl->w || y < -1) return 0.0f;
    if (y == -1) return floor;
    if (y >= pl->h) y = pl->h - 1;
    return pl->score[(size_t)y * pl->w + x];
}

static inline float ox_hist_waux(const ox_planes *pl, float floor, int y, int x)
{
    if (x < 0 || x >= pl->w || y < -1) return 0.0f;
    if (y == -1) return pl->aux[x] * floor;
    if (y >= pl->h) y = pl->h - 1;
    return pl->waux[(size_t)y * pl->w + x];
}

static inline float ox_hist_wrgb(const ox_planes *pl, float floor, int y, int x, int c)
{
    if (x < 0 || x >= pl->w || y < -1) return 0.0f;
    if (y == -1) return pl->working[(size_t)x * 4 + c] * floor;
    if (y >= pl->h) y = pl->h - 1;
    return pl->wrgb[((size_t)y * pl->w + x) * 3 + c];
}

/* streaming.py:236-308: the record centred at (cy, cx) of the public
 * history, with the point rule for rows above/below the image. */
static void ox_public_record(const ox_planes *pl, float floor, int cy, int cx,
                             float fallback, float weights[4], float feature[4])
{
    float sp[9][9], wp[9][9];
    for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j) {
            sp[i][j] = ox_hist_score(pl, floor, cy - 4 + i, cx - 4 + j);
            wp[i][j] = ox_hist_waux(pl, floor, cy - 4 + i, cx - 4 + j);
        }
    float point_aux, point_score;
    if (cy < 0) {
        point_aux = pl->aux[cx];
        point_score = floor;
    } else {
        const int yy = cy >= pl->h ? pl->h - 1 : cy;
        point_aux = pl->aux[(size_t)yy * pl->w + cx];
        point_score = pl->score[(size_t)yy * pl->w + cx];
    }
    ox_feature_record(sp, wp, point_aux, point_score, fallback, weights, feature);
}

/* streaming.py:157-198 (_decision_fallback_row, edge-replicated). */
static int ox_decision_fallback(const ox_planes *pl, const ox_params *prm, int y, int x)
{
    const int h = pl->h, w = pl->w, r = prm->radius;
    const float thr = prm->decision_threshold;
    int left = x - r, right = x + r;
    if (left < 0) left = 0;
    if (left > w - 1) left = w - 1;
    if (right < 0) right = 0;
    if (right > w - 1) right = w - 1;
    int vl = 0, vr = 0;
    for (int dy = -4; dy <= 4; ++dy) {
        int yy = y + dy;
        if (yy < 0) yy = 0;
        if (yy > h - 1) yy = h - 1;
        vl += pl->aux[(size_t)yy * w + left] < thr;
        vr += pl->aux[(size_t)yy * w + right] < thr;
    }
    int ay = y - r, by = y + r;
    if (ay < 0) ay = 0;
    if (by > h - 1) by = h - 1;
    int ha = 0, hb = 0;
    for (int dx = -4; dx <= 4; ++dx) {
        int xx = x + dx;
        if (xx < 0) xx = 0;
        if (xx > w - 1) xx = w - 1;
        ha += pl->aux[(size_t)ay * w + xx] < thr;
        hb += pl->aux[(size_t)by * w + xx] < thr;
    }
    const int lim = prm->count_limit;
    return (vl > lim) || (ha > lim) || (vr > lim) || (hb > lim);
}

/* One public row's RNG-free analysis (streaming.py:444-521; the same split
 * as fast_cpu/kernels.py:859-1068).  Writes attempted flags and combined
 * candidates for the row. */
static int ox_analyze_row(const ox_planes *pl, const ox_params *prm,
                          const ox_stage *stages, int y, uint8_t *attempted,
                          double *cands)
{
    const int w = pl->w;
    const ox_stage *ws = &stages[y + 6]; /* writer stage y+7 */
    const int floor_enabled = prm->driver_gate_primary || ws->gate_secondary;
    const float fallback = ws->coarse;
    const float floor = prm->score_floor;
    const int records = prm->cross_neighbor ? 5 : 1;
    for (int x = 0; x < w; ++x) {
        attempted[x] = 0;
        if (ox_decision_fallback(pl, prm, y, x)) continue;
        if (ws->row_gate != 0) continue;
        if (floor_enabled && !(pl->score[(size_t)y * w + x] < 1.0f)) continue;
        float weights[4], feats[5][4];
        ox_public_record(pl, floor, y, x, fallback, weights, feats[0]);
        /* reconstruction.py:890-904 driver_forces_fallback */
        if (ws->row_gate != 0) continue;
        if (floor_enabled && weights[3] >= 1.0f) continue;
        if (records == 5) {
            static const int dys[4] = {0, 0, -1, 1};
            static const int dxs[4] = {-1, 1, 0, 0};
            for (int k = 0; k < 4; ++k) {
                const int nx = x + dxs[k], ny = y + dys[k];
                float wn[4];
                if (nx < 0 || nx >= w) {
                    for (int l = 0; l < 4; ++l) feats[k + 1][l] = 0.0f;
                    continue;
                }
                ox_public_record(pl, floor, ny, nx, fallback, wn, feats[k + 1]);
            }
        }
        float rp[3][9][9];
        for (int i = 0; i < 9; ++i)
            for (int j = 0; j < 9; ++j)
                for (int c = 0; c < 3; ++c)
                    rp[c][i][j] = ox_hist_wrgb(pl, floor, y - 4 + i, x - 4 + j, c);
        float cand[3][3];
        ox_rgb_candidates(rp, weights, cand);
        float source[3];
        for (int c = 0; c < 3; ++c) source[c] = pl->working[((size_t)y * w + x) * 4 + c];
        const int rc = ox_combine(cand, source, weights, feats, records,
                                  ws->coarse, prm, &cands[(size_t)x * 3]);
        if (rc) return rc;
        attempted[x] = 1;
    }
    return OX_OK;
}

/* ======================================================================
 * Hidden startup replay (startup.py:74-353)
 * ====================================================================== */

typedef struct {
    const ox_planes *pl;
    int rows;     /* first_row_count: 5 (cross) or 4 */
    float floor;
} ox_startup_ctx;

/* startup.py:74-128 history rules, evaluated lazily. */
static inline float ox_su_score(const ox_startup_ctx *s, int y, int x)
{
    if (x < 0 || x >= s->pl->w) return 0.0f;
    if (y == -1) return s->floor;
    if (y >= 0 && y < s->rows) return s->pl->score[(size_t)y * s->pl->w + x];
    return 0.0f;
}

static inline float ox_su_waux(const ox_startup_ctx *s, int y, int x)
{
    if (x < 0 || x >= s->pl->w) return 0.0f;
    const size_t w = s->pl->w;
    if (y == -1) return s->pl->aux[x] * s->floor;
    if (y >= 0 && y < s->rows) return s->pl->score[y * w + x] * s->pl->aux[y * w + x];
    return 0.0f;
}

static inline float ox_su_wrgb(const ox_startup_ctx *s, int y, int x, int c)
{
    if (x < 0 || x >= s->pl->w) return 0.0f;
    const size_t w = s->pl->w;
    if (y == -1) return s->pl->working[(size_t)x * 4 + c] * s->floor;
    if (y >= 0 && y < s->rows)
        return s->pl->score[y * w + x] * s->pl->working[(y * w + x) * 4 + c];
    return 0.0f;
}

/* Raw decision history (startup.py:119-126), addressed by padded column
 * xp = x + 4: the left guard replicates, the right guard replicates only
 * for real rows (negative rows keep the allocator-zero guard). */
static inline float ox_su_raw(const ox_startup_ctx *s, int y, int xp)
{
    const int w = s->pl->w;
    const float *src = s->pl->aux + (size_t)(y < 0 ? 0 : y) * w;
    if (xp < 4) return src[0];
    if (xp < 4 + w) return src[xp - 4];
    return y >= 0 ? src[w - 1] : 0.0f;
}

/* startup.py:131-183 */
static void ox_su_record(const ox_startup_ctx *s, int ly, int x, float fallback,
                         float weights[4], float feature[4])
{
    if (ly <= -6 || x < 0 || x >= s->pl->w) {
        for (int l = 0; l < 4; ++l) weights[l] = feature[l] = 0.0f;
        return;
    }
    float sp[9][9], wp[9][9];
    for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j) {
            sp[i][j] = ox_su_score(s, ly - 4 + i, x - 4 + j);
            wp[i][j] = ox_su_waux(s, ly - 4 + i, x - 4 + j);
        }
    double wq[3], nq[3];
    ox_unscaled_averages(sp, wq);
    weights[0] = (float)wq[0];
    weights[1] = (float)wq[1];
    weights[2] = (float)wq[2];
    weights[3] = ox_su_score(s, ly, x);
    ox_unscaled_averages(wp, nq);
    for (int lane = 0; lane < 3; ++lane)
        feature[lane] = (wq[lane] > 0.0) ? (float)(nq[lane] / wq[lane]) : fallback;
    feature[3] = (weights[3] > 0.0f) ? ox_su_raw(s, ly, x + 4) : fallback;
}

static inline int ox_max1(int v) { return v < 1 ? 1 : v; }

/* startup.py:186-353 (replay_hidden_startup_rows). */
static int ox_startup(const ox_planes *pl, const ox_params *prm,
                      const ox_stage *stages, uint32_t *state,
                      ox_counters *ctr)
{
    ox_startup_ctx s;
    s.pl = pl;
    s.rows = prm->cross_neighbor ? 5 : 4;
    s.floor = prm->score_floor;
    if (pl->h < s.rows) return OX_ERR_GEOMETRY;
    if (!(s.floor > 0.0f) || !ox_finite_f(s.floor)) return OX_ERR_ARG;
    const int w = pl->w;
    const int r = prm->radius;
    const int records = prm->cross_neighbor ? 5 : 1;
    for (int center = -6; center <= -1; ++center) {
        const int hit = center + 7;
        const ox_stage *act = &stages[hit - 1];
        const int floor_enabled = prm->driver_gate_primary || act->gate_secondary;
        const int writer_width = (prm->cross_neighbor && hit <= 2) ? w - 4 : w;
        if (writer_width < 0) return OX_ERR_GEOMETRY;
        const float fb_center = stages[ox_max1(center + 6) - 1].coarse;
        const float fb_up = stages[ox_max1(center + 5) - 1].coarse;
        const float fb_down = stages[ox_max1(center + 7) - 1].coarse;
        int64_t attempted = 0, advances = 0;
        for (int x = 0; x < writer_width; ++x) {
            /* x3a.py:366-385 bars + x3a.py:388-406 group fallback */
            int fallback_hit = 0;
            for (int g = 0; g < 4 && !fallback_hit; ++g) {
                int count = 0;
                for (int k = 0; k < 9; ++k) {
                    const int axis = k - 4;
                    int dy, dx;
                    if (g == 0) { dy = axis; dx = -r; }
                    else if (g == 1) { dy = -r; dx = axis; }
                    else if (g == 2) { dy = axis; dx = r; }
                    else { dy = r; dx = axis; }
                    count += ox_su_raw(&s, center + dy, x + 4 + dx) < prm->decision_threshold;
                }
                if (count > prm->count_limit) fallback_hit = 1;
            }
            float weights[4], feats[5][4];
            ox_su_record(&s, center, x, fb_center, weights, feats[0]);
            if (fallback_hit) continue;
            if (act->row_gate != 0) continue;
            if (floor_enabled && weights[3] >= 1.0f) continue;
            ++attempted;
            float rp[3][9][9];
            for (int i = 0; i < 9; ++i)
                for (int j = 0; j < 9; ++j)
                    for (int c = 0; c < 3; ++c)
                        rp[c][i][j] = ox_su_wrgb(&s, center - 4 + i, x - 4 + j, c);
            float cand[3][3];
            ox_rgb_candidates(rp, weights, cand);
            if (records == 5) {
                float wn[4];
                ox_su_record(&s, center, x - 1, fb_center, wn, feats[1]);
                ox_su_record(&s, center, x + 1, fb_center, wn, feats[2]);
                ox_su_record(&s, center - 1, x, fb_up, wn, feats[3]);
                ox_su_record(&s, center + 1, x, fb_down, wn, feats[4]);
            }
            const float *orig = pl->working + (size_t)x * 4; /* row 0 */
            float source[3] = {orig[0], orig[1], orig[2]};
            double combined[3];
            int rc = ox_combine(cand, source, weights, feats, records, act->coarse,
                                prm, combined);
            if (rc) return rc;
            float values[3];
            int64_t adv;
            rc = ox_write_pixel(combined, source, floor_enabled, prm, state, values, &adv);
            if (rc) return rc;
            advances += adv;
        }
        ctr->startup_attempted[hit - 1] = attempted;
        ctr->startup_advances[hit - 1] = advances;
    }
    ctr->startup_final_state = *state;
    return OX_OK;
}

/* ======================================================================
 * Full replay (streaming.py:365-552)
 * ====================================================================== */

int ox_replay(const uint16_t *px, int h, int w, const float *lut,
              const ox_params *prm, const ox_stage *stages,
              uint32_t rng_state, const uint32_t *factor_hi,
              const uint32_t *factor_lo, uint16_t *out_rgb,
              float *score_out, uint8_t *changed_out, ox_counters *ctr,
              int threads)
{
    if (!px || !lut || !prm || !stages || !out_rgb || !ctr || h < 1 || w < 1)
        return OX_ERR_ARG;
    if (h < 4) return OX_ERR_GEOMETRY;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    memset(ctr, 0, sizeof(*ctr));
    ox_planes pl;
    memset(&pl, 0, sizeof(pl));
    int rc = ox_build_planes(px, h, w, lut, prm, stages, &pl);
    if (rc) return rc;
    uint32_t state = rng_state & LCG_MASK;
    rc = ox_startup(&pl, prm, stages, &state, ctr);
    if (rc) { ox_free_planes(&pl); return rc; }

    uint8_t *att = (uint8_t *)malloc((size_t)h * w);
    double *cands = (double *)malloc((size_t)h * w * 3 * sizeof(double));
    if (!att || !cands) { free(att); free(cands); ox_free_planes(&pl); return OX_ERR_NOMEM; }
    int status = OX_OK;
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < h; ++y) {
        const int r = ox_analyze_row(&pl, prm, stages, y, att + (size_t)y * w,
                                     cands + (size_t)y * w * 3);
        if (r) {
#pragma omp critical
            { if (status == OX_OK) status = r; }
        }
    }
    if (status) { free(att); free(cands); ox_free_planes(&pl); return status; }

    /* Serial writer, emit and counters in row-major order. */
    float values[3];
    for (int y = 0; y < h && status == OX_OK; ++y) {
        const ox_stage *ws = &stages[y + 6];
        const int floor_enabled = prm->driver_gate_primary || ws->gate_secondary;
        for (int x = 0; x < w; ++x) {
            const size_t i = (size_t)y * w + x;
            const float *orig = pl.working + i * 4;
            float out[3] = {orig[0], orig[1], orig[2]};
            if (att[i]) {
                int64_t adv;
                status = ox_write_pixel(cands + i * 3, orig, floor_enabled, prm,
                                        &state, values, &adv);
                if (status) break;
                ctr->attempted += 1;
                ctr->public_advances += adv;
                if (values[0] != orig[0] || values[1] != orig[1] || values[2] != orig[2])
                    ctr->written += 1;
                out[0] = values[0];
                out[1] = values[1];
                out[2] = values[2];
            }
            int changed = 0;
            for (int c = 0; c < 3; ++c) {
                uint16_t e, e0;
                status = ox_emit(out[c], factor_hi, factor_lo, &e);
                if (status) break;
                status = ox_emit(orig[c], factor_hi, factor_lo, &e0);
                if (status) break;
                out_rgb[i * 3 + c] = e;
                changed |= (e != e0);
            }
            if (status) break;
            ctr->changed += changed;
            if (changed_out) changed_out[i] = (uint8_t)changed;
        }
    }
    ctr->final_state = state;
    if (score_out && status == OX_OK)
        memcpy(score_out, pl.score, (size_t)h * w * sizeof(float));
    free(att);
    free(cands);
    ox_free_planes(&pl);
    return status;
}

/* ======================================================================
 * Calibration prelude
 * ====================================================================== */

static void put_u32(uint8_t *p, int off, uint32_t v) { memcpy(p + off, &v, 4); }
static void put_f32(uint8_t *p, int off, float v) { memcpy(p + off, &v, 4); }
static void put_f64(uint8_t *p, int off, double v) { memcpy(p + off, &v, 8); }

/* prepass.py:325-341 */
static float ox_pp_quadrant(const float v[8][8], int fy, int fx)
{
    double total = 0.0;
    for (int y = fy; y < fy + 4; ++y)
        for (int x = fx; x < fx + 4; ++x) total += (double)v[y][x];
    return (float)(total * 0.0625);
}

/* prepass.py:96-236 (reduce_prepass_frame) with a fresh (all-zero) prior
 * record and the captured LS-5000 selector-8 parameters (prepass.py:42-53). */
int ox_prepass(const uint16_t *px, int h, int w, const float *lut,
               uint8_t payload[64], int64_t *valid_pixels, int64_t *fully_valid_tiles)
{
    if (!px || !lut || h < 1 || w < 1) return OX_ERR_ARG;
    const float threshold = 8847.2255859375f;
    const double ratio_min = (double)-0.2f, ratio_max = (double)0.2f;
    const double alpha_scale = (double)1.5f;
    const int ph = (h + 7) & ~7, pw = (w + 7) & ~7;
    double cal_r = 0.0, cal_ir = 0.0, cal_sq = 0.0;
    float reg_den = 0.0f, reg_num = 0.0f;
    int64_t valid = 0, tiles = 0;
    for (int fy = 0; fy < ph; fy += 8) {
        for (int fx = 0; fx < pw; fx += 8) {
            float rr[8][8], ri[8][8];
            float sum_raw_ir = 0.0f;
            int tile_valid = 1;
            for (int y = 0; y < 8; ++y) {
                for (int x = 0; x < 8; ++x) {
                    const int yy = fy + y, xx = fx + x;
                    uint32_t raw_r = 0, raw_ir = 0;
                    if (yy < h && xx < w) {
                        raw_r = px[((size_t)yy * w + xx) * 4 + 0];
                        raw_ir = px[((size_t)yy * w + xx) * 4 + 3];
                    }
                    if ((float)raw_ir <= threshold) { tile_valid = 0; continue; }
                    ++valid;
                    const float cr = lut[raw_r], ci = lut[raw_ir];
                    rr[y][x] = cr;
                    ri[y][x] = ci;
                    const double sq = (double)((uint64_t)raw_ir * raw_ir);
                    cal_r += sq * (double)cr;
                    cal_ir += sq * (double)ci;
                    cal_sq += sq;
                    sum_raw_ir = (float)((double)sum_raw_ir + (double)raw_ir);
                }
            }
            if (!tile_valid) continue;
            ++tiles;
            float rm[4], im[4];
            const int qy[4] = {0, 0, 4, 4}, qx[4] = {0, 4, 0, 4};
            for (int q = 0; q < 4; ++q) {
                rm[q] = ox_pp_quadrant(rr, qy[q], qx[q]);
                im[q] = ox_pp_quadrant(ri, qy[q], qx[q]);
            }
            /* prepass.py:344-351 */
            double tr = (double)rm[0]; tr += rm[1]; tr += rm[2]; tr += rm[3];
            double ti = (double)im[0]; ti += im[1]; ti += im[2]; ti += im[3];
            const float rg = (float)(tr * 0.25), ig = (float)(ti * 0.25);
            double den = (double)reg_den, num = (double)reg_num;
            const double scalar = (double)sum_raw_ir;
            for (int q = 0; q < 4; ++q) {
                const float rd = (float)((double)rm[q] - (double)rg);
                const float id = (float)((double)im[q] - (double)ig);
                if (rd == 0.0f) continue;
                const double ratio = (double)id / (double)rd;
                if (ratio < ratio_min || ratio > ratio_max) continue;
                const double weight = (double)rd * (double)rd * scalar * scalar;
                den += weight;
                num += ratio * weight;
            }
            reg_den = (float)den;
            reg_num = (float)num;
        }
    }
    double unrounded;
    if (reg_den == 0.0f) unrounded = (double)0.17f;
    else unrounded = (double)reg_num / (double)reg_den;
    const float alpha = (float)unrounded;
    const float scaled = (float)(unrounded * alpha_scale);
    memset(payload, 0, 64);
    put_u32(payload, 0x00, 1u);
    put_f32(payload, 0x04, alpha);
    put_f32(payload, 0x08, scaled);
    put_f64(payload, 0x10, cal_r);
    put_f64(payload, 0x18, cal_ir);
    put_f64(payload, 0x20, cal_sq);
    if (cal_sq != 0.0) {
        put_f32(payload, 0x28, (float)(cal_r / cal_sq));
        put_f32(payload, 0x2C, (float)(cal_ir / cal_sq));
    }
    put_f32(payload, 0x30, reg_den);
    put_f32(payload, 0x34, reg_num);
    put_u32(payload, 0x38, 16u);
    if (valid_pixels) *valid_pixels = valid;
    if (fully_valid_tiles) *fully_valid_tiles = tiles;
    return OX_OK;
}

/* producer_parameters.py:136-167: the asymmetric x87 tree. */
static float ox_prod_quadrant(const float v[8][8], int ry, int cx)
{
    double first = (double)v[ry][cx];
    first += (double)v[ry][cx + 1];
    first += (double)v[ry][cx + 2];
    first += (double)v[ry][cx + 3];
    first += (double)v[ry + 1][cx];
    first += (double)v[ry + 1][cx + 1];
    const double second_tail = (double)v[ry + 1][cx + 2] + (double)v[ry + 1][cx + 3];
    first += second_tail;
    double third = (double)v[ry + 2][cx] + (double)v[ry + 2][cx + 1];
    const double third_tail = (double)v[ry + 2][cx + 2] + (double)v[ry + 2][cx + 3];
    third += third_tail;
    double fourth = (double)v[ry + 3][cx] + (double)v[ry + 3][cx + 1];
    const double fourth_tail = (double)v[ry + 3][cx + 2] + (double)v[ry + 3][cx + 3];
    fourth += fourth_tail;
    third += fourth;
    const double total = first + third;
    return (float)(total * 0.0625);
}

/* producer_parameters.py:170-180 */
static void ox_prod_center(const float q[4], float out[4])
{
    double t = (double)q[0];
    t += (double)q[1];
    t += (double)q[2];
    t += (double)q[3];
    const float mean = (float)(t * 0.25);
    for (int i = 0; i < 4; ++i) out[i] = (float)((double)q[i] - (double)mean);
}

/* producer_parameters.py:183-263 (_scale_epoch_additions) for the eight
 * rows ending at `last_row`. */
static void ox_scale_epoch(const uint16_t *px, int w, int active_width, int last_row,
                           const float *lut, float *add_den, float *add_num)
{
    const float threshold = 8847.2255859375f;
    const double low = (double)-0.125f, full_low = 0.0, full_high = (double)0.3f;
    const double high = (double)0.425f, outer = (double)0.70710677f;
    const double thr = (double)threshold;
    double den = 0.0, num = 0.0;
    const int start = last_row - 7;
    for (int col = 0; col < active_width; col += 8) {
        int ok = 1;
        for (int y = 0; y < 8 && ok; ++y)
            for (int x = 0; x < 8; ++x)
                if ((double)px[((size_t)(start + y) * w + col + x) * 4 + 3] <= thr) { ok = 0; break; }
        if (!ok) continue;
        float vr[8][8], ir[8][8];
        float raw_sum = 0.0f;
        for (int y = 0; y < 8; ++y)
            for (int x = 0; x < 8; ++x) {
                const uint16_t *p = px + ((size_t)(start + y) * w + col + x) * 4;
                vr[y][x] = lut[p[0]];
                ir[y][x] = lut[p[3]];
                raw_sum = (float)((double)raw_sum + (double)p[3]);
            }
        const int qy[4] = {0, 0, 4, 4}, qx[4] = {0, 4, 0, 4};
        float vq[4], iq[4], vd[4], id[4];
        for (int q = 0; q < 4; ++q) {
            vq[q] = ox_prod_quadrant(vr, qy[q], qx[q]);
            iq[q] = ox_prod_quadrant(ir, qy[q], qx[q]);
        }
        ox_prod_center(vq, vd);
        ox_prod_center(iq, id);
        const double rs = (double)raw_sum;
        for (int q = 0; q < 4; ++q) {
            const double vw = (double)vd[q];
            double ratio, weight;
            if (vw == 0.0) { ratio = 0.0; weight = 0.0; }
            else {
                ratio = (double)id[q] / vw;
                if (ratio < low || ratio > high) weight = 0.0;
                else if (ratio < full_low || ratio > full_high) weight = vw * outer;
                else weight = vw;
            }
            double term = weight * weight;
            term *= rs;
            term *= rs;
            den += term;
            num += ratio * term;
        }
    }
    *add_den = (float)den;
    *add_num = (float)num;
}

/* producer_parameters.py:266-495 (derive_producer_mean_schedule +
 * derive_producer_record_schedule) with the R4000 defaults (:36-49).
 * Outputs one float32 per row for each record field the setter reads. */
int ox_producer(const uint16_t *px, int h, int w, const float *lut,
                float *p1_out, float *p2_out, float *mean_vis_out,
                float *mean_ir_out, double *cum_vis, double *cum_ir,
                double *cum_w, uint32_t *accepted_out)
{
    if (!px || !lut || h < 1 || w < 1) return OX_ERR_ARG;
    const int active_width = (w / 8) * 8;
    if (active_width <= 0) return OX_ERR_GEOMETRY;
    const double thr = (double)8847.2255859375f;
    const int cells = (active_width + 7) / 8;
    uint8_t *valid = (uint8_t *)malloc((size_t)cells);
    if (!valid) return OX_ERR_NOMEM;
    double tv = 0.0, ti = 0.0, tw = 0.0;
    float mv = 46618.78515625f, mi = 56239.65625f;
    for (int row = 0; row < h; ++row) {
        if (row % 8 == 0) memset(valid, 1, (size_t)cells);
        double rv = 0.0, ri = 0.0, rw = 0.0;
        uint32_t acc = 0;
        for (int col = 0; col < active_width; ++col) {
            const int cell = col / 8;
            if (!valid[cell]) continue;
            const uint16_t *p = px + ((size_t)row * w + col) * 4;
            const uint32_t raw_ir = p[3];
            if (!(thr < (double)raw_ir)) { valid[cell] = 0; continue; }
            const double weight = (double)((uint64_t)raw_ir * raw_ir);
            rv += weight * (double)lut[p[0]];
            ri += weight * (double)lut[raw_ir];
            rw += weight;
            ++acc;
        }
        tv += rv;
        ti += ri;
        tw += rw;
        if (tw != 0.0) {
            mv = (float)(tv / tw);
            mi = (float)(ti / tw);
        }
        if (cum_vis) cum_vis[row] = tv;
        if (cum_ir) cum_ir[row] = ti;
        if (cum_w) cum_w[row] = tw;
        mean_vis_out[row] = mv;
        mean_ir_out[row] = mi;
        if (accepted_out) accepted_out[row] = acc;
    }
    free(valid);
    const float mult = 1.5f;
    float p1 = 0.15f, p2 = 0.15f, den = 0.0f, num = 0.0f;
    for (int row = 0; row < h; ++row) {
        if (row % 8 == 7) {
            float ad, an;
            ox_scale_epoch(px, w, active_width, row, lut, &ad, &an);
            const double dw = (double)den + (double)ad;
            const double nw = (double)num + (double)an;
            den = (float)dw;
            num = (float)nw;
            if (dw != 0.0) {
                const double ratio = nw / dw;
                p2 = (float)ratio;
                p1 = (float)((double)mult * ratio);
            }
        }
        p1_out[row] = p1;
        p2_out[row] = p2;
    }
    return OX_OK;
}

/* stage_parameters.py:93-128 (derive_x3a_setter_fields) and :151-197
 * (StageCalibration.from_setter_inputs), driven by
 * producer_parameters.py:498-541: stage s (1-based) reads producer row
 * min(s-1, h-1) and the table holds stages 1..h+6. */
int ox_stage_table(int h, const float *p1_rows, const float *p2_rows,
                   const float *mean_vis_rows, const float *mean_ir_rows,
                   float factor_b, ox_stage *stages)
{
    if (h < 1 || !stages) return OX_ERR_ARG;
    for (int s = 1; s <= h + 6; ++s) {
        const int row = (s - 1) < (h - 1) ? (s - 1) : (h - 1);
        float p1 = p1_rows[row], p2 = p2_rows[row];
        const float p3 = mean_vis_rows[row], p4 = mean_ir_rows[row];
        if (!ox_finite_f(p1) || !ox_finite_f(p2) || !ox_finite_f(p3) || !ox_finite_f(p4))
            return OX_ERR_STAGE_NONFINITE;
        if (p2 < 0.0f) { p1 = -p1; p2 = -p2; }
        const double d1 = 1.0 - (double)p1, d2 = 1.0 - (double)p2;
        if (d1 == 0.0 || d2 == 0.0) return OX_ERR_SETTER_ONE;
        const float base = (float)(((double)p4 - (double)p3 * (double)p2) / d2);
        const int gate_secondary = !(p3 != 0.0f && p2 <= 0.075f);
        const float alpha = p2 * factor_b;
        if (!ox_finite_f(alpha) || !ox_finite_f(base)) return OX_ERR_STAGE_NONFINITE;
        ox_stage *st = &stages[s - 1];
        st->alpha = alpha;
        st->offset = 1.0f;
        st->replacement = base;
        st->replacement_valid = 1;
        st->score_base = base;
        st->coarse = base;
        st->gate_secondary = gate_secondary;
        st->row_gate = 0;
    }
    return OX_OK;
}

/* Sizes for the ctypes wrapper to verify struct layouts. */
int ox_sizeof_params(void) { return (int)sizeof(ox_params); }
int ox_sizeof_stage(void) { return (int)sizeof(ox_stage); }
int ox_sizeof_counters(void) { return (int)sizeof(ox_counters); }
