/*
 * fauxice_b200.h -- C ABI of the B200 Digital ICE processing core.
 *
 * One shared library, libfauxice_b200.so, built for sm_100a.  Every entry
 * point takes plain pointers and sizes and returns an int status (FX_OK on
 * success); no C++ exception crosses the boundary.  Host buffers are caller
 * owned; device memory is owned by the context.
 *
 * The reference package (portable_digital_ice 0.3.1) has no foreign-function
 * interface of its own: its backends are Python functions.  Each entry point
 * below states which reference function (src/portable_digital_ice/...:line)
 * it stands in for, so a Python shim can expose the reference's backend
 * contract (process_cuda / run_streaming_replay_cuda signatures) on top.
 */
#ifndef FAUXICE_B200_H
#define FAUXICE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define FX_API __attribute__((visibility("default")))
#else
#define FX_API
#endif

#define FX_ABI_VERSION 1

/* Status codes.  The non-finite and geometry codes carry the same meaning as
 * the ValueError messages the reference raises (messages in comments). */
enum fx_status {
    FX_OK = 0,
    FX_ERR_INVALID_ARGUMENT = 1,
    FX_ERR_NO_DEVICE = 2,          /* no CUDA device visible */
    FX_ERR_UNSUPPORTED_DEVICE = 3, /* not an sm_100 (B200-class) device */
    FX_ERR_OUT_OF_MEMORY = 4,      /* device allocation / admission failed */
    FX_ERR_NONFINITE_AUX = 5,      /* "auxiliary score input must be a finite HxW plane" */
    FX_ERR_NONFINITE_WORK = 6,     /* "work RGB must be finite" */
    FX_ERR_COMBINER_INPUT = 7,     /* "combiner inputs must be finite" */
    FX_ERR_DITHER_INPUT = 8,       /* "dither inputs must be finite" */
    FX_ERR_SETTER_ONE = 9,         /* "X3A setter scale cannot equal one" */
    FX_ERR_STAGE_NONFINITE = 10,   /* stage calibration field not finite float32 */
    FX_ERR_ALPHA_ONE_UNBOUND = 11, /* "alpha==1 requires the runtime-configured ..." */
    FX_ERR_GEOMETRY = 12,          /* frame too small for the startup replay */
    FX_ERR_CANCELLED = 13,
    FX_ERR_TIMEOUT = 14,
    FX_ERR_CUDA = 15,              /* a CUDA runtime call failed */
    FX_ERR_INTERNAL = 16,          /* a device self-consistency check failed */
    FX_ERR_TABLES = 17,            /* fx_set_tables was not called */
    FX_PENDING = 18                /* fx_poll: request still running */
};

/* Constants of the hot path, as float32 values.  Field meanings follow the
 * reference's AuxiliaryParameters / ScoreParameters (x3a.py:166-242),
 * DecisionParameters (x3a.py:337-348), ReconstructionParameters
 * (reconstruction.py:613-669) and DitherBounds (dither.py:34-56). */
typedef struct fx_params {
    float score_addend, score_scale, score_offset, score_floor;
    int32_t horizontal_minimum; /* cutoff < resolution metric (x3a.py:266-268) */
    int32_t visible_channel;    /* 0, 1 or 2 */
    float decision_threshold;
    int32_t count_limit, radius;
    int32_t cross_neighbor;     /* metric > cross-neighbor cutoff */
    int32_t coarse_enabled;
    float coarse_slopes[3];
    int32_t band_enabled[3];
    float band_scales[3];
    float factors_a[9], factors_b[9]; /* [band][channel] */
    float configured_strengths[3];
    int32_t driver_gate_primary;
    float dither_scales[3];
    float dither_low, dither_high;
} fx_params;

/* Dynamic calibration of one scheduler stage (stage_parameters.py:131-149).
 * A table holds stages 1..H+6 at indices 0..H+5.  Row y reads the auxiliary
 * fields of stage y+1, the score base of stage y+2 and the writer fields of
 * stage y+7 (stage_parameters.py:207-232). */
typedef struct fx_stage {
    float alpha, offset, replacement;
    int32_t replacement_valid;
    float score_base, coarse;
    int32_t gate_secondary, row_gate;
} fx_stage;

/* StreamingReplayResult / StartupReplayResult counters
 * (streaming.py:63-75, startup.py:37-43). */
typedef struct fx_counters {
    int64_t attempted, written, public_advances, changed;
    uint32_t final_state, startup_final_state;
    int64_t startup_attempted[6];
    int64_t startup_advances[6];
    int64_t rng_dependent;  /* channels whose draw count depends on the state
                               (no reference counterpart) */
    int64_t walk_fallbacks; /* walk segments resolved by the exact serial path */
    int64_t walk_candidate_steps, walk_candidates, walk_survivors; /* walk work */
    int64_t walk_packed_segments; /* segments whose settled phase ran two
                                     candidates per lane (walk diagnostics) */
    int64_t capacity_reruns;      /* 1 when the pass ran a second time because
                                     its RNG-dependent list overflowed (later
                                     passes of the context list that many
                                     channels per site) */
} fx_counters;

/* One frame for fx_process / fx_submit.  Host pointers. */
typedef struct fx_frame {
    const uint16_t *main_rgbi; /* H x W x 4, C order */
    int32_t height, width;
    const fx_params *params;
    const fx_stage *stages;    /* H+6 entries, or NULL: derive them on the device
                                  from the frame (content-derived provider) */
    uint32_t rng_state;        /* 24-bit LCG state at job start (0x3045) */
    uint16_t *rgb_out;         /* H x W x 3 */
    float *score_out;          /* optional H x W */
    uint8_t *changed_out;      /* optional H x W */
} fx_frame;

typedef struct fx_context fx_context;

/* Library ABI version (FX_ABI_VERSION). */
FX_API int fx_version(void);

/* 0 when `device` is a usable sm_100 GPU; otherwise a status and a reason.
 * Stands in for the device probe of cuda_backend/engine.py:168-224. */
FX_API int fx_device_check(int device, char *reason, size_t reason_len);

FX_API int fx_context_create(int device, fx_context **out);
FX_API void fx_context_destroy(fx_context *ctx);

/* Last error text of the context (or of the library when ctx is NULL). */
FX_API int fx_last_error(const fx_context *ctx, char *buf, size_t len);

/* Upload the response LUT (x3a.py:111-132) and the two inverse-response
 * factor tables (output.py:40-58).  The caller hash-checks them.  The call
 * also builds, on the device, the emitted value of every raw sample (the
 * output of every unattempted channel), and refuses a LUT holding a
 * non-finite value with FX_ERR_NONFINITE_WORK ("work RGB must be finite");
 * the context then has no tables until a valid set is uploaded. */
FX_API int fx_set_tables(fx_context *ctx, const float *lut65536, const uint32_t *high256,
                         const uint32_t *low256);

/* prepass.py:96-236 (reduce_prepass_frame) for a fresh record with the
 * captured selector-8 parameters; host computation. */
FX_API int fx_reduce_prepass(const uint16_t *prepass_rgbi, int32_t height, int32_t width,
                             const float *lut65536, uint8_t payload[64], int64_t *valid_pixels,
                             int64_t *fully_valid_tiles);

/* producer_parameters.py:266-495 (derive_producer_record_schedule) on the
 * device: the four per-row record fields the X3A setter reads. */
FX_API int fx_producer_rows(fx_context *ctx, const uint16_t *main_rgbi, int32_t height,
                            int32_t width, float *scaled_input, float *input_scale,
                            float *mean_visible, float *mean_infrared);

/* No counterpart in the reference.  fx_producer_rows plus the stage table
 * (fx_stage_table with auxiliary_factor_b 1) for a frame already in device
 * memory, for callers that cannot allocate device memory when they need it
 * (a service whose HBM is claimed by its own pool; acquisition loops that
 * cannot afford the device-wide synchronization of a cudaFree).  The call
 * makes no device allocation: its scratch is a fixed 24 MiB device array per
 * device (frames up to a full 5782x3946 scan); larger frames return
 * FX_ERR_INVALID_ARGUMENT with the sizes in fx_last_error.  d_rows receives
 * 4*height floats (scaled_input, input_scale, mean_visible, mean_infrared,
 * one row after another), d_stages height+6 records.  Work is enqueued on
 * `stream` (a cudaStream_t, NULL for the legacy default stream) and the call
 * returns after it finishes.  The scratch is shared by all calls on one
 * device, so calls are serialized; the first call on a device reserves the
 * array (under the CUDA runtime's default lazy module loading; with
 * CUDA_MODULE_LOADING=EAGER every context reserves it at creation) and
 * should come before any stream capture.  FX_ERR_OUT_OF_MEMORY when the
 * device has no room left for the array.  The call holds the context's lock
 * and leaves the caller's current device as it found it. */
FX_API int fx_producer_rows_static(fx_context *ctx, const uint16_t *d_main_rgbi, int32_t height,
                                   int32_t width, float *d_rows, fx_stage *d_stages, void *stream);

/* producer_parameters.py:498-541 with stage_parameters.py:93-197: the stage
 * table (H+6 entries) built from per-row producer fields; host computation. */
FX_API int fx_stage_table(int32_t height, const float *scaled_input, const float *input_scale,
                          const float *mean_visible, const float *mean_infrared,
                          float auxiliary_factor_b, fx_stage *stages);

/* The whole main-scan pass for one frame, synchronous, host buffers:
 * streaming.py:365-552 (run_streaming_replay) / cuda_backend/engine.py:183
 * (run_streaming_replay_cuda), including the hidden startup replay, the
 * sequential dither writer, emit, counters and diagnostics. */
FX_API int fx_process(fx_context *ctx, const fx_frame *frame, fx_counters *counters);

/* Same pass on device-resident buffers, enqueued on `stream` (a
 * cudaStream_t, or NULL for the context stream).  d_rgbi, d_rgb_out,
 * d_score_out and d_changed_out are device pointers.  When `counters` is
 * non-NULL the call waits for completion and fills it; otherwise it returns
 * after enqueueing and fx_sync_counters fetches them later. */
FX_API int fx_process_device(fx_context *ctx, const uint16_t *d_rgbi, int32_t height,
                             int32_t width, const fx_params *params, const fx_stage *stages,
                             uint32_t rng_state, uint16_t *d_rgb_out, float *d_score_out,
                             uint8_t *d_changed_out, void *stream, fx_counters *counters);
FX_API int fx_sync_counters(fx_context *ctx, fx_counters *counters);

/* Asynchronous requests for batching and serving (no reference counterpart:
 * the reference processes one job per call).  Up to `slots` frames run
 * concurrently, each on its own stream with its own device buffers. */
FX_API int fx_set_slots(fx_context *ctx, int32_t slots);
/* 1 (default): the speculative parallel walk; 0: one warp walks the whole
 * chain (leaves the rest of the GPU to other frames' kernels). */
FX_API int fx_set_parallel_walk(fx_context *ctx, int enable);
/* Segments of 4096 RNG-dependent channels walked speculatively per wave
 * (0, the default: three per SM).  Fewer segments per wave mean narrower
 * candidate windows (less total work, for throughput when several frames
 * are in flight) and more waves (longer latency for one frame). */
FX_API int fx_set_walk_wave(fx_context *ctx, int32_t segments);
/* 1 (default): the latency-bound kernels of a pass (the producer's scan, the
 * writer's prefix, interval and jump kernels, the walk) are launched at the
 * device's greatest execution priority, so that with several frames in
 * flight their blocks are dispatched ahead of other frames' stencil and
 * emit blocks; 0: every launch at the default priority.  No effect on
 * results, nor on a single frame (no reference counterpart). */
FX_API int fx_set_launch_priority(fx_context *ctx, int enable);
/* SHA-256 of the RGB16 output of fx_process, little-endian bytes in
 * row-major order (the replay result's output_sha256, streaming.py:533-536).
 * When enabled, fx_process hashes each staged chunk of the output as soon as
 * its device-to-host copy lands, while the other chunks are still copied,
 * instead of leaving a second pass over the output to the caller.
 * fx_output_digest returns the digest of the last successful fx_process. */
FX_API int fx_set_output_digest(fx_context *ctx, int enable);
FX_API int fx_output_digest(fx_context *ctx, uint8_t *digest32);
/* Size every slot's device buffers for frames up to max_height x max_width
 * now, so that later frames within both bounds never reallocate (a
 * reallocation frees device memory, which waits for the whole device and
 * stalls the frames in flight).  No reference counterpart; call it after
 * fx_set_slots and before submitting.  FX_ERR_OUT_OF_MEMORY when the device
 * cannot hold them. */
FX_API int fx_reserve_frames(fx_context *ctx, int32_t max_height, int32_t max_width);
/* Submit a host-buffer frame.  A frame with rgb_out NULL keeps its results
 * (RGB16 output, score plane, changed mask) staged in pinned memory until
 * fx_fetch; otherwise fx_wait copies them into the frame's own buffers.
 * FX_PENDING when every slot is busy. */
FX_API int fx_submit(fx_context *ctx, const fx_frame *frame, int64_t *ticket);
/* Free the device buffers of every slot without a request in flight (no
 * reference counterpart).  A slot's buffers are otherwise kept and reused by
 * later frames they hold; a frame larger than every idle slot's buffers
 * grows the largest of them.  Both free device memory, which waits for the
 * whole device, so a request loop calls this only when nothing is in flight.
 * *released_bytes (may be NULL) receives the bytes freed. */
FX_API int fx_release_idle_slots(fx_context *ctx, int64_t *released_bytes);
/* fx_reserve_frames for the first `count` slots only (creating them as
 * needed), no reference counterpart: a request loop sizes a few slots for
 * its largest frame before its clock starts and lets memory decide how many
 * more it adds. */
FX_API int fx_reserve_slots(fx_context *ctx, int32_t count, int32_t max_height,
                            int32_t max_width);
/* fx_submit for a frame already in device memory: the pass is enqueued on
 * a free slot's stream and writes d_rgb_out / d_score_out / d_changed_out
 * (device pointers, NULL for the optional planes) directly.  The caller
 * keeps every buffer valid until fx_wait returns for the ticket.
 * FX_PENDING when every slot is busy. */
FX_API int fx_submit_device(fx_context *ctx, const uint16_t *d_rgbi, int32_t height,
                            int32_t width, const fx_params *params, const fx_stage *stages,
                            uint32_t rng_state, uint16_t *d_rgb_out, float *d_score_out,
                            uint8_t *d_changed_out, int64_t *ticket);
FX_API int fx_poll(fx_context *ctx, int64_t ticket);
FX_API int fx_wait(fx_context *ctx, int64_t ticket, int64_t timeout_ns, fx_counters *counters);
/* Cooperative cancellation of a request in flight, the device-side form of
 * the `cancelled` callback the reference polls between phases
 * (engine.py:103-106, checked by tests/test_engine.py:46-73).  Sets the
 * request's cancel word; the pass reads it at its next stage boundary
 * (after the producer, the analysis, the chain scan and the walk) and every
 * later kernel returns at once, so a device output buffer is left untouched
 * unless the last boundary had already passed.  fx_wait / fx_fetch then
 * return FX_ERR_CANCELLED (or FX_OK when the pass had already finished) and
 * release the slot; host buffers are written only on FX_OK. */
FX_API int fx_cancel(fx_context *ctx, int64_t ticket);
/* fx_wait for an fx_submit ticket that delivers the results into the
 * buffers given here, any of which may be NULL: the RGB16 output, the
 * counters, the score plane, the at-floor mask (score == the profile's
 * score floor, engine.py:175-199) and the changed mask.  The planes must
 * have been staged (a frame submitted with rgb_out NULL stages all of
 * them); FX_ERR_INVALID_ARGUMENT otherwise, or for a device-buffer ticket. */
FX_API int fx_fetch(fx_context *ctx, int64_t ticket, int64_t timeout_ns, uint16_t *rgb_out,
                    fx_counters *counters, float *score_out, uint8_t *at_floor_out,
                    uint8_t *changed_out);

/* Test knobs, no reference counterpart.  Neither changes a result, only
 * which code path produces it; both exist so the tests can drive the rare
 * paths of the writer.
 * fx_set_walk_window: half-width of the speculative walk's candidate
 * windows in standard deviations of the predicted count (default 4.5, plus
 * 16 candidates).  Narrow windows make entry counts fall outside them, so
 * the affected segments are walked by the exact serial fallback
 * (fx_counters.walk_fallbacks counts them).
 * fx_set_list_capacity: entries of the RNG-dependent channel list each pass
 * reserves (0, the default: half the frame's chain sites).  A frame with
 * more such channels reruns with room for all of them. */
/* Height of the analysis stencil's tiles, no reference counterpart: 8 rows
 * (four resident blocks per SM, the default; 0 selects it) or 16 rows (two
 * blocks per SM, less halo work per pixel).  Both compute the same values;
 * the batching autotuner picks one per device and frame shape. */
FX_API int fx_set_stencil_tile(fx_context *ctx, int32_t rows);
FX_API int fx_set_walk_window(fx_context *ctx, double sigmas);
FX_API int fx_set_list_capacity(fx_context *ctx, int64_t channels);

/* Device time per pipeline stage, from CUDA events recorded on the frame's
 * stream between kernel groups (measurement only; no reference
 * counterpart).  Stages: 0 producer, 1 auxiliary + history planes,
 * 2 stencil, 3 hidden startup, 4 chain scan + copy intervals + jumps,
 * 5 serial walk, 6 apply + emit + counters.  fx_profile_read waits for the
 * context stream, adds the elapsed times of every profiled pass since the
 * last reset into ms[FX_PROFILE_STAGES] and reports how many passes were
 * profiled. */
#define FX_PROFILE_STAGES 7
FX_API int fx_profile_enable(fx_context *ctx, int enable);
FX_API int fx_profile_read(fx_context *ctx, double *ms, int64_t *passes, int reset);

/* Free / total device memory, for admission control. */
FX_API int fx_mem_info(fx_context *ctx, size_t *free_bytes, size_t *total_bytes);

/* Device bytes one frame of the given size needs (admission estimate), with
 * the default RNG-dependent list of half the sites. */
FX_API int64_t fx_frame_bytes(int32_t height, int32_t width);
/* The same on this context: after a frame's list overflowed (heavy damage),
 * later passes list up to the longest list per site seen so far, and their
 * buffers grow by that much (no reference counterpart). */
FX_API int fx_pass_bytes(fx_context *ctx, int32_t height, int32_t width, int64_t *bytes);

/* ------------------------------------------------------------------------
 * At-floor routing census (hybrid routing.py:447-682, route_at_floor_mask).
 * Context-free device primitives; the per-component tables, reasons and
 * budget are host logic (fauxice_b200.routing).  Every pointer named d_* is
 * device memory; `stream` is a cudaStream_t or NULL.  Each call waits for
 * its own work before returning.
 * ---------------------------------------------------------------------- */

/* 8-connected components of a uint8 mask, ids 1..K in raster order of each
 * component's first pixel, 0 for background (ndimage.label with a 3x3
 * structure, routing.py:467-473 and :327-333).  d_forest int32[h*w] is
 * scratch distinct from d_labels, d_block_scratch holds ceil(h*w/256) + 1
 * uint32, d_err one uint32.  h*w < 2^31. */
FX_API int fx_label8(const uint8_t *d_mask, int32_t h, int32_t w, int32_t *d_labels,
                     int32_t *d_forest, uint32_t *d_block_scratch, uint32_t *d_err,
                     int64_t *count, void *stream);
/* Chessboard distance of every set pixel to the nearest in-frame unset pixel,
 * 0 on unset pixels (distance_transform_cdt metric "chessboard",
 * routing.py:277); the mask must hold at least one unset pixel.  d_work is
 * int32[h*w] scratch, d_flag one uint32. */
FX_API int fx_chessboard_distance(const uint8_t *d_mask, int32_t h, int32_t w, int32_t *d_dist,
                                  int32_t *d_work, uint32_t *d_flag, void *stream);
/* Per label 1..k (entry l-1): pixel count, half-open box [y0, x0, y1, x1)
 * and, when d_plane is non-NULL, the maximum of d_plane over the label
 * (bincount, find_objects and ndimage.maximum, routing.py:474-488, :278). */
FX_API int fx_label_stats(const int32_t *d_labels, const int32_t *d_plane, int32_t h, int32_t w,
                          int64_t k, unsigned long long *d_area, int32_t *d_box, int32_t *d_vmax,
                          void *stream);
/* Square (Chebyshev) dilation by `radius`, zero outside the frame, the
 * radius clipped per axis to the frame (routing.py:304-336).  d_work is
 * uint8[h*w] scratch. */
FX_API int fx_dilate_square(const uint8_t *d_in, int32_t h, int32_t w, int32_t radius,
                            uint8_t *d_work, uint8_t *d_out, void *stream);
/* Distinct (a, b) pairs of two label planes over pixels where both are
 * positive, written as int32 pairs to d_pairs with possible repeats (the
 * caller sorts them unique, as routing.py:552-556 does).  FX_ERR_OUT_OF_MEMORY
 * with *count set when more than `capacity` pairs were found. */
FX_API int fx_label_pairs(const int32_t *d_a, const int32_t *d_b, int32_t h, int32_t w,
                          int64_t capacity, int32_t *d_pairs, unsigned long long *d_count,
                          int64_t *count, void *stream);
/* out[i] = map[labels[i]] as int32 (d_out_i32) and/or as map != 0 (d_out_u8),
 * for a map of k + 1 entries; labels outside 0..k give 0 (the lookups
 * routed_lookup[...] and old_to_new[...], routing.py:504, :434). */
FX_API int fx_map_labels(const int32_t *d_labels, int64_t n, const int32_t *d_map, int64_t k,
                         int32_t *d_out_i32, uint8_t *d_out_u8, void *stream);
/* Clear the mask where labels == id; *cleared = how many of those pixels were
 * set (the perimeter rule, routing.py:517-522).  d_scratch one uint64. */
FX_API int fx_clear_label(uint8_t *d_mask, const int32_t *d_labels, int64_t n, int32_t id,
                          unsigned long long *d_scratch, int64_t *cleared, void *stream);
/* d_counts[key] = pixels with 0 < key <= k and cond > 0, for keys 0..k (the
 * overlap bincounts, routing.py:533-546). */
FX_API int fx_count_where(const int32_t *d_key, const int32_t *d_cond, int64_t n, int64_t k,
                          unsigned long long *d_counts, void *stream);
/* tile = (labels[y0+ty][x0+tx] == id) over a th x tw window, and the write
 * back of a labelled tile offset by `base` (the oversized-region tiling,
 * routing.py:376-410). */
FX_API int fx_tile_extract(const int32_t *d_labels, int32_t h, int32_t w, int32_t y0, int32_t x0,
                           int32_t th, int32_t tw, int32_t id, uint8_t *d_tile, void *stream);
FX_API int fx_tile_scatter(const int32_t *d_tile_labels, int32_t h, int32_t w, int32_t y0,
                           int32_t x0, int32_t th, int32_t tw, int32_t base, int32_t *d_plane,
                           void *stream);

/* Canonical JSON text of the census's two region lists (host code): the
 * "provisional_regions" and "final_regions" arrays of routing_json_document
 * (routing.py:736-777) as serialize_routing_json writes them (sorted keys, no
 * whitespace, routing.py:782-793).  Tables are flat, ids run 1..count in
 * order; box holds [y0, x0, y1, x1) per region; each id list is an offset
 * range (count + 1 offsets) into its values.  reason and disposition are
 * codes: reason 0 not_routed, 1 chessboard_radius, 2 area,
 * 3 area+chessboard_radius; disposition 0 routed, 1 absorbed, 2 pristine,
 * 3 perimeter_excluded.  Returns the bytes written, or -1 for a bad argument
 * or too small a buffer. */
FX_API int64_t fx_census_provisional_json(int64_t k, const int64_t *box, const int64_t *area,
                                          const int64_t *radius, const int32_t *reason,
                                          const int32_t *disposition, const int64_t *absorbed,
                                          const int64_t *final_offsets, const int64_t *final_ids,
                                          char *out, int64_t capacity);
FX_API int64_t fx_census_final_json(int64_t count, const int64_t *box, const int64_t *area,
                                    const int64_t *direct_offsets, const int64_t *direct_ids,
                                    const int64_t *absorbed_offsets, const int64_t *absorbed_ids,
                                    const int64_t *non_floor, char *out, int64_t capacity);

#ifdef __cplusplus
}
#endif

#endif /* FAUXICE_B200_H */
