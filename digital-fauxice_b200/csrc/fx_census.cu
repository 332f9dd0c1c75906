// fx_census.cu -- canonical JSON text of the routing census's region lists.
//
// The census document (hybrid routing.py:685-779) is serialized with sorted
// keys, no whitespace and no ASCII escaping (routing.py:782-793).  Nearly all
// of its bytes are the two region lists: one object per provisional region
// (tens of thousands on a real frame) and one per final region.  These two
// writers format those lists from flat tables in one pass, byte for byte as
// the canonical serializer does; the host splices them into the small rest
// of the document.  Host code only.
#include <cstring>

#include "fx_internal.cuh"

namespace {

struct Writer {
    char *p;
    char *end;
    bool ok = true;

    void raw(const char *s, size_t n) {
        if (!ok || (size_t)(end - p) < n) {
            ok = false;
            return;
        }
        std::memcpy(p, s, n);
        p += n;
    }
    template <size_t N>
    void lit(const char (&s)[N]) { raw(s, N - 1); }
    void str(const char *s) { raw(s, std::strlen(s)); }
    void num(int64_t v) {
        char buf[24];
        int n = 0;
        uint64_t u = v < 0 ? (uint64_t)0 - (uint64_t)v : (uint64_t)v;
        do {
            buf[n++] = (char)('0' + u % 10);
            u /= 10;
        } while (u);
        if (v < 0) buf[n++] = '-';
        if (!ok || end - p < n) {
            ok = false;
            return;
        }
        while (n) *p++ = buf[--n];
    }
    void list(const int64_t *v, int64_t count) {
        lit("[");
        for (int64_t i = 0; i < count; ++i) {
            if (i) lit(",");
            num(v[i]);
        }
        lit("]");
    }
    void box(const int64_t *b) { list(b, 4); }
};

// routing.py:35-41 and :44-50, indexed by the codes the host passes
const char *const kReason[4] = {"not_routed", "chessboard_radius", "area",
                                "area+chessboard_radius"};
const char *const kDisposition[4] = {"routed", "absorbed", "pristine", "perimeter_excluded"};

}  // namespace

// provisional_regions: region i (id i + 1) has box[4i..4i+3] = [y0, x0, y1,
// x1), final ids final_ids[final_offsets[i] .. final_offsets[i + 1]).
FX_API int64_t fx_census_provisional_json(int64_t k, const int64_t *box, const int64_t *area,
                                          const int64_t *radius, const int32_t *reason,
                                          const int32_t *disposition, const int64_t *absorbed,
                                          const int64_t *final_offsets, const int64_t *final_ids,
                                          char *out, int64_t capacity) {
    if (k < 0 || !out || capacity < 2 ||
        (k > 0 && (!box || !area || !radius || !reason || !disposition || !absorbed ||
                   !final_offsets || !final_ids)))
        return -1;
    Writer w{out, out + capacity};
    w.lit("[");
    for (int64_t i = 0; i < k && w.ok; ++i) {
        if ((unsigned)reason[i] > 3u || (unsigned)disposition[i] > 3u) return -1;
        if (i) w.lit(",");
        w.lit("{\"absorbed_pixel_count\":");
        w.num(absorbed[i]);
        w.lit(",\"area\":");
        w.num(area[i]);
        w.lit(",\"bbox_yxyx_half_open\":");
        w.box(box + 4 * i);
        w.lit(",\"disposition\":\"");
        w.str(kDisposition[disposition[i]]);
        w.lit("\",\"final_component_ids\":");
        w.list(final_ids + final_offsets[i], final_offsets[i + 1] - final_offsets[i]);
        w.lit(",\"id\":");
        w.num(i + 1);
        w.lit(",\"max_chessboard_radius\":");
        w.num(radius[i]);
        w.lit(",\"routed_reason\":\"");
        w.str(kReason[reason[i]]);
        w.lit("\"}");
    }
    w.lit("]");
    return w.ok ? (int64_t)(w.p - out) : -1;
}

// final_regions: region f (id f + 1) with its direct and absorbed provisional
// ids as offset ranges, like the final ids above.
FX_API int64_t fx_census_final_json(int64_t count, const int64_t *box, const int64_t *area,
                                    const int64_t *direct_offsets, const int64_t *direct_ids,
                                    const int64_t *absorbed_offsets, const int64_t *absorbed_ids,
                                    const int64_t *non_floor, char *out, int64_t capacity) {
    if (count < 0 || !out || capacity < 2 ||
        (count > 0 && (!box || !area || !direct_offsets || !direct_ids || !absorbed_offsets ||
                       !absorbed_ids || !non_floor)))
        return -1;
    Writer w{out, out + capacity};
    w.lit("[");
    for (int64_t f = 0; f < count && w.ok; ++f) {
        if (f) w.lit(",");
        w.lit("{\"absorbed_region_ids\":");
        w.list(absorbed_ids + absorbed_offsets[f], absorbed_offsets[f + 1] - absorbed_offsets[f]);
        w.lit(",\"area\":");
        w.num(area[f]);
        w.lit(",\"bbox_yxyx_half_open\":");
        w.box(box + 4 * f);
        w.lit(",\"direct_region_ids\":");
        w.list(direct_ids + direct_offsets[f], direct_offsets[f + 1] - direct_offsets[f]);
        w.lit(",\"id\":");
        w.num(f + 1);
        w.lit(",\"non_floor_synthesis_pixels\":");
        w.num(non_floor[f]);
        w.lit("}");
    }
    w.lit("]");
    return w.ok ? (int64_t)(w.p - out) : -1;
}
