// fx_route.cu -- device primitives of the at-floor routing census.
//
// The routing step downstream of the diagnostics (hybrid routing.py:447-682,
// route_at_floor_mask) measures the 8-connected components of the at-floor
// mask, routes the large ones, dilates them by a square margin and labels
// the result again.  Every per-pixel step runs here; the per-component
// bookkeeping (reasons, budget, overlap tables, the JSON census) is host
// logic in fauxice_b200/routing.py.
//
//   k_ccl_*        8-connected components by lock-free union-find.  A root
//                  is only ever linked under a smaller root, so each root is
//                  its component's smallest raster index and the final ids
//                  (1..K by root order) follow scipy.ndimage.label's
//                  raster order of first pixels.
//   k_dist_*       chessboard distance to the nearest in-frame background
//                  pixel (distance_transform_cdt, metric "chessboard"), by
//                  Jacobi relaxation in shared-memory tiles until no change.
//   k_stats        per-label area, bounding box and maximum of a plane.
//   k_dilate_*     square (Chebyshev) dilation, separable: nearest set
//                  pixel along each column, then along each row, within a
//                  radius clipped to the frame.
//   k_pairs        (label, label) pairs of two label planes, emitted only
//                  where a pixel starts a new pair locally (the host removes
//                  the remaining duplicates).
#include "fx_internal.cuh"

namespace fx {

constexpr int kRouteThreads = 256;
constexpr uint32_t kFindLimit = 1u << 26;  // bounds every pointer walk

// Root of x.  Path halving (each visited slot is pointed at its
// grandparent) only ever stores an ancestor, so concurrent finds and links
// stay consistent.
__device__ __forceinline__ int32_t find_root(int32_t *parent, int32_t x, uint32_t *err) {
    uint32_t steps = 0;
    int32_t p = parent[x];
    while (p != x) {
        const int32_t gp = parent[p];
        if (gp != p) parent[x] = gp;
        x = p;
        p = parent[x];
        if (++steps > kFindLimit) {
            raise_error(err, FX_ERR_INTERNAL);
            break;
        }
    }
    return x;
}

__global__ void k_ccl_init(const uint8_t *__restrict__ mask, int64_t n, int32_t *parent) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        parent[i] = mask[i] ? (int32_t)i : -1;
}

// Link the components of pixel a and pixel b: the larger root goes under the
// smaller one.  A failed link (the root moved meanwhile) retries from the
// new roots; each retry strictly lowers the larger root, so the loop ends.
__device__ void ccl_union(int32_t *parent, int32_t a, int32_t b, uint32_t *err) {
    for (uint32_t tries = 0; tries < kFindLimit; ++tries) {
        a = find_root(parent, a, err);
        b = find_root(parent, b, err);
        if (a == b) return;
        if (a < b) {
            const int32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(&parent[a], a, b) == a) return;
    }
    raise_error(err, FX_ERR_INTERNAL);
}

__global__ void k_ccl_union(const uint8_t *__restrict__ mask, int h, int w, int32_t *parent,
                            uint32_t *err) {
    const int64_t n = (int64_t)h * w;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (!mask[i]) continue;
        const int y = (int)(i / w), x = (int)(i % w);
        if (x > 0 && mask[i - 1]) ccl_union(parent, (int32_t)i, (int32_t)(i - 1), err);
        if (y > 0) {
            const int64_t u = i - w;
            if (x > 0 && mask[u - 1]) ccl_union(parent, (int32_t)i, (int32_t)(u - 1), err);
            if (mask[u]) ccl_union(parent, (int32_t)i, (int32_t)u, err);
            if (x + 1 < w && mask[u + 1]) ccl_union(parent, (int32_t)i, (int32_t)(u + 1), err);
        }
    }
}

// After every link: point each foreground pixel straight at its root.  The
// walk only reads (every slot it meets holds an ancestor, the old one or the
// root), and each slot is written only by its own thread, so every slot
// ends up holding its root.
__global__ void k_ccl_flatten(int32_t *parent, int64_t n, uint32_t *err) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int32_t x = parent[i];
        if (x < 0) continue;
        uint32_t steps = 0;
        int32_t p = parent[x];
        while (p != x) {
            x = p;
            p = parent[x];
            if (++steps > kFindLimit) {
                raise_error(err, FX_ERR_INTERNAL);
                break;
            }
        }
        parent[i] = x;
    }
}

// Roots per block of pixels (a root is its own parent after flattening).
__global__ void k_ccl_count_roots(const int32_t *parent, int64_t n, uint32_t *block_roots) {
    __shared__ uint32_t count;
    if (threadIdx.x == 0) count = 0;
    __syncthreads();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool root = i < n && parent[i] == (int32_t)i;
    const uint32_t warp_roots = __popc(__ballot_sync(0xFFFFFFFFu, root));
    if ((threadIdx.x & 31) == 0 && warp_roots) atomicAdd(&count, warp_roots);
    __syncthreads();
    if (threadIdx.x == 0) block_roots[blockIdx.x] = count;
}

// Exclusive scan of the per-block root counts (one block); total at [n].
__global__ void k_ccl_scan(uint32_t *block_roots, int64_t nblocks) {
    __shared__ uint32_t warp_sums[32];
    uint32_t carry = 0;
    for (int64_t base = 0; base < nblocks; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const uint32_t v = i < nblocks ? block_roots[i] : 0u;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0u;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
                if (lane >= o) s += y;
            }
            warp_sums[lane] = s;
        }
        __syncthreads();
        const uint32_t prefix = (warp ? warp_sums[warp - 1] : 0u) + x - v;
        if (i < nblocks) block_roots[i] = carry + prefix;
        carry += warp_sums[(blockDim.x >> 5) - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) block_roots[nblocks] = carry;
}

// Ids 1..K to the roots in raster order (pixel order inside a block by a
// block scan), stored in the root's own slot as -(id) - 1.  Each thread
// reads and writes only its own slot.
__global__ void k_ccl_number(int32_t *parent, int64_t n, const uint32_t *block_base) {
    __shared__ uint32_t warp_sums[kRouteThreads / 32];
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool root = i < n && parent[i] == (int32_t)i;
    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, root);
    if (lane == 0) warp_sums[warp] = __popc(bal);
    __syncthreads();
    uint32_t before = 0;
    for (int k = 0; k < warp; ++k) before += warp_sums[k];
    before += __popc(bal & ((1u << lane) - 1u));
    if (root) parent[i] = -(int32_t)(block_base[blockIdx.x] + before + 1) - 1;
}

// Labels: background slots hold -1, numbered roots -(id) - 1, every other
// foreground slot its root's index (flattened).
__global__ void k_ccl_labels(const int32_t *parent, int64_t n, int32_t *labels) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int32_t p = parent[i];
        if (p == -1) {
            labels[i] = 0;
            continue;
        }
        if (p >= 0) p = parent[p];
        labels[i] = -p - 1;
    }
}

// ---------------------------------------------------------------------------
// Chessboard distance: dist = 0 on background; foreground relaxes to
// min(dist, min over the 8 neighbours + 1).  A block relaxes a 32x32 tile
// with an 8-pixel halo in shared memory for 8 steps (the tile's centre is
// exact for those steps), and reports whether anything changed.
// ---------------------------------------------------------------------------

constexpr int kDistTile = 32, kDistHalo = 8, kDistSide = kDistTile + 2 * kDistHalo;
constexpr int32_t kDistInf = 0x3FFFFFFF;

__global__ void k_dist_init(const uint8_t *__restrict__ mask, int64_t n, int32_t *dist) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        dist[i] = mask[i] ? kDistInf : 0;
}

__global__ void __launch_bounds__(kRouteThreads)
    k_dist_relax(const int32_t *__restrict__ in, int32_t *__restrict__ out, int h, int w,
                 uint32_t *changed) {
    __shared__ int32_t t[2][kDistSide][kDistSide];
    const int y0 = blockIdx.y * kDistTile - kDistHalo, x0 = blockIdx.x * kDistTile - kDistHalo;
    for (int k = threadIdx.x; k < kDistSide * kDistSide; k += blockDim.x) {
        const int r = k / kDistSide, c = k % kDistSide;
        const int y = y0 + r, x = x0 + c;
        // outside the frame: no background and no path (never lowers a value)
        t[0][r][c] = (y >= 0 && y < h && x >= 0 && x < w) ? in[(int64_t)y * w + x] : kDistInf;
    }
    __syncthreads();
    int b = 0;
    for (int step = 0; step < kDistHalo; ++step) {
        for (int k = threadIdx.x; k < kDistSide * kDistSide; k += blockDim.x) {
            const int r = k / kDistSide, c = k % kDistSide;
            int32_t v = t[b][r][c];
            if (v > 0 && r > 0 && r < kDistSide - 1 && c > 0 && c < kDistSide - 1) {
                int32_t m = kDistInf;
#pragma unroll
                for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
                    for (int dx = -1; dx <= 1; ++dx) m = min(m, t[b][r + dy][c + dx]);
                if (m < kDistInf && m + 1 < v) v = m + 1;
            }
            t[b ^ 1][r][c] = v;
        }
        __syncthreads();
        b ^= 1;
    }
    bool any = false;
    for (int k = threadIdx.x; k < kDistTile * kDistTile; k += blockDim.x) {
        const int r = k / kDistTile + kDistHalo, c = k % kDistTile + kDistHalo;
        const int y = y0 + r, x = x0 + c;
        if (y < h && x < w) {
            const int32_t v = t[b][r][c];
            const int64_t o = (int64_t)y * w + x;
            any |= v != in[o];
            out[o] = v;
        }
    }
    if (__syncthreads_or(any) && threadIdx.x == 0) atomicOr(changed, 1u);
}

// ---------------------------------------------------------------------------
// Per-label statistics: area, bounding box [y0, x0, y1, x1) and maximum of
// an optional plane.
// ---------------------------------------------------------------------------

__global__ void k_stats_init(int64_t k, unsigned long long *area, int32_t *box, int32_t *vmax) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k;
         i += (int64_t)gridDim.x * blockDim.x) {
        area[i] = 0;
        box[4 * i] = box[4 * i + 1] = 0x7FFFFFFF;
        box[4 * i + 2] = box[4 * i + 3] = -1;
        if (vmax) vmax[i] = -1;
    }
}

__global__ void k_stats(const int32_t *__restrict__ labels, const int32_t *__restrict__ plane,
                        int h, int w, int64_t k_max, unsigned long long *area, int32_t *box,
                        int32_t *vmax) {
    const int64_t n = (int64_t)h * w;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t l = labels[i];
        if (l <= 0 || l > k_max) continue;
        const int32_t k = l - 1;
        const int y = (int)(i / w), x = (int)(i % w);
        atomicAdd(&area[k], 1ull);
        atomicMin(&box[4 * k], y);
        atomicMin(&box[4 * k + 1], x);
        atomicMax(&box[4 * k + 2], y + 1);
        atomicMax(&box[4 * k + 3], x + 1);
        if (vmax) atomicMax(&vmax[k], plane[i]);
    }
}

// ---------------------------------------------------------------------------
// Square dilation, separable: a pixel is set when a set pixel lies within
// `r` along the column (pass 1), then within `r` along the row (pass 2).
// Each thread sweeps one column or one row twice (nearest set pixel before
// and after), so any radius costs the same.
// ---------------------------------------------------------------------------

__global__ void k_dilate_cols(const uint8_t *__restrict__ in, int h, int w, int r,
                              uint8_t *__restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= w) return;
    int last = -0x3FFFFFFF;  // last set row at or above y
    for (int y = 0; y < h; ++y) {
        if (in[(int64_t)y * w + x]) last = y;
        out[(int64_t)y * w + x] = (y - last) <= r;
    }
    int next = 0x3FFFFFFF;  // next set row at or below y
    for (int y = h - 1; y >= 0; --y) {
        if (in[(int64_t)y * w + x]) next = y;
        if (next - y <= r) out[(int64_t)y * w + x] = 1;
    }
}

__global__ void k_dilate_rows(const uint8_t *__restrict__ in, int h, int w, int r,
                              uint8_t *__restrict__ out) {
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= h) return;
    const uint8_t *row = in + (int64_t)y * w;
    uint8_t *dst = out + (int64_t)y * w;
    int last = -0x3FFFFFFF;
    for (int x = 0; x < w; ++x) {
        if (row[x]) last = x;
        dst[x] = (x - last) <= r;
    }
    int next = 0x3FFFFFFF;
    for (int x = w - 1; x >= 0; --x) {
        if (row[x]) next = x;
        if (next - x <= r) dst[x] = 1;
    }
}

// ---------------------------------------------------------------------------
// (a, b) label pairs where both are positive and the pixel has no earlier
// 8-neighbour (W, NW, N, NE) carrying the same pair; every distinct pair has
// at least one such pixel.
// ---------------------------------------------------------------------------

__global__ void k_pairs(const int32_t *__restrict__ la, const int32_t *__restrict__ lb, int h,
                        int w, int64_t capacity, int2 *pairs, unsigned long long *count) {
    const int64_t n = (int64_t)h * w;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t a = la[i], b = lb[i];
        if (a <= 0 || b <= 0) continue;
        const int y = (int)(i / w), x = (int)(i % w);
        auto same = [&](int64_t j) { return la[j] == a && lb[j] == b; };
        bool seen = x > 0 && same(i - 1);
        if (!seen && y > 0) {
            const int64_t u = i - w;
            seen = (x > 0 && same(u - 1)) || same(u) || (x + 1 < w && same(u + 1));
        }
        if (seen) continue;
        const unsigned long long at = atomicAdd(count, 1ull);
        if ((int64_t)at < capacity) pairs[at] = make_int2(a, b);
    }
}

static unsigned grid_for(int64_t n) {
    const int64_t b = (n + kRouteThreads - 1) / kRouteThreads;
    return (unsigned)(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

}  // namespace fx

using namespace fx;

// Work buffers are the caller's (device): forest int32[n] (distinct from
// labels), block_scratch ceil(n / 256) + 1 uint32, err one uint32.
FX_API int fx_label8(const uint8_t *d_mask, int32_t h, int32_t w, int32_t *d_labels,
                     int32_t *d_forest, uint32_t *d_block_scratch, uint32_t *d_err,
                     int64_t *count, void *stream) {
    if (!d_mask || !d_labels || !d_forest || !d_block_scratch || !d_err || !count || h < 1 ||
        w < 1 || (int64_t)h * w >= ((int64_t)1 << 31))
        return FX_ERR_INVALID_ARGUMENT;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int64_t n = (int64_t)h * w;
    const int64_t nblocks = (n + kRouteThreads - 1) / kRouteThreads;
    if (cudaMemsetAsync(d_err, 0, sizeof(uint32_t), st) != cudaSuccess) return FX_ERR_CUDA;
    k_ccl_init<<<grid_for(n), kRouteThreads, 0, st>>>(d_mask, n, d_forest);
    k_ccl_union<<<grid_for(n), kRouteThreads, 0, st>>>(d_mask, h, w, d_forest, d_err);
    k_ccl_flatten<<<grid_for(n), kRouteThreads, 0, st>>>(d_forest, n, d_err);
    k_ccl_count_roots<<<(unsigned)nblocks, kRouteThreads, 0, st>>>(d_forest, n, d_block_scratch);
    k_ccl_scan<<<1, 1024, 0, st>>>(d_block_scratch, nblocks);
    k_ccl_number<<<(unsigned)nblocks, kRouteThreads, 0, st>>>(d_forest, n, d_block_scratch);
    k_ccl_labels<<<grid_for(n), kRouteThreads, 0, st>>>(d_forest, n, d_labels);
    uint32_t total = 0, err = 0;
    cudaMemcpyAsync(&total, d_block_scratch + nblocks, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&err, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return FX_ERR_CUDA;
    if (err) return FX_ERR_INTERNAL;
    *count = total;
    return FX_OK;
}

FX_API int fx_chessboard_distance(const uint8_t *d_mask, int32_t h, int32_t w, int32_t *d_dist,
                                  int32_t *d_work, uint32_t *d_flag, void *stream) {
    if (!d_mask || !d_dist || !d_work || !d_flag || h < 1 || w < 1) return FX_ERR_INVALID_ARGUMENT;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int64_t n = (int64_t)h * w;
    k_dist_init<<<grid_for(n), kRouteThreads, 0, st>>>(d_mask, n, d_dist);
    const dim3 grid((w + kDistTile - 1) / kDistTile, (h + kDistTile - 1) / kDistTile);
    int32_t *a = d_dist, *b = d_work;
    // every launch moves each front by up to kDistHalo pixels; the distance
    // of any pixel is below max(h, w), which bounds the launches
    const int64_t limit = (h > w ? h : w) / kDistHalo + 2;
    uint32_t changed = 1;
    for (int64_t it = 0; it < limit && changed; ++it) {
        changed = 0;
        if (cudaMemsetAsync(d_flag, 0, sizeof(uint32_t), st) != cudaSuccess) return FX_ERR_CUDA;
        k_dist_relax<<<grid, kRouteThreads, 0, st>>>(a, b, h, w, d_flag);
        cudaMemcpyAsync(&changed, d_flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return FX_ERR_CUDA;
        int32_t *t = a;
        a = b;
        b = t;
    }
    if (changed) return FX_ERR_INTERNAL;
    if (a != d_dist &&
        cudaMemcpyAsync(d_dist, a, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToDevice, st) !=
            cudaSuccess)
        return FX_ERR_CUDA;
    return cudaStreamSynchronize(st) == cudaSuccess ? FX_OK : FX_ERR_CUDA;
}

FX_API int fx_label_stats(const int32_t *d_labels, const int32_t *d_plane, int32_t h, int32_t w,
                          int64_t k, unsigned long long *d_area, int32_t *d_box, int32_t *d_vmax,
                          void *stream) {
    if (!d_labels || !d_area || !d_box || h < 1 || w < 1 || k < 0) return FX_ERR_INVALID_ARGUMENT;
    if (k == 0) return FX_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_stats_init<<<grid_for(k), kRouteThreads, 0, st>>>(k, d_area, d_box, d_plane ? d_vmax : nullptr);
    k_stats<<<grid_for((int64_t)h * w), kRouteThreads, 0, st>>>(
        d_labels, d_plane, h, w, k, d_area, d_box, d_plane ? d_vmax : nullptr);
    return cudaStreamSynchronize(st) == cudaSuccess ? FX_OK : FX_ERR_CUDA;
}

FX_API int fx_dilate_square(const uint8_t *d_in, int32_t h, int32_t w, int32_t radius,
                            uint8_t *d_work, uint8_t *d_out, void *stream) {
    if (!d_in || !d_work || !d_out || h < 1 || w < 1 || radius < 0) return FX_ERR_INVALID_ARGUMENT;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int rv = radius < h - 1 ? radius : h - 1, rh = radius < w - 1 ? radius : w - 1;
    k_dilate_cols<<<(w + 127) / 128, 128, 0, st>>>(d_in, h, w, rv, d_work);
    k_dilate_rows<<<(h + 127) / 128, 128, 0, st>>>(d_work, h, w, rh, d_out);
    return cudaStreamSynchronize(st) == cudaSuccess ? FX_OK : FX_ERR_CUDA;
}

FX_API int fx_label_pairs(const int32_t *d_a, const int32_t *d_b, int32_t h, int32_t w,
                          int64_t capacity, int32_t *d_pairs, unsigned long long *d_count,
                          int64_t *count, void *stream) {
    if (!d_a || !d_b || !d_pairs || !d_count || !count || h < 1 || w < 1)
        return FX_ERR_INVALID_ARGUMENT;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), st) != cudaSuccess)
        return FX_ERR_CUDA;
    k_pairs<<<grid_for((int64_t)h * w), kRouteThreads, 0, st>>>(
        d_a, d_b, h, w, capacity, reinterpret_cast<int2 *>(d_pairs), d_count);
    unsigned long long c = 0;
    cudaMemcpyAsync(&c, d_count, sizeof(c), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return FX_ERR_CUDA;
    *count = (int64_t)c;
    return (int64_t)c > capacity ? FX_ERR_OUT_OF_MEMORY : FX_OK;
}

// ---------------------------------------------------------------------------
// Label-plane helpers of the routing census
// ---------------------------------------------------------------------------

namespace fx {

__global__ void k_map_labels(const int32_t *__restrict__ labels, int64_t n,
                             const int32_t *__restrict__ map, int64_t k, int32_t *out_i32,
                             uint8_t *out_u8) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t l = labels[i];
        const int32_t v = (l >= 0 && l <= k) ? map[l] : 0;
        if (out_i32) out_i32[i] = v;
        if (out_u8) out_u8[i] = v != 0;
    }
}

__global__ void k_clear_label(uint8_t *mask, const int32_t *__restrict__ labels, int64_t n,
                              int32_t id, unsigned long long *cleared) {
    unsigned long long mine = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (labels[i] == id) {
            mine += mask[i] != 0;
            mask[i] = 0;
        }
    }
    if (mine) atomicAdd(cleared, mine);
}

__global__ void k_count_where(const int32_t *__restrict__ key, const int32_t *__restrict__ cond,
                              int64_t n, int64_t k, unsigned long long *counts) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t l = key[i];
        if (l > 0 && l <= k && cond[i] > 0) atomicAdd(&counts[l], 1ull);
    }
}

__global__ void k_tile_extract(const int32_t *__restrict__ labels, int w, int y0, int x0, int th,
                               int tw, int32_t id, uint8_t *tile) {
    const int64_t n = (int64_t)th * tw;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int ty = (int)(i / tw), tx = (int)(i % tw);
        tile[i] = labels[(int64_t)(y0 + ty) * w + (x0 + tx)] == id;
    }
}

__global__ void k_tile_scatter(const int32_t *__restrict__ tile_labels, int w, int y0, int x0,
                               int th, int tw, int32_t base, int32_t *plane) {
    const int64_t n = (int64_t)th * tw;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t l = tile_labels[i];
        if (l > 0) plane[(int64_t)(y0 + i / tw) * w + (x0 + i % tw)] = base + l;
    }
}

}  // namespace fx

// out[i] = map[labels[i]] (int32 and/or nonzero as uint8); map holds k + 1
// entries, labels outside 0..k map to 0.
FX_API int fx_map_labels(const int32_t *d_labels, int64_t n, const int32_t *d_map, int64_t k,
                         int32_t *d_out_i32, uint8_t *d_out_u8, void *stream) {
    if (!d_labels || !d_map || (!d_out_i32 && !d_out_u8) || n < 1 || k < 0)
        return FX_ERR_INVALID_ARGUMENT;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_map_labels<<<grid_for(n), kRouteThreads, 0, st>>>(d_labels, n, d_map, k, d_out_i32,
                                                       d_out_u8);
    return cudaStreamSynchronize(st) == cudaSuccess ? FX_OK : FX_ERR_CUDA;
}

// Clear mask where labels == id; *cleared = how many of those were set.
FX_API int fx_clear_label(uint8_t *d_mask, const int32_t *d_labels, int64_t n, int32_t id,
                          unsigned long long *d_scratch, int64_t *cleared, void *stream) {
    if (!d_mask || !d_labels || !d_scratch || !cleared || n < 1) return FX_ERR_INVALID_ARGUMENT;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(d_scratch, 0, sizeof(unsigned long long), st) != cudaSuccess)
        return FX_ERR_CUDA;
    k_clear_label<<<grid_for(n), kRouteThreads, 0, st>>>(d_mask, d_labels, n, id, d_scratch);
    unsigned long long c = 0;
    cudaMemcpyAsync(&c, d_scratch, sizeof(c), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return FX_ERR_CUDA;
    *cleared = (int64_t)c;
    return FX_OK;
}

// counts[key] += 1 over pixels where 0 < key <= k and cond > 0; counts holds
// k + 1 entries and is cleared first.
FX_API int fx_count_where(const int32_t *d_key, const int32_t *d_cond, int64_t n, int64_t k,
                          unsigned long long *d_counts, void *stream) {
    if (!d_key || !d_cond || !d_counts || n < 1 || k < 0) return FX_ERR_INVALID_ARGUMENT;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(d_counts, 0, (size_t)(k + 1) * sizeof(unsigned long long), st) !=
        cudaSuccess)
        return FX_ERR_CUDA;
    k_count_where<<<grid_for(n), kRouteThreads, 0, st>>>(d_key, d_cond, n, k, d_counts);
    return cudaStreamSynchronize(st) == cudaSuccess ? FX_OK : FX_ERR_CUDA;
}

// Tile of a label plane: tile = (labels[y0 + ty][x0 + tx] == id), th x tw.
FX_API int fx_tile_extract(const int32_t *d_labels, int32_t h, int32_t w, int32_t y0, int32_t x0,
                           int32_t th, int32_t tw, int32_t id, uint8_t *d_tile, void *stream) {
    if (!d_labels || !d_tile || th < 1 || tw < 1 || y0 < 0 || x0 < 0 || y0 + th > h ||
        x0 + tw > w)
        return FX_ERR_INVALID_ARGUMENT;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_tile_extract<<<grid_for((int64_t)th * tw), kRouteThreads, 0, st>>>(d_labels, w, y0, x0, th,
                                                                        tw, id, d_tile);
    return cudaStreamSynchronize(st) == cudaSuccess ? FX_OK : FX_ERR_CUDA;
}

// plane[y0 + ty][x0 + tx] = base + tile_labels[ty][tx] where tile_labels > 0.
FX_API int fx_tile_scatter(const int32_t *d_tile_labels, int32_t h, int32_t w, int32_t y0,
                           int32_t x0, int32_t th, int32_t tw, int32_t base, int32_t *d_plane,
                           void *stream) {
    if (!d_tile_labels || !d_plane || th < 1 || tw < 1 || y0 < 0 || x0 < 0 || y0 + th > h ||
        x0 + tw > w)
        return FX_ERR_INVALID_ARGUMENT;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_tile_scatter<<<grid_for((int64_t)th * tw), kRouteThreads, 0, st>>>(d_tile_labels, w, y0, x0,
                                                                        th, tw, base, d_plane);
    return cudaStreamSynchronize(st) == cudaSuccess ? FX_OK : FX_ERR_CUDA;
}
