// supertile.cu -- per-tile splat lists from the supertile-sorted slots.
//
// The reference pushes every projected splat, in depth order, into the list
// of each 16x16 tile its rectangle meets (src/cpu/backward.rs:190-205). Here
// the depth-ordered slots are first binned by supertile -- ST_EDGE x ST_EDGE
// CTA tiles, so a splat meets only a few of them -- with a short stable radix
// sort of (supertile, slot) entries. The sorted entries are then cut into
// chunks of ST_CHUNK, whatever supertiles they belong to, so every CTA gets
// the same work however unevenly the splats crowd the supertiles:
//   k_st_masks: per entry, the tiles of its supertile the slot keeps (the
//               rectangle, or with pruning each tile row's kept span: the same
//               test on the same floats the projection counted with) as a
//               16-bit mask, bit t for tile position t = row * ST_EDGE + col;
//               per chunk and position, the entries with that bit set;
//   k_st_scan:  one CTA per position: an exclusive scan of its chunk counts;
//   k_st_lists: the lists. The pairs of position t form plane t of the list
//               buffer, in entry order, the planes one after another; the
//               list of a tile (the entries of one supertile with bit t) is
//               then one contiguous run of its plane. An entry's place in
//               plane t is the plane's start + its chunk's scanned count + the
//               entries before it in the chunk with bit t (one ballot per
//               position per 32 entries). The first and the last entry of each
//               supertile write the [start, end) of its tiles.
// The supertile sort is stable and its input is in depth order, so each list
// holds its splats in depth order with ties in slot order: the lists the
// per-pair (tile, slot) sort produced, element for element, with the pairs
// never materialised as keys.
#include <algorithm>

#include "rgs_internal.cuh"
#include "tiles.cuh"

namespace rgs {

constexpr int ST_THREADS = 256;
constexpr int ST_WARPS = ST_THREADS / 32;
constexpr int ST_RUN = 4;                      // rounds of 32 entries per warp and chunk
constexpr int ST_CHUNK = ST_THREADS * ST_RUN;  // a warp takes 32 * ST_RUN consecutive entries
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_PER = 8;
static_assert(ST_TILES <= 32, "one lane per tile position");

size_t supertile_chunks(size_t entries) { return ((entries + ST_CHUNK - 1) / ST_CHUNK + 3) & ~(size_t)3; }

__device__ __forceinline__ uint32_t st_entries(const SupertileArgs& a) { return min(*a.n_ent, a.cap); }

__device__ __forceinline__ int st_view(const DevCam* cams, int nviews, int st) {
    int v = 0;
    while (v + 1 < nviews && cams[v + 1].st_base <= st) ++v;
    return v;
}

// The tiles of supertile (sx, sy) of view c that `slot` keeps: bit
// r * ST_EDGE + q for the tile in column sx * ST_EDGE + q, row sy * ST_EDGE + r.
__device__ __forceinline__ uint32_t slot_mask(const SupertileArgs& a, const DevCam& c, uint32_t slot, int sx, int sy) {
    const uint2 d = a.tdesc[slot];
    const int lt = (int)d.x - c.tile_base;
    const int ty0 = lt / c.tiles_x, cx0 = lt - ty0 * c.tiles_x;
    const int cx1 = cx0 + (int)(d.y & 0xffffu), ty1 = ty0 + (int)(d.y >> 16);
    const int r0 = max(ty0, sy * ST_EDGE), r1 = min(ty1, sy * ST_EDGE + ST_EDGE);
    const int q0 = sx * ST_EDGE, q1 = q0 + ST_EDGE;
    SpanSetup u{};
    if (a.prune) {
        const float4 A = a.rec[slot], Q = a.rec[a.S + slot];
        u = span_setup(A.x, A.y, Q.x, Q.y, Q.z, power_floor(A.z));
    }
    uint32_t m = 0;
    for (int r = r0; r < r1; ++r) {
        int c0 = cx0, c1 = cx1;
        if (a.prune) kept_cols(u, r, a.tile_w, a.tile_h, c.height, cx0, cx1, c0, c1);
        c0 = max(c0, q0);
        c1 = min(c1, q1);
        if (c1 > c0) m |= ((1u << (c1 - c0)) - 1u) << ((r - sy * ST_EDGE) * ST_EDGE + (c0 - q0));
    }
    return m;
}

// Adds, in lane t, the entries of this round of 32 whose mask has bit t.
__device__ __forceinline__ void count_bits(uint32_t m, int lane, uint32_t& my) {
#pragma unroll
    for (int t = 0; t < ST_TILES; ++t) {
        const uint32_t b = __ballot_sync(0xffffffffu, (m >> t) & 1u);
        if (lane == t) my += (uint32_t)__popc(b);
    }
}

__global__ void __launch_bounds__(ST_THREADS) k_st_masks(SupertileArgs a) {
    __shared__ uint32_t s_wt[ST_TILES][ST_WARPS];
    const uint32_t n = st_entries(a), nch = (n + ST_CHUNK - 1) / ST_CHUNK;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
        const uint32_t e0 = ch * ST_CHUNK + (uint32_t)(w * 32 * ST_RUN + lane);
        uint32_t my = 0;
#pragma unroll
        for (int r = 0; r < ST_RUN; ++r) {
            const uint32_t e = e0 + (uint32_t)(32 * r);
            uint32_t m = 0;
            if (e < n) {
                const int st = (int)a.ent_key[e];
                const DevCam& c = a.cams[st_view(a.cams, a.nviews, st)];
                const int local = st - c.st_base, sy = local / c.st_x, sx = local - sy * c.st_x;
                m = slot_mask(a, c, a.ent_slot[e], sx, sy);
                a.masks[e] = (uint16_t)m;
            }
            count_bits(m, lane, my);
        }
        if (lane < ST_TILES) s_wt[lane][w] = my;
        __syncthreads();
        if (threadIdx.x < ST_TILES) {
            uint32_t s = 0;
#pragma unroll
            for (int k = 0; k < ST_WARPS; ++k) s += s_wt[threadIdx.x][k];
            a.chunk_cnt[(size_t)threadIdx.x * a.chunk_stride + ch] = s;
        }
        __syncthreads();
    }
}

// Block t: exclusive scan, in place, of position t's chunk counts; the
// plane's total to plane_tot[t]. Every plane holds at most the entry count,
// so 32 bits suffice.
__global__ void __launch_bounds__(SCAN_THREADS) k_st_scan(SupertileArgs a) {
    __shared__ uint32_t s_w[SCAN_THREADS / 32];
    const uint32_t n = st_entries(a), nch = (n + ST_CHUNK - 1) / ST_CHUNK;
    uint32_t* cnt = a.chunk_cnt + (size_t)blockIdx.x * a.chunk_stride;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t carry = 0;  // the same in every thread
    for (uint32_t base = 0; base < nch; base += SCAN_THREADS * SCAN_PER) {
        const uint32_t i0 = base + (uint32_t)threadIdx.x * SCAN_PER;
        uint32_t v[SCAN_PER], sum = 0;
#pragma unroll
        for (int k = 0; k < SCAN_PER; ++k) {
            v[k] = i0 + k < nch ? cnt[i0 + k] : 0u;
            sum += v[k];
        }
        uint32_t x = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_w[w] = x;
        __syncthreads();
        uint32_t wpre = 0, tot = 0;
        for (int k = 0; k < SCAN_THREADS / 32; ++k) {
            const uint32_t t = s_w[k];
            if (k < w) wpre += t;
            tot += t;
        }
        uint32_t run = carry + wpre + x - sum;
#pragma unroll
        for (int k = 0; k < SCAN_PER; ++k) {
            if (i0 + k < nch) cnt[i0 + k] = run;
            run += v[k];
        }
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) a.plane_tot[blockIdx.x] = carry;
}

__global__ void __launch_bounds__(ST_THREADS) k_st_lists(SupertileArgs a) {
    __shared__ uint32_t s_wt[ST_TILES][ST_WARPS];
    const uint32_t n = st_entries(a), nch = (n + ST_CHUNK - 1) / ST_CHUNK;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    // lane t: where plane t starts (the planes before it, in 64 bits)
    unsigned long long plane0 = 0;
    if (lane < ST_TILES)
        for (int t = 0; t < lane; ++t) plane0 += a.plane_tot[t];
    for (uint32_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
        const uint32_t e0 = ch * ST_CHUNK + (uint32_t)(w * 32 * ST_RUN + lane);
        uint32_t m[ST_RUN], key[ST_RUN], slot[ST_RUN], my = 0;
#pragma unroll
        for (int r = 0; r < ST_RUN; ++r) {
            const uint32_t e = e0 + (uint32_t)(32 * r);
            const bool valid = e < n;
            m[r] = valid ? (uint32_t)a.masks[e] : 0u;
            key[r] = valid ? a.ent_key[e] : 0xffffffffu;
            slot[r] = valid ? a.ent_slot[e] : 0u;
            count_bits(m[r], lane, my);
        }
        if (lane < ST_TILES) s_wt[lane][w] = my;
        __syncthreads();
        // lane t: the next place in plane t for this warp's entries
        unsigned long long run = 0;
        if (lane < ST_TILES) {
            run = plane0 + a.chunk_cnt[(size_t)lane * a.chunk_stride + ch];
            for (int k = 0; k < w; ++k) run += s_wt[lane][k];
        }
#pragma unroll
        for (int r = 0; r < ST_RUN; ++r) {
            const uint32_t e = e0 + (uint32_t)(32 * r);
            const bool valid = e < n;
            // the neighbouring entries' supertiles (the warp's runs are
            // consecutive entries: round r - 1's lane 31 precedes lane 0)
            uint32_t prev = __shfl_up_sync(0xffffffffu, key[r], 1);
            uint32_t next = __shfl_down_sync(0xffffffffu, key[r], 1);
            const uint32_t pw = r > 0 ? __shfl_sync(0xffffffffu, key[r > 0 ? r - 1 : 0], 31) : 0u;
            const uint32_t nw = r + 1 < ST_RUN ? __shfl_sync(0xffffffffu, key[r + 1 < ST_RUN ? r + 1 : r], 0) : 0u;
            if (lane == 0) prev = r > 0 ? pw : (valid && e > 0 ? a.ent_key[e - 1] : 0xffffffffu);
            if (lane == 31) next = r + 1 < ST_RUN ? nw : (valid && e + 1 < n ? a.ent_key[e + 1] : 0xffffffffu);
            const bool first = valid && prev != key[r], last = valid && next != key[r];
            int tile0 = 0, tiles_x = 0, tiles_y = 0, sx = 0, sy = 0;
            if (first || last) {
                const int st = (int)key[r];
                const DevCam& c = a.cams[st_view(a.cams, a.nviews, st)];
                const int local = st - c.st_base;
                sy = local / c.st_x;
                sx = local - sy * c.st_x;
                tile0 = c.tile_base;
                tiles_x = c.tiles_x;
                tiles_y = c.tiles_y;
            }
#pragma unroll
            for (int t = 0; t < ST_TILES; ++t) {
                const uint32_t bit = (m[r] >> t) & 1u;
                const uint32_t b = __ballot_sync(0xffffffffu, bit);
                const unsigned long long at = __shfl_sync(0xffffffffu, run, t) + (uint32_t)__popc(b & lt_mask);
                if (bit) {
                    if (at < a.cap) a.vals_out[at] = slot[r];
                    else *a.overflow = 1;
                }
                if (first || last) {
                    const int tx = sx * ST_EDGE + t % ST_EDGE, ty = sy * ST_EDGE + t / ST_EDGE;
                    if (tx < tiles_x && ty < tiles_y) {
                        uint32_t* rg = reinterpret_cast<uint32_t*>(a.ranges + (tile0 + ty * tiles_x + tx));
                        if (first) rg[0] = (uint32_t)min(at, (unsigned long long)a.cap);
                        if (last) rg[1] = (uint32_t)min(at + bit, (unsigned long long)a.cap);
                    }
                }
                if (lane == t) run += (uint32_t)__popc(b);
            }
        }
        __syncthreads();  // s_wt is rewritten by the next chunk
    }
}

void launch_supertile_lists(const SupertileArgs& a, cudaStream_t st) {
    const int grid = (int)std::max<size_t>(1, std::min<size_t>(a.chunk_stride, (size_t)device_sm_count() * 8));
    k_st_masks<<<grid, ST_THREADS, 0, st>>>(a);
    k_st_scan<<<ST_TILES, SCAN_THREADS, 0, st>>>(a);
    k_st_lists<<<grid, ST_THREADS, 0, st>>>(a);
}

}  // namespace rgs
