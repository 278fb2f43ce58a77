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
//               rectangle, or with pruning each tile row's kept span, read
//               from the spans the projection packed in the slot's 32-byte
//               record, or for rectangles too large to pack recomputed by
//               the same test on the same floats the projection counted
//               with) as a 16-bit mask, bit t for tile position
//               t = row * ST_EDGE + col; per chunk and position, the entries
//               with that bit set (packed byte counters);
//   k_st_scan:  one CTA per position: an exclusive scan of its chunk counts;
//   k_st_lists: the lists. The pairs of position t form plane t of the list
//               buffer, in entry order, the planes one after another; the
//               list of a tile (the entries of one supertile with bit t) is
//               then one contiguous run of its plane. An entry's place in
//               plane t is the plane's start + its chunk's scanned count + the
//               entries before it in the chunk with bit t (a lane scan of the
//               byte counters). The first and the last entry of each
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

// A slot's CTA-tile rectangle within its view.
struct SlotRect {
    int cx0, ty0, w, h;
};

__device__ __forceinline__ SlotRect slot_rect(const DevCam& c, uint2 d) {
    SlotRect q;
    const int lt = (int)d.x - c.tile_base;
    q.ty0 = lt / c.tiles_x;
    q.cx0 = lt - q.ty0 * c.tiles_x;
    q.w = (int)(d.y & 0xffffu);
    q.h = (int)(d.y >> 16);
    return q;
}

// Bits of row k of a supertile whose first column is q0 for the kept columns
// [c0, c1): bit k * ST_EDGE + q for column q0 + q.
__device__ __forceinline__ uint32_t row_bits(int c0, int c1, int q0, int k) {
    c0 = max(c0, q0);
    c1 = min(c1, q0 + ST_EDGE);
    return c1 > c0 ? ((1u << (c1 - c0)) - 1u) << (k * ST_EDGE + (c0 - q0)) : 0u;
}

// The tiles of supertile (sx, sy) the slot's rectangle holds (no pruning).
__device__ __forceinline__ uint32_t mask_rect(const SlotRect& q, int sx, int sy) {
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < ST_EDGE; ++k) {
        const int rr = sy * ST_EDGE + k - q.ty0;
        if (rr >= 0 && rr < q.h) m |= row_bits(q.cx0, q.cx0 + q.w, sx * ST_EDGE, k);
    }
    return m;
}

// The same with pruning, from the spans the projection packed (byte rr: first
// kept column - cx0 | kept count << 4 of rectangle row rr).
__device__ __forceinline__ uint32_t mask_packed(const SlotRect& q, uint4 pk, int sx, int sy) {
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < ST_EDGE; ++k) {
        const int rr = sy * ST_EDGE + k - q.ty0;
        if (rr >= 0 && rr < q.h) {
            const uint32_t wd = rr < 4 ? pk.x : rr < 8 ? pk.y : rr < 12 ? pk.z : pk.w;
            const uint32_t b = (wd >> (8 * (rr & 3))) & 0xffu;
            const int c0 = q.cx0 + (int)(b & 0xfu);
            m |= row_bits(c0, c0 + (int)(b >> 4), sx * ST_EDGE, k);
        }
    }
    return m;
}

// The same with the spans recomputed from the slot's records (rectangles too
// large to pack): the test the projection counted with, on the same floats.
__device__ __forceinline__ uint32_t mask_computed(const float4* __restrict__ rec, uint32_t S, int tile_w, int tile_h,
                                                  int height, uint32_t slot, const SlotRect& q, int sx, int sy) {
    const float4 A = rec[slot], Q = rec[S + slot];
    const SpanSetup u = span_setup(A.x, A.y, Q.x, Q.y, Q.z, power_floor(A.z));
    uint32_t m = 0;
    const int r0 = max(q.ty0, sy * ST_EDGE), r1 = min(q.ty0 + q.h, sy * ST_EDGE + ST_EDGE);
    for (int r = r0; r < r1; ++r) {
        int c0, c1;
        kept_cols(u, r, tile_w, tile_h, height, q.cx0, q.cx0 + q.w, c0, c1);
        m |= row_bits(c0, c1, sx * ST_EDGE, r - sy * ST_EDGE);
    }
    return m;
}

// A mask's 16 tile positions as byte counters: word k holds positions
// 4k .. 4k + 3, one byte each (bit j of the nibble moves to bit 8j; the four
// copies n << 7j of the nibble do not overlap, so the product has no carries).
// Sums of up to 255 masks stay within their bytes.
__device__ __forceinline__ void spread_mask(uint32_t m, uint32_t w[4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) w[k] = (((m >> (4 * k)) & 0xfu) * 0x00204081u) & 0x01010101u;
}

__device__ __forceinline__ uint32_t byte_of(uint32_t w, int j) { return (w >> (8 * j)) & 0xffu; }

// Warp sums of the byte counters (at most 32 * ST_RUN per byte) to s_w.
__device__ __forceinline__ void warp_counts(uint32_t acc[4], int lane, uint32_t* s_w) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) s_w[k] = acc[k];
    }
}

// Thread tid of the CTA takes entries ch * ST_CHUNK + tid + ST_THREADS * r:
// all ST_RUN entries' keys and slots are loaded before their rectangles and
// spans, so the gathers of the four are in flight together. Capped at 64
// registers for four CTAs per SM.
__global__ void __launch_bounds__(ST_THREADS, 4) k_st_masks(SupertileArgs a) {
    __shared__ uint32_t s_w[ST_WARPS][4];
    const uint32_t* __restrict__ ent_key = a.ent_key;
    const uint32_t* __restrict__ ent_slot = a.ent_slot;
    const uint2* __restrict__ tdesc = a.tdesc;
    const uint4* __restrict__ spans = a.spans;
    const uint32_t n = st_entries(a), nch = (n + ST_CHUNK - 1) / ST_CHUNK;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
        const uint32_t e0 = ch * ST_CHUNK + threadIdx.x;
        uint32_t st[ST_RUN], slot[ST_RUN];
#pragma unroll
        for (int r = 0; r < ST_RUN; ++r) {
            const uint32_t e = e0 + (uint32_t)(ST_THREADS * r);
            st[r] = e < n ? ent_key[e] : 0u;
            slot[r] = e < n ? ent_slot[e] : 0u;
        }
        uint2 d[ST_RUN];
        uint4 sp[ST_RUN];
#pragma unroll
        for (int r = 0; r < ST_RUN; ++r) {
            const uint32_t e = e0 + (uint32_t)(ST_THREADS * r);
            sp[r] = make_uint4(0u, 0u, 0u, 0u);
            d[r] = make_uint2(0u, 0u);
            if (e < n) {
                if (a.prune) {
                    // one 32-byte record: the spans, then the rectangle
                    sp[r] = spans[2 * (size_t)slot[r]];
                    const uint4 td = spans[2 * (size_t)slot[r] + 1];
                    d[r] = make_uint2(td.x, td.y);
                } else {
                    d[r] = tdesc[slot[r]];
                }
            }
        }
        uint32_t acc[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int r = 0; r < ST_RUN; ++r) {
            const uint32_t e = e0 + (uint32_t)(ST_THREADS * r);
            if (e < n) {
                const DevCam& c = a.cams[slot[r] / a.n_per_view];
                const int local = (int)st[r] - c.st_base, sy = local / c.st_x, sx = local - sy * c.st_x;
                const SlotRect q = slot_rect(c, d[r]);
                const uint32_t m = !a.prune                                 ? mask_rect(q, sx, sy)
                                   : (sp[r].x & 0xffu) != (SPANS_NONE & 0xffu) ? mask_packed(q, sp[r], sx, sy)
                                                      : mask_computed(a.rec, a.S, a.tile_w, a.tile_h, c.height, slot[r], q,
                                                                      sx, sy);
                a.masks[e] = (uint16_t)m;
                uint32_t x[4];
                spread_mask(m, x);
#pragma unroll
                for (int k = 0; k < 4; ++k) acc[k] += x[k];
            }
        }
        warp_counts(acc, lane, s_w[w]);
        __syncthreads();
        if (threadIdx.x < ST_TILES) {
            const int t = threadIdx.x;
            uint32_t s = 0;
#pragma unroll
            for (int k = 0; k < ST_WARPS; ++k) s += byte_of(s_w[k][t >> 2], t & 3);
            a.chunk_cnt[(size_t)t * a.chunk_stride + ch] = s;
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

// Warp w of the CTA takes the ST_RUN * 32 consecutive entries
// ch * ST_CHUNK + w * 32 * ST_RUN + [0, 32 * ST_RUN), in rounds of 32. An
// entry's place in plane t: the warp's start in that plane (s_base) + the
// entries of the warp's earlier rounds and earlier lanes with bit t, read off
// a lane scan of the byte counters.
__global__ void __launch_bounds__(ST_THREADS) k_st_lists(SupertileArgs a) {
    __shared__ uint32_t s_w[ST_WARPS][4];
    // the warp's start in each plane, clamped to the capacity: every place
    // formed from it then stays below 2^32 (cap <= 0xF0000000, the offsets
    // below 256) and a clamped start still flags the overflow
    __shared__ uint32_t s_base[ST_WARPS][ST_TILES];
    const uint32_t* __restrict__ ent_key = a.ent_key;
    const uint32_t* __restrict__ ent_slot = a.ent_slot;
    const uint16_t* __restrict__ masks = a.masks;
    const uint32_t n = st_entries(a), nch = (n + ST_CHUNK - 1) / ST_CHUNK;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    // lane t: where plane t starts (the planes before it, in 64 bits)
    unsigned long long plane0 = 0;
    if (lane < ST_TILES)
        for (int t = 0; t < lane; ++t) plane0 += a.plane_tot[t];
    for (uint32_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
        const uint32_t e0 = ch * ST_CHUNK + (uint32_t)(w * 32 * ST_RUN + lane);
        uint32_t m[ST_RUN], key[ST_RUN], slot[ST_RUN], acc[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int r = 0; r < ST_RUN; ++r) {
            const uint32_t e = e0 + (uint32_t)(32 * r);
            const bool valid = e < n;
            m[r] = valid ? (uint32_t)masks[e] : 0u;
            key[r] = valid ? ent_key[e] : 0xffffffffu;
            slot[r] = valid ? ent_slot[e] : 0u;
            uint32_t x[4];
            spread_mask(m[r], x);
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[k] += x[k];
        }
        warp_counts(acc, lane, s_w[w]);
        __syncthreads();
        if (lane < ST_TILES) {
            unsigned long long b = plane0 + a.chunk_cnt[(size_t)lane * a.chunk_stride + ch];
            for (int k = 0; k < w; ++k) b += byte_of(s_w[k][lane >> 2], lane & 3);
            s_base[w][lane] = (uint32_t)min(b, (unsigned long long)a.cap);
        }
        __syncwarp();
        uint32_t before[4] = {0u, 0u, 0u, 0u};  // the warp's earlier rounds, per byte (< 128)
#pragma unroll
        for (int r = 0; r < ST_RUN; ++r) {
            const uint32_t e = e0 + (uint32_t)(32 * r);
            const bool valid = e < n;
            uint32_t own[4], x[4], excl[4];
            spread_mask(m[r], own);
#pragma unroll
            for (int k = 0; k < 4; ++k) x[k] = own[k];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, x[k], o);
                    if (lane >= o) x[k] += y;
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                excl[k] = before[k] + x[k] - own[k];
                before[k] += __shfl_sync(0xffffffffu, x[k], 31);
            }
            // each set bit: the slot into its tile's list
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                uint32_t nib = (m[r] >> (4 * k)) & 0xfu;
                while (nib) {
                    const int j = __ffs(nib) - 1;
                    nib &= nib - 1u;
                    const uint32_t at = s_base[w][4 * k + j] + byte_of(excl[k], j);
                    if (at < a.cap) a.vals_out[at] = slot[r];
                    else *a.overflow = 1;
                }
            }
            // the neighbouring entries' supertiles (the warp's runs are
            // consecutive entries: round r - 1's lane 31 precedes lane 0)
            uint32_t prev = __shfl_up_sync(0xffffffffu, key[r], 1);
            uint32_t next = __shfl_down_sync(0xffffffffu, key[r], 1);
            const uint32_t pw = r > 0 ? __shfl_sync(0xffffffffu, key[r > 0 ? r - 1 : 0], 31) : 0u;
            const uint32_t nw = r + 1 < ST_RUN ? __shfl_sync(0xffffffffu, key[r + 1 < ST_RUN ? r + 1 : r], 0) : 0u;
            if (lane == 0) prev = r > 0 ? pw : (valid && e > 0 ? ent_key[e - 1] : 0xffffffffu);
            if (lane == 31) next = r + 1 < ST_RUN ? nw : (valid && e + 1 < n ? ent_key[e + 1] : 0xffffffffu);
            const bool first = valid && prev != key[r], last = valid && next != key[r];
            if (first || last) {
                // a supertile's first entry starts, its last ends, the lists
                // of all of its tiles
                const int st = (int)key[r];
                const DevCam& c = a.cams[slot[r] / a.n_per_view];
                const int local = st - c.st_base, sy = local / c.st_x, sx = local - sy * c.st_x;
#pragma unroll
                for (int t = 0; t < ST_TILES; ++t) {
                    const int tx = sx * ST_EDGE + t % ST_EDGE, ty = sy * ST_EDGE + t / ST_EDGE;
                    if (tx < c.tiles_x && ty < c.tiles_y) {
                        const uint32_t at = s_base[w][t] + byte_of(excl[t >> 2], t & 3);
                        uint32_t* rg = reinterpret_cast<uint32_t*>(a.ranges + (c.tile_base + ty * c.tiles_x + tx));
                        if (first) rg[0] = min(at, a.cap);
                        if (last) rg[1] = min(at + ((m[r] >> t) & 1u), a.cap);
                    }
                }
            }
        }
        __syncthreads();  // s_w and s_base are rewritten by the next chunk
    }
}

void launch_supertile_lists(const SupertileArgs& a, cudaStream_t st) {
    const int grid = (int)std::max<size_t>(1, std::min<size_t>(a.chunk_stride, (size_t)device_sm_count() * 8));
    k_st_masks<<<grid, ST_THREADS, 0, st>>>(a);
    k_st_scan<<<ST_TILES, SCAN_THREADS, 0, st>>>(a);
    k_st_lists<<<grid, ST_THREADS, 0, st>>>(a);
}

}  // namespace rgs
