// bin.cu -- binning the depth-sorted slots by supertile.
//
// The reference sorts visible splats by depth and then, serially, pushes each
// splat's index into every tile its 3-sigma rectangle touches
// (src/cpu/backward.rs:190-205). Here:
//   compact:    the slots with at least one tile pair are gathered in slot
//               order with their depth keys (the depth sort, sort.cu, then
//               orders only them), and each gets its supertile rectangle;
//   count scan: exclusive scans of per-slot counts in depth order, in 64 bits
//               (pruned tile pairs, and supertile entries; the totals stay
//               on the device, a count past 32 bits is reported, never
//               wrapped);
//   emit:       every block expands its chunk of depth-sorted slots into
//               (supertile id, slot) entries, load-balanced by a binary
//               search over the sub-tile's offsets in shared memory;
// then a stable radix sort on the supertile id (sort.cu) groups the entries
// by supertile while keeping depth order inside each, and supertile.cu
// expands them into the per-tile lists. Each slot's CTA-tile rectangle comes
// from the projection as one 8-byte descriptor (first tile id, width |
// height << 16).
#include "rgs_internal.cuh"
#include "tiles.cuh"

namespace rgs {

constexpr int BIN_THREADS = 256;
constexpr int BIN_SUB = 1024;  // ranks per emit sub-tile
constexpr int EMIT_VT = 8;     // consecutive pairs per thread per emit round
// staged-pair index with one pad word per 32, so a warp writing EMIT_VT-strided
// words hits 32 distinct banks
__device__ __forceinline__ int emit_pad(int i) { return i + (i >> 5); }

int bin_grid_blocks() { return device_sm_count() * 6; }

__device__ __forceinline__ void bin_chunk(uint32_t n, int G, int b, uint32_t& begin, uint32_t& end) {
    uint32_t chunk = (uint32_t)(((uint64_t)n + G - 1) / G);
    chunk = (chunk + 31u) & ~31u;
    uint64_t bg = (uint64_t)chunk * b;
    begin = (uint32_t)(bg < (uint64_t)n ? bg : (uint64_t)n);
    end = (uint32_t)(bg + chunk < (uint64_t)n ? bg + chunk : (uint64_t)n);
}

__device__ __forceinline__ uint32_t tiles_of(uint2 d) { return (d.y & 0xffffu) * (d.y >> 16); }

__global__ void __launch_bounds__(BIN_THREADS) k_count_reduce(const uint32_t* __restrict__ order, const uint32_t* __restrict__ cnt,
                                                              uint32_t S_host, const uint32_t* __restrict__ S_dev,
                                                              unsigned long long* __restrict__ block_sums) {
    __shared__ uint32_t s_w[BIN_THREADS / 32];
    const uint32_t S = S_dev ? *S_dev : S_host;
    uint32_t begin, end;
    bin_chunk(S, gridDim.x, blockIdx.x, begin, end);
    uint32_t s = 0;
    for (uint32_t r = begin + threadIdx.x; r < end; r += BIN_THREADS) s += cnt[order[r]];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < BIN_THREADS / 32; ++w) t += s_w[w];
        block_sums[blockIdx.x] = t;
    }
}

// Exclusive scan of the G block sums (single block) in 64 bits; writes the
// total to *total64 and, saturated at 2^32 - 1, to *total.
__global__ void __launch_bounds__(1024) k_scan_block_sums(unsigned long long* __restrict__ block_sums, int G,
                                                          uint32_t* __restrict__ total,
                                                          unsigned long long* __restrict__ total64) {
    __shared__ unsigned long long s[1024];
    __shared__ unsigned long long s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int base = 0; base < G; base += 1024) {
        int i = base + threadIdx.x;
        unsigned long long v = i < G ? block_sums[i] : 0ull;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            unsigned long long t = threadIdx.x >= o ? s[threadIdx.x - o] : 0ull;
            __syncthreads();
            s[threadIdx.x] += t;
            __syncthreads();
        }
        unsigned long long incl = s[threadIdx.x];
        if (i < G) block_sums[i] = s_carry + incl - v;
        __syncthreads();
        if (threadIdx.x == 1023) s_carry += incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *total = s_carry > 0xffffffffull ? 0xffffffffu : (uint32_t)s_carry;
        *total64 = s_carry;
    }
}

void launch_count_scan(const uint32_t* order, const uint32_t* cnt, uint32_t S, const uint32_t* S_dev,
                       unsigned long long* block_sums, uint32_t* total, unsigned long long* total64, int grid, cudaStream_t st) {
    k_count_reduce<<<grid, BIN_THREADS, 0, st>>>(order, cnt, S, S_dev, block_sums);
    k_scan_block_sums<<<1, 1024, 0, st>>>(block_sums, grid, total, total64);
}

__global__ void __launch_bounds__(BIN_THREADS) k_view_pairs(const uint32_t* __restrict__ cnt, uint32_t n,
                                                            unsigned long long* __restrict__ out) {
    __shared__ unsigned long long s_w[BIN_THREADS / 32];
    const uint32_t* c = cnt + (size_t)blockIdx.x * n;
    unsigned long long t = 0;
    for (uint32_t i = threadIdx.x; i < n; i += BIN_THREADS) t += c[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long v = 0;
        for (int w = 0; w < BIN_THREADS / 32; ++w) v += s_w[w];
        out[blockIdx.x] = v;
    }
}

void launch_view_pairs(const uint32_t* cnt, uint32_t n, int V, unsigned long long* out, cudaStream_t st) {
    if (V > 0) k_view_pairs<<<V, BIN_THREADS, 0, st>>>(cnt, n, out);
}

// Expands each slot's supertile rectangle (first supertile id, width |
// height << 16; a view's supertiles are row-major, st_x per row) into
// (supertile id, slot) entries.
__global__ void __launch_bounds__(BIN_THREADS) k_emit(const uint32_t* __restrict__ order, const uint2* __restrict__ tdesc,
                                                      uint32_t S_host, const uint32_t* __restrict__ S_dev,
                                                      const unsigned long long* __restrict__ block_sums, uint32_t* __restrict__ pkeys,
                                                      uint32_t* __restrict__ pvals, uint32_t cap, int* __restrict__ overflow,
                                                      const uint32_t* __restrict__ total, uint32_t* __restrict__ eff,
                                                      const DevCam* __restrict__ cams, uint32_t n_per_view) {
    __shared__ uint32_t s_off[BIN_SUB + 1];
    __shared__ uint32_t s_slot[BIN_SUB];
    __shared__ uint2 s_desc[BIN_SUB];  // (first supertile id, rect width | view st_x << 16)
    __shared__ uint32_t s_w[BIN_THREADS / 32];
    __shared__ uint32_t s_ek[BIN_THREADS * EMIT_VT + BIN_THREADS * EMIT_VT / 32];
    __shared__ uint32_t s_ev[BIN_THREADS * EMIT_VT + BIN_THREADS * EMIT_VT / 32];
    constexpr int PER = BIN_SUB / BIN_THREADS;
    int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    uint32_t begin, end;
    // S_host: slots (the stride of the record planes); the order may hold fewer
    const uint32_t S = S_host, n_order = S_dev ? *S_dev : S_host;
    bin_chunk(n_order, gridDim.x, blockIdx.x, begin, end);
    if (blockIdx.x == 0 && threadIdx.x == 0) *eff = min(*total, cap);
    unsigned long long base = block_sums[blockIdx.x];
    for (uint32_t r0 = begin; r0 < end; r0 += BIN_SUB) {
        // per-thread consecutive ranks r0 + tid*PER + k
        uint32_t c[PER], local = 0;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            uint32_t r = r0 + (uint32_t)(tid * PER + k);
            uint32_t slot = r < end ? order[r] : 0u;
            uint2 d = r < end ? tdesc[slot] : make_uint2(0u, 0u);
            c[k] = tiles_of(d);
            s_slot[tid * PER + k] = slot;
            if (c[k]) {
                const DevCam& cm = cams[slot / n_per_view];
                d.y = (d.y & 0xffffu) | ((uint32_t)cm.st_x << 16);
            }
            s_desc[tid * PER + k] = d;
            local += c[k];
        }
        uint32_t x = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_w[w] = x;
        __syncthreads();
        uint32_t wpre = 0, sub_total = 0;
        for (int k = 0; k < BIN_THREADS / 32; ++k) {
            uint32_t t = s_w[k];
            if (k < w) wpre += t;
            sub_total += t;
        }
        uint32_t run = wpre + x - local;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            s_off[tid * PER + k] = run;
            run += c[k];
        }
        if (tid == 0) s_off[BIN_SUB] = sub_total;
        __syncthreads();
        // Expansion in rounds of BIN_THREADS * EMIT_VT outputs: every thread
        // produces EMIT_VT consecutive pairs (one binary search for the first,
        // then a walk along the rectangles), stages them in shared memory, and
        // the block writes the round out with consecutive threads on
        // consecutive addresses.
        for (uint32_t o0 = 0; o0 < sub_total; o0 += BIN_THREADS * EMIT_VT) {
            const uint32_t qb = o0 + (uint32_t)(tid * EMIT_VT);
            if (qb < sub_total) {
                // largest r with s_off[r] <= qb (that entry has a non-zero count)
                int lo = 0, hi = BIN_SUB - 1;
                while (lo < hi) {
                    int mid = (lo + hi + 1) >> 1;
                    if (s_off[mid] <= qb) lo = mid;
                    else hi = mid - 1;
                }
                int r = lo;
                uint2 d = s_desc[r];
                uint32_t wt = d.y & 0xffffu;
                uint32_t j = qb - s_off[r];
                uint32_t row = j / wt, col = j - row * wt;
                uint32_t next = s_off[r + 1];
#pragma unroll
                for (int k = 0; k < EMIT_VT; ++k) {
                    const uint32_t q = qb + (uint32_t)k;
                    if (q >= sub_total) break;
                    while (q >= next) {  // next rectangle with a non-zero count
                        ++r;
                        next = s_off[r + 1];
                        d = s_desc[r];
                        wt = d.y & 0xffffu;
                        row = 0;
                        col = 0;
                    }
                    // supertile ids of one view are row-major: row `row` of the
                    // rectangle starts row * st_x after its first supertile
                    const int sp = emit_pad(tid * EMIT_VT + k);
                    s_ek[sp] = d.x + row * (d.y >> 16) + col;
                    s_ev[sp] = s_slot[r];
                    if (++col == wt) {
                        col = 0;
                        ++row;
                    }
                }
            }
            __syncthreads();
            const uint32_t n_round = min((uint32_t)(BIN_THREADS * EMIT_VT), sub_total - o0);
            for (uint32_t i = tid; i < n_round; i += BIN_THREADS) {
                const unsigned long long out = base + o0 + i;
                if (out < cap) {
                    pkeys[out] = s_ek[emit_pad((int)i)];
                    pvals[out] = s_ev[emit_pad((int)i)];
                } else {
                    *overflow = 1;
                }
            }
            __syncthreads();
        }
        base += sub_total;
        __syncthreads();
    }
}

void launch_emit_supertiles(const uint32_t* order, const uint2* st_desc, uint32_t S, const uint32_t* S_dev,
                            const unsigned long long* block_sums, uint32_t* keys, uint32_t* vals, uint32_t cap, int* overflow,
                            const uint32_t* total, uint32_t* eff, const DevCam* cams, uint32_t n_per_view, int grid,
                            cudaStream_t st) {
    k_emit<<<grid, BIN_THREADS, 0, st>>>(order, st_desc, S, S_dev, block_sums, keys, vals, cap, overflow, total, eff, cams,
                                               n_per_view);
}

// ---- slots with tile pairs, compacted in slot order ------------------------
// Before the depth sort, the slots that emit at least one pair are gathered,
// in slot order, with their depth keys: the sort then orders only them, and
// because it is stable and the gather keeps slot order, equal depths still
// leave Gaussians of a view in index order. Chunks of CMP_CHUNK consecutive
// slots: count per chunk, one exclusive scan, then a stable in-chunk scatter.
constexpr int CMP_PER = 4;
constexpr int CMP_CHUNK = BIN_THREADS * CMP_PER;

__global__ void __launch_bounds__(BIN_THREADS) k_visible_counts(const uint32_t* __restrict__ cnt, uint32_t S,
                                                                unsigned long long* __restrict__ chunk_counts) {
    __shared__ uint32_t s_w[BIN_THREADS / 32];
    const uint32_t base = blockIdx.x * (uint32_t)CMP_CHUNK + threadIdx.x * CMP_PER;
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < CMP_PER; ++k) c += (base + k < S && cnt[base + k] != 0u) ? 1u : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < BIN_THREADS / 32; ++w) t += s_w[w];
        chunk_counts[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(BIN_THREADS) k_compact_visible(const uint32_t* __restrict__ cnt, const uint32_t* __restrict__ key,
                                                                 uint32_t S, const unsigned long long* __restrict__ chunk_offs,
                                                                 uint32_t* __restrict__ ckey, uint32_t* __restrict__ cslot,
                                                                 const uint2* __restrict__ tdesc, const DevCam* __restrict__ cams,
                                                                 uint32_t n_per_view, uint32_t* __restrict__ st_cnt,
                                                                 uint2* __restrict__ st_desc) {
    __shared__ uint32_t s_w[BIN_THREADS / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t base = blockIdx.x * (uint32_t)CMP_CHUNK + threadIdx.x * CMP_PER;
    // every slot's count, depth key and tile rectangle in one round trip
    // (a culled slot's key and rectangle are read and dropped)
    bool f[CMP_PER];
    uint32_t kv[CMP_PER];
    uint2 dv[CMP_PER];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < CMP_PER; ++k) {
        const bool in = base + k < S;
        f[k] = in && cnt[base + k] != 0u;
        kv[k] = in ? key[base + k] : 0u;
        dv[k] = in ? tdesc[base + k] : make_uint2(0u, 0u);
        local += f[k] ? 1u : 0u;
    }
    uint32_t x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[w] = x;
    __syncthreads();
    uint32_t wpre = 0;
    for (int k = 0; k < w; ++k) wpre += s_w[k];
    uint32_t pos = (uint32_t)chunk_offs[blockIdx.x] + wpre + x - local;
#pragma unroll
    for (int k = 0; k < CMP_PER; ++k) {
        if (f[k]) {
            const uint32_t slot = base + k;
            ckey[pos] = kv[k];
            cslot[pos] = slot;
            ++pos;
            // the supertiles its tile rectangle meets
            const DevCam& c = cams[slot / n_per_view];
            const uint2 d = dv[k];
            const int lt = (int)d.x - c.tile_base;
            const int ty0 = lt / c.tiles_x, cx0 = lt - ty0 * c.tiles_x;
            const int sx0 = cx0 / ST_EDGE, sx1 = (cx0 + (int)(d.y & 0xffffu) - 1) / ST_EDGE;
            const int sy0 = ty0 / ST_EDGE, sy1 = (ty0 + (int)(d.y >> 16) - 1) / ST_EDGE;
            st_cnt[slot] = (uint32_t)((sx1 - sx0 + 1) * (sy1 - sy0 + 1));
            st_desc[slot] = make_uint2((uint32_t)(c.st_base + sy0 * c.st_x + sx0),
                                       (uint32_t)(sx1 - sx0 + 1) | ((uint32_t)(sy1 - sy0 + 1) << 16));
        }
    }
}

size_t compact_chunks(size_t S) { return (S + CMP_CHUNK - 1) / CMP_CHUNK; }

void launch_compact_visible(const uint32_t* cnt, const uint32_t* key, uint32_t S, unsigned long long* chunk_counts,
                            uint32_t* ckey, uint32_t* cslot, uint32_t* n_out, unsigned long long* n_out64,
                            const uint2* tdesc, const DevCam* cams, uint32_t n_per_view, uint32_t* st_cnt, uint2* st_desc,
                            cudaStream_t st) {
    const unsigned chunks = (unsigned)compact_chunks(S);
    if (chunks == 0) {
        cudaMemsetAsync(n_out, 0, 4, st);
        cudaMemsetAsync(n_out64, 0, 8, st);
        return;
    }
    k_visible_counts<<<chunks, BIN_THREADS, 0, st>>>(cnt, S, chunk_counts);
    k_scan_block_sums<<<1, 1024, 0, st>>>(chunk_counts, (int)chunks, n_out, n_out64);
    k_compact_visible<<<chunks, BIN_THREADS, 0, st>>>(cnt, key, S, chunk_counts, ckey, cslot, tdesc, cams, n_per_view, st_cnt,
                                                      st_desc);
}

}  // namespace rgs
