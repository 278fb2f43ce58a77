// bin.cu -- tile binning: (CTA tile, slot) pairs in front-to-back order.
//
// The reference sorts visible splats by depth and then, serially, pushes each
// splat's index into every tile its 3-sigma rectangle touches
// (src/cpu/backward.rs:190-205). Here the depth-sorted slot order comes from
// sort.cu; this file turns it into pairs:
//   count scan: exclusive scan of per-slot tile counts in depth order, in
//               64 bits (the total pair count stays on the device; a batch
//               whose count passes 32 bits is reported, never wrapped);
//   emit:       every block expands its chunk of depth-sorted slots into
//               (global CTA tile id, slot) pairs, load-balanced by a binary
//               search over the sub-tile's offsets in shared memory;
// then a stable radix sort on the tile id (sort.cu) groups the pairs by tile
// while keeping depth order inside each tile, and `tile_ranges` records each
// tile's [start, end). Each slot's CTA-tile rectangle comes from the
// projection as one 8-byte descriptor (first tile id, width | height << 16),
// the only per-splat gather of these kernels.
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

__global__ void __launch_bounds__(BIN_THREADS) k_emit(const uint32_t* __restrict__ order, const uint2* __restrict__ tdesc,
                                                      uint32_t S_host, const uint32_t* __restrict__ S_dev,
                                                      const unsigned long long* __restrict__ block_sums, uint32_t* __restrict__ pkeys,
                                                      uint32_t* __restrict__ pvals, uint32_t cap, int* __restrict__ overflow,
                                                      const uint32_t* __restrict__ total, uint32_t* __restrict__ eff,
                                                      const DevCam* __restrict__ cams, uint32_t n_per_view) {
    __shared__ uint32_t s_off[BIN_SUB + 1];
    __shared__ uint32_t s_slot[BIN_SUB];
    __shared__ uint2 s_desc[BIN_SUB];  // (first tile id, rect width | view tiles_x << 16)
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
            if (c[k]) d.y = (d.y & 0xffffu) | ((uint32_t)cams[slot / n_per_view].tiles_x << 16);
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
                    // tile ids of one view are row-major: row `row` of the
                    // rectangle starts row * tiles_x after its first tile
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

// Pruned emission: a slot's pairs are the tiles of its rows' kept spans
// (tiles.cuh), recomputed here from the stored record exactly as the
// projection counted them. Each slot of a sub-tile goes to a group of EG
// lanes, one lane per rectangle row (EG rows at a time): the lanes compute
// their rows' spans, a group scan turns the span lengths into offsets, and
// every lane writes its row's run of consecutive pairs. The warp's groups
// step together for the tallest of their rectangles. Four lanes per slot:
// most rectangles are a few rows tall, so eight left half the lanes idle
// (measured 12 % slower).
constexpr int EG = 4;
__global__ void __launch_bounds__(BIN_THREADS) k_emit_pruned(const uint32_t* __restrict__ order, const uint2* __restrict__ tdesc,
                                                             const uint32_t* __restrict__ cnt, const float4* __restrict__ rec,
                                                             uint32_t S_host, const uint32_t* __restrict__ S_dev,
                                                             const unsigned long long* __restrict__ block_sums,
                                                             uint32_t* __restrict__ pkeys, uint32_t* __restrict__ pvals,
                                                             uint32_t cap, int* __restrict__ overflow,
                                                             const uint32_t* __restrict__ total, uint32_t* __restrict__ eff,
                                                             const unsigned long long* __restrict__ total64,
                                                             const DevCam* __restrict__ cams, uint32_t n_per_view, int tile_w,
                                                             int tile_h) {
    __shared__ uint32_t s_off[BIN_SUB + 1];
    __shared__ uint32_t s_slot[BIN_SUB];
    __shared__ uint32_t s_w[BIN_THREADS / 32];
    constexpr int PER = BIN_SUB / BIN_THREADS;
    constexpr int NGROUPS = BIN_THREADS / EG;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int grp = tid / EG, gl = tid % EG;
    uint32_t begin, end;
    // S_host: slots (the stride of the record planes); the order may hold fewer
    const uint32_t S = S_host, n_order = S_dev ? *S_dev : S_host;
    bin_chunk(n_order, gridDim.x, blockIdx.x, begin, end);
    if (blockIdx.x == 0 && threadIdx.x == 0) *eff = min(*total, cap);
    unsigned long long base = block_sums[blockIdx.x];
    // culled slots sort last (depth key ~0), so whole chunks of the depth
    // order emit nothing: such a block leaves at once
    const unsigned long long block_end = blockIdx.x + 1 < gridDim.x ? block_sums[blockIdx.x + 1] : *total64;
    if (block_end == base) return;
    for (uint32_t r0 = begin; r0 < end; r0 += BIN_SUB) {
        uint32_t c[PER], local = 0;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const uint32_t r = r0 + (uint32_t)(tid * PER + k);
            const uint32_t slot = r < end ? order[r] : 0u;
            c[k] = r < end ? cnt[slot] : 0u;
            s_slot[tid * PER + k] = slot;
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
        if (sub_total == 0) continue;  // block-uniform; s_w was read before the barrier
        for (int k0 = 0; k0 < BIN_SUB; k0 += NGROUPS) {
            const int k = k0 + grp;
            const uint32_t nk = s_off[k + 1] - s_off[k];
            const unsigned long long out0 = base + s_off[k];
            // entries of this slot's run that fit below the capacity
            const uint32_t room = out0 >= cap ? 0u : (uint32_t)min((unsigned long long)nk, cap - out0);
            uint32_t* const pk = pkeys + (out0 < cap ? out0 : 0ull);
            uint32_t* const pv = pvals + (out0 < cap ? out0 : 0ull);
            uint32_t slot = 0, tbase = 0;
            int cx0 = 0, cx1 = 0, ty0 = 0, rows = 0, tiles_x = 1, height = 0;
            SpanSetup u{};
            if (nk) {
                slot = s_slot[k];
                const uint2 d = tdesc[slot];
                const DevCam* cam = cams + slot / n_per_view;
                tiles_x = cam->tiles_x;
                height = cam->height;
                tbase = (uint32_t)cam->tile_base;
                const int lt = (int)d.x - cam->tile_base;
                ty0 = lt / tiles_x;
                cx0 = lt - ty0 * tiles_x;
                cx1 = cx0 + (int)(d.y & 0xffffu);
                rows = (int)(d.y >> 16);
                const float4 A = rec[slot], Q = rec[S + slot];
                u = span_setup(A.x, A.y, Q.x, Q.y, Q.z, power_floor(A.z));
            }
            const int steps = __reduce_max_sync(0xffffffffu, (rows + EG - 1) / EG);
            uint32_t written = 0;
            for (int it = 0; it < steps; ++it) {
                const int row = it * EG + gl;
                int c0 = 0, c1 = 0;
                if (row < rows) kept_cols(u, ty0 + row, tile_w, tile_h, height, cx0, cx1, c0, c1);
                const uint32_t span = (uint32_t)(c1 - c0);
                uint32_t incl = span;
#pragma unroll
                for (int o = 1; o < EG; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o, EG);
                    if (gl >= o) incl += y;
                }
                const uint32_t gtot = __shfl_sync(0xffffffffu, incl, EG - 1, EG);
                uint32_t p = written + incl - span;
                const uint32_t key0 = tbase + (uint32_t)((ty0 + row) * tiles_x + c0);
                // two entries per 8-byte store once the output index is even
                // (pk, pv hold the run that starts at entry out0)
                uint32_t t = 0;
                if (((out0 + p) & 1ull) && t < span) {
                    if (p < room) {
                        pk[p] = key0;
                        pv[p] = slot;
                    } else {
                        *overflow = 1;
                    }
                    ++t;
                    ++p;
                }
                for (; t + 1 < span; t += 2, p += 2) {
                    if (p + 1 < room) {
                        *reinterpret_cast<uint2*>(pk + p) = make_uint2(key0 + t, key0 + t + 1);
                        *reinterpret_cast<uint2*>(pv + p) = make_uint2(slot, slot);
                    } else {
                        if (p < room) {
                            pk[p] = key0 + t;
                            pv[p] = slot;
                        }
                        *overflow = 1;
                    }
                }
                if (t < span) {
                    if (p < room) {
                        pk[p] = key0 + t;
                        pv[p] = slot;
                    } else {
                        *overflow = 1;
                    }
                }
                written += gtot;
            }
            // the projection counted the same spans; a disagreement would
            // leave stale pairs, so it fails the step
            if (gl == 0 && written != nk) *overflow = 1;
        }
        base += sub_total;
        __syncthreads();
    }
}

void launch_emit_pairs(const uint32_t* order, const uint2* tdesc, const uint32_t* cnt, const float4* rec, uint32_t S,
                       const uint32_t* S_dev, const unsigned long long* block_sums, uint32_t* pair_keys, uint32_t* pair_vals,
                       uint32_t cap, int* overflow, const uint32_t* total, const unsigned long long* total64, uint32_t* eff,
                       const DevCam* cams, uint32_t n_per_view, int tile_w, int tile_h, int prune, int grid, cudaStream_t st) {
    if (prune)
        k_emit_pruned<<<grid, BIN_THREADS, 0, st>>>(order, tdesc, cnt, rec, (uint32_t)S, S_dev, block_sums, pair_keys, pair_vals,
                                                    cap, overflow, total, eff, total64, cams, n_per_view, tile_w, tile_h);
    else
        k_emit<<<grid, BIN_THREADS, 0, st>>>(order, tdesc, S, S_dev, block_sums, pair_keys, pair_vals, cap, overflow, total, eff,
                                             cams, n_per_view);
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
                                                                 uint32_t* __restrict__ ckey, uint32_t* __restrict__ cslot) {
    __shared__ uint32_t s_w[BIN_THREADS / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t base = blockIdx.x * (uint32_t)CMP_CHUNK + threadIdx.x * CMP_PER;
    bool f[CMP_PER];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < CMP_PER; ++k) {
        f[k] = base + k < S && cnt[base + k] != 0u;
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
            ckey[pos] = key[base + k];
            cslot[pos] = base + k;
            ++pos;
        }
    }
}

size_t compact_chunks(size_t S) { return (S + CMP_CHUNK - 1) / CMP_CHUNK; }

void launch_compact_visible(const uint32_t* cnt, const uint32_t* key, uint32_t S, unsigned long long* chunk_counts,
                            uint32_t* ckey, uint32_t* cslot, uint32_t* n_out, unsigned long long* n_out64, cudaStream_t st) {
    const unsigned chunks = (unsigned)compact_chunks(S);
    if (chunks == 0) {
        cudaMemsetAsync(n_out, 0, 4, st);
        cudaMemsetAsync(n_out64, 0, 8, st);
        return;
    }
    k_visible_counts<<<chunks, BIN_THREADS, 0, st>>>(cnt, S, chunk_counts);
    k_scan_block_sums<<<1, 1024, 0, st>>>(chunk_counts, (int)chunks, n_out, n_out64);
    k_compact_visible<<<chunks, BIN_THREADS, 0, st>>>(cnt, key, S, chunk_counts, ckey, cslot);
}

// Tile boundaries of the sorted pair keys: each thread takes four consecutive
// keys with one 16-byte load (the key buffers are 256-byte aligned), its
// neighbours' edge keys come from the adjacent lanes (or memory at warp
// edges).
__global__ void __launch_bounds__(256) k_tile_ranges(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ total,
                                                     uint32_t cap, uint2* __restrict__ ranges) {
    const uint32_t K = min(*total, cap);
    const uint32_t nq = (K + 3u) / 4u;
    const int lane = threadIdx.x & 31;
    const uint32_t stride = gridDim.x * blockDim.x;
    // uniform trip count per warp so the shuffles see every lane
    for (uint32_t q0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); q0 < nq; q0 += stride) {
        const uint32_t q = q0 + (uint32_t)lane;
        const uint32_t i = q * 4u;
        uint32_t k[4];
        if (i + 3u < K) {
            const uint4 v = *reinterpret_cast<const uint4*>(keys + i);
            k[0] = v.x; k[1] = v.y; k[2] = v.z; k[3] = v.w;
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) k[j] = i + (uint32_t)j < K ? keys[i + j] : 0xffffffffu;
        }
        uint32_t prev = __shfl_up_sync(0xffffffffu, k[3], 1);
        uint32_t next = __shfl_down_sync(0xffffffffu, k[0], 1);
        if (lane == 0 && i > 0 && i < K) prev = keys[i - 1];
        if (lane == 31 && i + 4u < K) next = keys[i + 4u];
        if (i < K) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t p = i + (uint32_t)j;
                if (p >= K) break;
                const uint32_t t = k[j];
                const uint32_t before = j == 0 ? prev : k[j - 1];
                const uint32_t after = j == 3 ? next : k[j + 1];
                if (p == 0 || before != t) ranges[t].x = p;
                if (p == K - 1 || after != t) ranges[t].y = p + 1;
            }
        }
    }
}

void launch_tile_ranges(const uint32_t* pair_keys, const uint32_t* total, uint32_t cap, uint2* ranges, cudaStream_t st) {
    k_tile_ranges<<<bin_grid_blocks() * 2, 256, 0, st>>>(pair_keys, total, cap, ranges);
}

}  // namespace rgs
