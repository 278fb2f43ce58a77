// sort.cu -- stable LSD radix sort of (u32 key, u32 value) pairs.
//
// Replaces the reference's serial `sort_unstable_by` on depth plus the serial
// per-tile push loop (src/cpu/backward.rs:190-205). Stability is what makes
// the result deterministic: inputs arrive in slot order, so equal keys keep
// index order, which is the (tile, depth bits, index) order the oracle uses.
//
// Each pass is reduce-then-scan with a fixed grid (no inter-block waiting):
// every block owns one contiguous chunk of the input.
//   upsweep:   per-block digit histogram of its chunk          -> hist[b][d]
//   scan:      one block turns hist into global offsets (digit-major order)
//   downsweep: each block walks its chunk in 2048-key sub-tiles, ranks keys
//              stably (warp match_any + per-warp counters), reorders the
//              sub-tile in shared memory by digit and writes it out with
//              consecutive threads hitting consecutive addresses. The next
//              full sub-tile's keys and values arrive meanwhile by bulk copy
//              (cp.async.bulk into the other of two shared-memory stages,
//              completion on an mbarrier), so the block never waits on a
//              global load; the stage that received a sub-tile then holds it
//              reordered. The only wait is on the block's own copies, with an
//              iteration limit: on expiry the block flags *fault, waits
//              (bounded) for its copies in flight and stops.
// The element count may live in device memory (pair counts are produced on
// the GPU), so the whole sort can be captured in a CUDA graph.
#include "rgs_internal.cuh"

namespace rgs {

constexpr int SORT_THREADS = 256;
constexpr int SORT_WARPS = SORT_THREADS / 32;
constexpr int SORT_IPT = 8;
constexpr int SORT_TILE = SORT_THREADS * SORT_IPT;

__device__ __forceinline__ uint32_t load_n(const uint32_t* n_dev, uint32_t n_host) { return n_dev ? *n_dev : n_host; }

__device__ __forceinline__ void chunk_of(uint32_t n, int G, int b, uint32_t& begin, uint32_t& end) {
    uint32_t chunk = (uint32_t)(((uint64_t)n + G - 1) / G);
    chunk = (chunk + 31u) & ~31u;
    uint64_t bg = (uint64_t)chunk * b;
    begin = (uint32_t)(bg < (uint64_t)n ? bg : (uint64_t)n);
    end = (uint32_t)(bg + chunk < (uint64_t)n ? bg + chunk : (uint64_t)n);
}

template <int BITS>
__global__ void __launch_bounds__(SORT_THREADS) k_upsweep(const uint32_t* __restrict__ keys, const uint32_t* n_dev,
                                                          uint32_t n_host, int shift, uint32_t* __restrict__ hist) {
    constexpr int R = 1 << BITS;
    __shared__ uint32_t s_h[SORT_WARPS][R];
    int tid = threadIdx.x, w = tid >> 5;
    for (int i = tid; i < SORT_WARPS * R; i += SORT_THREADS) (&s_h[0][0])[i] = 0;
    __syncthreads();
    uint32_t n = load_n(n_dev, n_host), begin, end;
    chunk_of(n, gridDim.x, blockIdx.x, begin, end);
    for (uint32_t p = begin + tid; p < end; p += SORT_THREADS) {
        uint32_t d = (keys[p] >> shift) & (R - 1);
        atomicAdd(&s_h[w][d], 1u);
    }
    __syncthreads();
    for (int d = tid; d < R; d += SORT_THREADS) {
        uint32_t s = 0;
#pragma unroll
        for (int k = 0; k < SORT_WARPS; ++k) s += s_h[k][d];
        hist[(size_t)d * gridDim.x + blockIdx.x] = s;  // digit-major: hist[d][b]
    }
}

// Block-wide exclusive scan of R values held D = R/256 per thread (consecutive).
template <int D>
__device__ __forceinline__ void block_exclusive_scan(uint32_t (&v)[D], uint32_t* s_warp, uint32_t& total) {
    int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) { uint32_t t = v[k]; v[k] = local; local += t; }
    uint32_t x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t t = lane < SORT_WARPS ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < SORT_WARPS) s_warp[lane] = t;
    }
    __syncthreads();
    uint32_t warp_prefix = w > 0 ? s_warp[w - 1] : 0;
    total = s_warp[SORT_WARPS - 1];
    uint32_t excl = warp_prefix + x - local;
#pragma unroll
    for (int k = 0; k < D; ++k) v[k] += excl;
    __syncthreads();
}

// Turns the digit-major histogram hist[d][b] into per-digit block offsets
// (exclusive over blocks b) and writes each digit's total to dtot[d]. One
// warp per digit: each lane loads its SCAN_PER consecutive-by-32 counts at
// once (no serial load latency), then the warp scans them chunk by chunk.
// The digit bases (an exclusive scan of the R totals) are formed by every
// downsweep CTA itself.
constexpr int SCAN_WARPS = 8;
constexpr int SCAN_PER = 32;  // G <= 32 * 32 blocks
template <int BITS>
__global__ void __launch_bounds__(SCAN_WARPS * 32) k_scan_hist(uint32_t* __restrict__ hist, uint32_t* __restrict__ dtot, int G) {
    constexpr int R = 1 << BITS;
    const int lane = threadIdx.x & 31;
    const int d = blockIdx.x * SCAN_WARPS + (threadIdx.x >> 5);
    if (d >= R) return;
    uint32_t* row = hist + (size_t)d * G;
    uint32_t v[SCAN_PER];
#pragma unroll
    for (int k = 0; k < SCAN_PER; ++k) {
        const int b = k * 32 + lane;
        v[k] = b < G ? row[b] : 0u;
    }
    uint32_t carry = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER; ++k) {
        if (k * 32 >= G) break;
        uint32_t x = v[k];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        const int b = k * 32 + lane;
        if (b < G) row[b] = carry + x - v[k];
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) dtot[d] = carry;
}

// ---- bulk-copy and mbarrier primitives (sm_90+ PTX) -----------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Orders this thread's generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) writes to the same memory.
__device__ __forceinline__ void proxy_async_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Untiled bulk copy global -> shared (both addresses 16-byte aligned, bytes a
// multiple of 16), completing bytes on the mbarrier. No multicast.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of an mbarrier (each try_wait suspends for
// a hardware-chosen slice): false once the limit is reached.
constexpr int SORT_WAIT_LIMIT = 1 << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (int i = 0; i < SORT_WAIT_LIMIT; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

template <int BITS>
__global__ void __launch_bounds__(SORT_THREADS) k_downsweep(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                            uint32_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                            const uint32_t* n_dev, uint32_t n_host, int shift,
                                                            const uint32_t* __restrict__ hist, const uint32_t* __restrict__ dtot,
                                                            int* __restrict__ fault) {
    constexpr int R = 1 << BITS;
    constexpr int D = R / SORT_THREADS;
    __shared__ uint32_t s_run[R];
    __shared__ uint32_t s_wcnt[SORT_WARPS][R];
    __shared__ uint32_t s_dstart[R];
    __shared__ uint32_t s_tot[R];
    __shared__ uint32_t s_warp[SORT_WARPS];
    // [stage][keys, values][position]: a stage receives a full sub-tile by bulk
    // copy, then holds that sub-tile reordered by digit
    __shared__ __align__(128) uint32_t s_stage[2][2][SORT_TILE];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ int s_ok;
    int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    uint32_t n = load_n(n_dev, n_host), begin, end;
    chunk_of(n, gridDim.x, blockIdx.x, begin, end);
    {
        // digit bases: exclusive scan of the digit totals, then this block's
        // offset within each digit
        uint32_t tb[D];
#pragma unroll
        for (int q = 0; q < D; ++q) tb[q] = dtot[tid * D + q];
        uint32_t all;
        block_exclusive_scan<D>(tb, s_warp, all);
#pragma unroll
        for (int q = 0; q < D; ++q) s_run[tid * D + q] = tb[q] + hist[(size_t)(tid * D + q) * gridDim.x + blockIdx.x];
    }
    // sub-tiles [begin, full_end) hold SORT_TILE keys each and come by bulk
    // copy (chunk starts are multiples of 32 keys: 128-byte aligned); a
    // shorter last sub-tile is loaded directly
    const uint32_t full_end = begin + (end - begin) / SORT_TILE * SORT_TILE;
    const bool bulk_ok = ((reinterpret_cast<uintptr_t>(kin) | reinterpret_cast<uintptr_t>(vin)) & 15u) == 0;
    const uint32_t bulk_end = bulk_ok ? full_end : begin;
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_init_fence();
        if (begin < bulk_end) {
            mbar_expect_tx(&s_bar[0], 2 * SORT_TILE * 4);
            bulk_copy_g2s(s_stage[0][0], kin + begin, SORT_TILE * 4, &s_bar[0]);
            bulk_copy_g2s(s_stage[0][1], vin + begin, SORT_TILE * 4, &s_bar[0]);
        }
    }
    __syncthreads();
    const uint32_t lt_mask = (1u << lane) - 1u;
    int it = 0;
    for (uint32_t base = begin; base < end; base += SORT_TILE, ++it) {
        const int stg = it & 1;
        const bool staged = base < bulk_end;  // block-uniform
        if (tid == 0 && base + SORT_TILE < bulk_end) {
            // the other stage was last read by the previous iteration, which
            // every thread fenced and left through a barrier
            mbar_expect_tx(&s_bar[stg ^ 1], 2 * SORT_TILE * 4);
            bulk_copy_g2s(s_stage[stg ^ 1][0], kin + base + SORT_TILE, SORT_TILE * 4, &s_bar[stg ^ 1]);
            bulk_copy_g2s(s_stage[stg ^ 1][1], vin + base + SORT_TILE, SORT_TILE * 4, &s_bar[stg ^ 1]);
        }
        for (int i = tid; i < SORT_WARPS * R; i += SORT_THREADS) (&s_wcnt[0][0])[i] = 0;
        if (staged && tid == 0) s_ok = mbar_wait_bounded(&s_bar[stg], (uint32_t)(it >> 1) & 1u) ? 1 : 0;
        __syncthreads();
        if (staged && !s_ok) {
            // the copy never completed: flag it, give this block's copies in
            // flight a bounded chance to land, and stop
            if (tid == 0) {
                atomicExch(fault, 1);
                mbar_wait_bounded(&s_bar[stg], (uint32_t)(it >> 1) & 1u);
                if (base + SORT_TILE < bulk_end) mbar_wait_bounded(&s_bar[stg ^ 1], (uint32_t)((it + 1) >> 1) & 1u);
            }
            return;
        }
        uint32_t k[SORT_IPT], v[SORT_IPT], rank[SORT_IPT];
        int dig[SORT_IPT];
#pragma unroll
        for (int i = 0; i < SORT_IPT; ++i) {
            const uint32_t local = (uint32_t)(w * 32 * SORT_IPT + i * 32 + lane);
            const uint32_t pos = base + local;
            const bool valid = pos < end;
            if (staged) {
                k[i] = s_stage[stg][0][local];
                v[i] = s_stage[stg][1][local];
            } else {
                k[i] = valid ? kin[pos] : 0u;
                v[i] = valid ? vin[pos] : 0u;
            }
            dig[i] = valid ? (int)((k[i] >> shift) & (R - 1)) : R;
        }
#pragma unroll
        for (int i = 0; i < SORT_IPT; ++i) {
            unsigned peers = __match_any_sync(0xffffffffu, dig[i]);
            int leader = __ffs(peers) - 1;
            uint32_t before = dig[i] < R ? s_wcnt[w][dig[i]] : 0u;
            __syncwarp();
            if (dig[i] < R && lane == leader) s_wcnt[w][dig[i]] = before + __popc(peers);
            __syncwarp();
            rank[i] = before + __popc(peers & lt_mask);
        }
        __syncthreads();
        uint32_t tot[D];
#pragma unroll
        for (int q = 0; q < D; ++q) {
            int d = tid * D + q;
            uint32_t acc = 0;
#pragma unroll
            for (int ww = 0; ww < SORT_WARPS; ++ww) {
                uint32_t c = s_wcnt[ww][d];
                s_wcnt[ww][d] = acc;
                acc += c;
            }
            tot[q] = acc;
            s_tot[d] = acc;
        }
        uint32_t total;
        block_exclusive_scan<D>(tot, s_warp, total);
#pragma unroll
        for (int q = 0; q < D; ++q) s_dstart[tid * D + q] = tot[q];
        __syncthreads();
        // every thread has read this stage's keys into registers (barriers
        // above): reorder the sub-tile into the same stage
#pragma unroll
        for (int i = 0; i < SORT_IPT; ++i) {
            if (dig[i] < R) {
                uint32_t lp = s_dstart[dig[i]] + s_wcnt[w][dig[i]] + rank[i];
                s_stage[stg][0][lp] = k[i];
                s_stage[stg][1][lp] = v[i];
            }
        }
        __syncthreads();
        uint32_t cnt = min((uint32_t)SORT_TILE, end - base);
        for (uint32_t j = tid; j < cnt; j += SORT_THREADS) {
            uint32_t key = s_stage[stg][0][j];
            uint32_t d = (key >> shift) & (R - 1);
            uint32_t g = s_run[d] + (j - s_dstart[d]);
            kout[g] = key;
            vout[g] = s_stage[stg][1][j];
        }
        proxy_async_fence();  // before this stage is refilled by bulk copy
        __syncthreads();
        for (int d = tid; d < R; d += SORT_THREADS) s_run[d] += s_tot[d];
        __syncthreads();
    }
}

int sort_grid_blocks() { return device_sm_count() * 4; }

int radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n_host, const uint32_t* n_dev, int bits, SortScratch& sc,
                     int grid, cudaStream_t st, cudaError_t* err) {
    *err = cudaSuccess;
    if (bits <= 0) return 0;
    size_t cap = n_host;
    if ((*err = sc.keys2.ensure(cap * 4 + 16)) != cudaSuccess) return 0;
    if ((*err = sc.vals2.ensure(cap * 4 + 16)) != cudaSuccess) return 0;
    if ((*err = sc.hist.ensure(sort_hist_bytes(grid))) != cudaSuccess) return 0;
    if (!sc.fault) {
        *err = cudaErrorInvalidValue;  // the owner provides the fault word
        return 0;
    }
    if (grid > 32 * SCAN_PER) {
        *err = cudaErrorInvalidValue;
        return 0;
    }
    uint32_t* k[2] = {keys, sc.keys2.as<uint32_t>()};
    uint32_t* v[2] = {vals, sc.vals2.as<uint32_t>()};
    int cur = 0;
    int shift = 0;
    // 8-bit digits; a final pass over fewer significant bits still reads 8
    // (the bits above `bits` are zero in every key, so they do not reorder).
    while (shift < bits) {
        uint32_t* hist = sc.hist.as<uint32_t>();
        uint32_t* dtot = hist + (size_t)grid * 256;
        k_upsweep<8><<<grid, SORT_THREADS, 0, st>>>(k[cur], n_dev, n_host, shift, hist);
        k_scan_hist<8><<<256 / SCAN_WARPS, SCAN_WARPS * 32, 0, st>>>(hist, dtot, grid);
        k_downsweep<8><<<grid, SORT_THREADS, 0, st>>>(k[cur], v[cur], k[cur ^ 1], v[cur ^ 1], n_dev, n_host, shift, hist, dtot,
                                                     sc.fault);
        cur ^= 1;
        shift += 8;
    }
    *err = cudaGetLastError();
    return cur;
}

}  // namespace rgs
