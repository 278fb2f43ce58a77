// densify.cu -- densification and pruning on the device.
//
// Follows src/pipeline/optimizer.rs:206-311 (`densify_and_prune`,
// `split_gaussian`, `clone_gaussian`):
//   prune  if sigmoid(logit) < prune_opacity_thresh or max scale > 0.1 * extent;
//   else, if the mean screen gradient >= threshold and N + (adds so far) <
//   max_gaussians: split (max scale > 0.01 * extent) into two children offset
//   by +-s0 along the rotated x axis, with log_scale[0] = ln(max(s0/sqrt2, 1e-6))
//   and opacity logit(clamp(0.8 sigma, 1e-6, 0.999)), removing the parent; or
//   clone with position.xy += 0.01 * mean gradient.
//   Survivors keep their order; new Gaussians are appended in parent order.
// The serial "adds so far" cap is a prefix condition: once N + adds >= cap it
// stays so, because a refused candidate adds nothing. So a scan of the uncapped
// adds decides every candidate at once. Three stream compactions (scans) then
// place survivors and children. The caller owns the Adam-moment policy.
#include "rgs_internal.cuh"
#include "rgs_math.cuh"

namespace rgs {

constexpr int DT = 256;

enum Kind : uint32_t { KEEP = 0, PRUNE = 1, SPLIT = 2, CLONE = 3 };

__global__ void k_densify_flags(DensifyArgs a, uint32_t* __restrict__ kind, unsigned long long* __restrict__ cand_adds) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    float4 p0 = a.params[i];
    float4 p2 = a.params[2 * (size_t)a.cap + i];
    uint32_t den = a.grad_denom[i];
    float avg = den > 0 ? a.grad_accum[i] / (float)den : 0.0f;
    float alpha = sigmoid(p0.w);
    float s0 = exp_cr(p2.x), s1 = exp_cr(p2.y), s2 = exp_cr(p2.z);
    float ms = fmaxf(fmaxf(s0, s1), s2);
    uint32_t k = KEEP;
    if (alpha < a.prune_opacity || ms > 0.1f * a.extent) k = PRUNE;
    else if (avg >= a.grad_threshold) k = ms > 0.01f * a.extent ? SPLIT : CLONE;
    kind[i] = k;
    cand_adds[i] = k == SPLIT ? 2ull : (k == CLONE ? 1ull : 0ull);
}

// Generic exclusive scan of u64 over n items: chunk sums, block-sum scan,
// chunk rescan. Fixed grid; the block-sum scan is one block.
__device__ __forceinline__ void d_chunk(int n, int G, int b, int& begin, int& end) {
    int chunk = (n + G - 1) / G;
    begin = min(chunk * b, n);
    end = min(begin + chunk, n);
}

__global__ void k_u64_chunk_sums(const unsigned long long* __restrict__ in, int n, unsigned long long* __restrict__ bs) {
    __shared__ unsigned long long s[DT];
    int begin, end;
    d_chunk(n, gridDim.x, blockIdx.x, begin, end);
    unsigned long long t = 0;
    for (int i = begin + threadIdx.x; i < end; i += DT) t += in[i];
    s[threadIdx.x] = t;
    __syncthreads();
    for (int o = DT / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) bs[blockIdx.x] = s[0];
}

__global__ void k_u64_scan_bs(unsigned long long* __restrict__ bs, int G, unsigned long long* __restrict__ total) {
    if (threadIdx.x != 0) return;
    unsigned long long run = 0;
    for (int b = 0; b < G; ++b) {
        unsigned long long v = bs[b];
        bs[b] = run;
        run += v;
    }
    *total = run;
}

__global__ void k_u64_chunk_scan(const unsigned long long* __restrict__ in, int n, const unsigned long long* __restrict__ bs,
                                 unsigned long long* __restrict__ out) {
    __shared__ unsigned long long s[DT];
    __shared__ unsigned long long s_base;
    int begin, end;
    d_chunk(n, gridDim.x, blockIdx.x, begin, end);
    if (threadIdx.x == 0) s_base = bs[blockIdx.x];
    __syncthreads();
    for (int b0 = begin; b0 < end; b0 += DT) {
        int i = b0 + threadIdx.x;
        unsigned long long v = i < end ? in[i] : 0ull;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < DT; o <<= 1) {
            unsigned long long t = threadIdx.x >= o ? s[threadIdx.x - o] : 0ull;
            __syncthreads();
            s[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < end) out[i] = s_base + s[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == DT - 1) s_base += s[DT - 1];
        __syncthreads();
    }
}

static void scan_u64(const unsigned long long* in, unsigned long long* out, int n, unsigned long long* bs, unsigned long long* total,
                     int G, cudaStream_t st) {
    k_u64_chunk_sums<<<G, DT, 0, st>>>(in, n, bs);
    k_u64_scan_bs<<<1, 32, 0, st>>>(bs, G, total);
    k_u64_chunk_scan<<<G, DT, 0, st>>>(in, n, bs, out);
}

// Resolve the max_gaussians cap and pack (keep, add) for the placement scan.
__global__ void k_densify_resolve(int n, uint64_t max_g, const uint32_t* __restrict__ kind,
                                  const unsigned long long* __restrict__ cand_excl, unsigned long long* __restrict__ packed) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t k = kind[i];
    unsigned long long keep = 1, add = 0;
    if (k == PRUNE) keep = 0;
    else if (k == SPLIT || k == CLONE) {
        bool ok = (unsigned long long)n + cand_excl[i] < (unsigned long long)max_g;
        if (ok) {
            if (k == SPLIT) { keep = 0; add = 2; }
            else add = 1;
        }
    }
    packed[i] = keep | (add << 32);
}

__global__ void k_densify_scatter(DensifyArgs a, const unsigned long long* __restrict__ packed,
                                  const unsigned long long* __restrict__ pos, const unsigned long long* __restrict__ totals,
                                  float4* __restrict__ out, int out_cap) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    unsigned long long pk = packed[i], ps = pos[i];
    uint32_t keep = (uint32_t)(pk & 0xffffffffull), add = (uint32_t)(pk >> 32);
    uint32_t kpos = (uint32_t)(ps & 0xffffffffull), apos = (uint32_t)(ps >> 32);
    uint32_t kept_total = (uint32_t)(totals[0] & 0xffffffffull);
    const size_t cap = (size_t)a.cap;
    if (keep) {
        for (int p = 0; p < NPL; ++p) out[(size_t)p * out_cap + kpos] = a.params[(size_t)p * cap + i];
    }
    if (!add) return;
    uint32_t dst = kept_total + apos;
    if (add == 1) {
        // clone_gaussian (optimizer.rs:303-311)
        uint32_t den = a.grad_denom[i];
        float avg = den > 0 ? a.grad_accum[i] / (float)den : 0.0f;
        float jitter = avg * 0.01f;
        for (int p = 0; p < NPL; ++p) {
            float4 v = a.params[(size_t)p * cap + i];
            if (p == 0) { v.x += jitter; v.y += jitter; }
            out[(size_t)p * out_cap + dst] = v;
        }
        return;
    }
    // split_gaussian (optimizer.rs:274-301)
    float4 p0 = a.params[i], p1 = a.params[cap + i], p2 = a.params[2 * cap + i];
    float q[4] = {p1.x, p1.y, p1.z, p1.w};
    float s0 = exp_cr(p2.x);
    M3 r = to_rotation_matrix(q);
    float ax0 = r.m[0][0] * s0, ax1 = r.m[1][0] * s0, ax2 = r.m[2][0] * s0;
    float nrm = sqrtf(ax0 * ax0 + ax1 * ax1 + ax2 * ax2);
    float o0 = ax0 / nrm * s0, o1 = ax1 / nrm * s0, o2 = ax2 / nrm * s0;
    const float SQRT_2 = 1.4142135623730951f;
    float ns = log_cr(fmaxf(s0 / SQRT_2, 1e-6f));
    float no = rclamp(sigmoid(p0.w) * 0.8f, 1e-6f, 0.999f);
    float nl = logit(no);
    for (int c = 0; c < 2; ++c) {
        float4 a0 = p0;
        if (c == 0) { a0.x += o0; a0.y += o1; a0.z += o2; }
        else { a0.x -= o0; a0.y -= o1; a0.z -= o2; }
        a0.w = nl;
        float4 a2 = p2;
        a2.x = ns;
        out[(size_t)dst + c] = a0;
        out[(size_t)out_cap + dst + c] = p1;
        out[2 * (size_t)out_cap + dst + c] = a2;
        for (int p = 3; p < NPL; ++p) out[(size_t)p * out_cap + dst + c] = a.params[(size_t)p * cap + i];
    }
}

// Scratch layout inside `scratch`: kind[n] u32 | cand[n] u64 | cand_excl[n] u64 |
// packed[n] u64 | pos[n] u64 | bs[G] u64 | totals[2] u64.
cudaError_t densify_and_prune(const DensifyArgs& a, DBuf& outbuf, int* out_cap_io, DBuf& scratch, int* n_out, cudaStream_t st) {
    int n = a.n;
    *n_out = 0;
    if (n <= 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int G = sms;
    size_t need = (size_t)n * 4 + 16 + (size_t)n * 8 * 4 + (size_t)G * 8 + 64;
    cudaError_t e = scratch.ensure(need);
    if (e != cudaSuccess) return e;
    char* base = scratch.as<char>();
    uint32_t* kind = (uint32_t*)base;
    size_t off = ((size_t)n * 4 + 15) & ~(size_t)15;
    unsigned long long* cand = (unsigned long long*)(base + off); off += (size_t)n * 8;
    unsigned long long* cand_excl = (unsigned long long*)(base + off); off += (size_t)n * 8;
    unsigned long long* packed = (unsigned long long*)(base + off); off += (size_t)n * 8;
    unsigned long long* pos = (unsigned long long*)(base + off); off += (size_t)n * 8;
    unsigned long long* bs = (unsigned long long*)(base + off); off += (size_t)G * 8;
    unsigned long long* totals = (unsigned long long*)(base + off);
    int blocks = (n + DT - 1) / DT;
    k_densify_flags<<<blocks, DT, 0, st>>>(a, kind, cand);
    scan_u64(cand, cand_excl, n, bs, totals + 1, G, st);
    k_densify_resolve<<<blocks, DT, 0, st>>>(n, a.max_gaussians, kind, cand_excl, packed);
    scan_u64(packed, pos, n, bs, totals, G, st);
    unsigned long long tot = 0;
    if ((e = cudaMemcpyAsync(&tot, totals, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    uint64_t kept = tot & 0xffffffffull, added = tot >> 32;
    uint64_t n_new = kept + added;
    int out_cap = (int)(n_new + n_new / 4 + 64);
    if ((e = outbuf.ensure((size_t)out_cap * NPL * sizeof(float4))) != cudaSuccess) return e;
    *out_cap_io = out_cap;
    k_densify_scatter<<<blocks, DT, 0, st>>>(a, packed, pos, totals, outbuf.as<float4>(), out_cap);
    *n_out = (int)(kept + added);
    return cudaGetLastError();
}

}  // namespace rgs
