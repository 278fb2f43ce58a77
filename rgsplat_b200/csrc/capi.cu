// capi.cu -- the C ABI (include/rgsplat.h): contexts, the stateless drop-ins
// for the reference's free functions, and the device-resident trainer with its
// plain (per-view launches) and batched (one launch per stage, CUDA graph per
// iteration) training steps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <filesystem>
#include <string>
#include <vector>

#include "../../include/rgsplat.h"
#include "../../include/rgsplat_debug.h"
#include "rgs_internal.cuh"

using namespace rgs;

namespace {

constexpr int LOSS_TILE = 32;
constexpr int MAX_VIEWS = 64;

struct Scene {
    int n = 0, cap = 0;
    DBuf params, grads, m1, m2, accum, denom;
    int mcap = 0;  // Gaussians the moment / accumulator buffers hold
    int mlen = 0;  // length of the reference's AdamState (grows only)
    uint64_t t = 0;
};

// Step header: uploaded to the device once per step (a graph memcpy node).
struct StepHdr {
    uint32_t total_tiles;
    uint32_t total_loss_blocks;
    float bc[2];
    uint32_t total_st;   // supertiles of the batch
    uint32_t pad[3];
    DevCam cams[MAX_VIEWS];
};

struct StepOut {
    uint32_t pairs;
    int overflow;
    uint32_t visible;
    uint32_t pad;
    float losses[MAX_VIEWS];
    unsigned long long pairs64;  // exact pair count (pairs saturates at 2^32 - 1)
    unsigned long long st_pairs64;  // (supertile, slot) entries of the batch
    int sort_fault;
    int pad2;
};

// Default of rgs_options.batch_pair_limit: a batched step whose (Gaussian,
// tile) pairs exceed it runs as consecutive view groups that each stay
// within it (pair buffers and sort scratch take 16 bytes per pair: 17 GB).
constexpr unsigned long long BATCH_PAIR_LIMIT = 1ull << 30;

enum {
    SC_PAIRS = 0,
    SC_OVERFLOW = 2,
    SC_WORK_F = 3,
    SC_WORK_B = 4,
    SC_FINITE = 5,
    SC_VISIBLE = 6,
    SC_FAULT = 7,    // sticky: a sort pass's staged copies timed out
    SC_PAIRS64 = 8,  // u64 over slots 8 and 9
    SC_NVIS64 = 10,  // u64 over slots 10 and 11: slots with tile pairs
    SC_NVIS = 12,    // the same, u32 (the depth sort's element count)
    SC_STPAIRS64 = 14,  // u64 over 14 and 15: (supertile, slot) entries
    SC_STPAIRS = 16,    // the same, saturated u32
    SC_STEFF = 17,      // entries held (the supertile sort's element count)
    SC_COUNT = 18
};

}  // namespace

struct rgs_ctx {
    rgs_options opt;
    int device = 0;
    int sms = 148;
    int sort_grid = 296;
    cudaStream_t st = nullptr;
    std::string err;
    Scene tr, sc;
    std::vector<rgs_camera> cams;
    std::vector<DBuf> targets;
    // per-step work buffers
    DBuf hdr;       // StepHdr (device)
    StepHdr* hdr_h = nullptr;  // pinned
    StepOut* out_h = nullptr;  // pinned
    DBuf outd;      // StepOut (device)
    DBuf rec, cnt, tdesc, spans, dkey, ids, acc, gv;
    DBuf ckey, cslot, chunk_counts;  // slots with tile pairs, compacted for the depth sort
    // supertile binning: per slot the supertile count and rectangle, per
    // entry the tile mask, per chunk of entries and tile position the counts,
    // per position the total, and the count scan's block sums
    DBuf st_cnt, st_desc, st_masks, st_chunks, st_planes, st_block_sums;
    DBuf gcache;  // per-Gaussian view-independent projection terms, [2][cap] float4
    DBuf pkeys, pvals;
    uint32_t pair_cap = 0;
    bool split_hint = false;  // the last batched step ran as view groups
    int batch_views = 0;      // views whose pixels the buffers hold from the last
                              // batched pass run as one group (0: none)
    DBuf ranges, rgb, final_t, last, dl, partials;
    DBuf scalars, block_sums, view_pairs;
    SortScratch sort;
    SfmScratch sfm;
    DBuf dens_scratch, dens_out, m_tmp;
    DBuf stage_a, stage_b, stage_c, stage_d, target_stage;
    DBuf tstore;  // store-all backward study only
    // batched-step graph
    cudaGraphExec_t gexec = nullptr;
    std::vector<uint64_t> g_key;
    rgs_stats stats{};
    MemCounter mem;  // device bytes held through this context's buffers
    cudaStream_t own_stream = nullptr;
    // host-target steps: targets copied on copy_st, the loss waits on ev_copy
    cudaStream_t copy_st = nullptr;
    cudaEvent_t ev_copy = nullptr;
    DBuf target_batch;
    // per-stage timing (boundaries 0..RGS_NUM_STAGES)
    bool prof = false;
    cudaEvent_t ev[RGS_NUM_STAGES + 1] = {};
    bool ev_marked[RGS_NUM_STAGES + 1] = {};
    bool graph_marked[RGS_NUM_STAGES + 1] = {};
    float stage_ms[RGS_NUM_STAGES] = {};
};

namespace {

int fail(rgs_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(rgs_ctx* c, cudaError_t e, const char* what) {
    int code = (e == cudaErrorMemoryAllocation) ? RGS_ERR_OOM : RGS_ERR_CUDA;
    cudaGetLastError();
    return fail(c, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                             \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

// Stage boundary i (0 = start, RGS_NUM_STAGES = end) of the step being issued.
void mark(rgs_ctx* ctx, int i) {
    if (!ctx->prof) return;
    // inside a stream capture only an "external" record becomes an event-record
    // node of the graph (a plain record is just a capture dependency)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(ctx->st, &cs);
    if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(ctx->ev[i], ctx->st, cudaEventRecordExternal);
    else cudaEventRecord(ctx->ev[i], ctx->st);
    ctx->ev_marked[i] = true;
}

// After the stream has drained: add the elapsed time of every stage whose two
// boundaries were recorded.
void prof_collect(rgs_ctx* ctx) {
    if (!ctx->prof) return;
    for (int i = 0; i < RGS_NUM_STAGES; ++i) {
        int j = i + 1;
        while (j <= RGS_NUM_STAGES && !ctx->ev_marked[j]) ++j;
        if (!ctx->ev_marked[i] || j > RGS_NUM_STAGES) continue;
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, ctx->ev[i], ctx->ev[j]) == cudaSuccess) ctx->stage_ms[i] += ms;
    }
    cudaGetLastError();
    for (int i = 0; i <= RGS_NUM_STAGES; ++i) ctx->ev_marked[i] = false;
}

// General 4x4 inverse by cofactors, in double (Camera::view_matrix inverts c2w,
// src/math/mod.rs:155-160).
bool invert4(const double m[16], double out[16]) {
    double inv[16];
    inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] + m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
    inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] - m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
    inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] + m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
    inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] - m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
    inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] - m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
    inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] + m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
    inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] - m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
    inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] + m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
    inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] + m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
    inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] - m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
    inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] + m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
    inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] - m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
    inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] - m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
    inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] + m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
    inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] - m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
    inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] + m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
    double det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
    if (det == 0.0 || det != det) return false;
    double id = 1.0 / det;
    for (int i = 0; i < 16; ++i) out[i] = inv[i] * id;
    return true;
}

int make_devcam(rgs_ctx* ctx, const rgs_camera& c, DevCam& d) {
    if (c.width == 0 || c.height == 0 || c.width > 65535 || c.height > 65535)
        return fail(ctx, RGS_ERR_INVALID_ARG, "camera size must be in [1, 65535]");
    double m[16], inv[16];
    for (int i = 0; i < 16; ++i) m[i] = (double)c.c2w[i];
    if (!invert4(m, inv)) return fail(ctx, RGS_ERR_SINGULAR_CAMERA, "c2w must be invertible");
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 4; ++k) d.view[r * 4 + k] = (float)inv[r * 4 + k];
    d.fx = c.fx; d.fy = c.fy; d.cx = c.cx; d.cy = c.cy;
    d.pos[0] = c.c2w[3]; d.pos[1] = c.c2w[7]; d.pos[2] = c.c2w[11];
    d.width = (int)c.width;
    d.height = (int)c.height;
    d.ref_tiles_x = (d.width + REF_TILE - 1) / REF_TILE;
    d.ref_tiles_y = (d.height + REF_TILE - 1) / REF_TILE;
    d.tiles_x = (d.width + ctx->opt.tile_w - 1) / ctx->opt.tile_w;
    d.tiles_y = (d.height + ctx->opt.tile_h - 1) / ctx->opt.tile_h;
    d.st_x = (d.tiles_x + ST_EDGE - 1) / ST_EDGE;
    d.st_base = 0;
    d.loss_bx = (d.width + LOSS_TILE - 1) / LOSS_TILE;
    d.tile_base = d.pix_base = d.loss_base = 0;
    d.target = nullptr;
    return RGS_OK;
}

// Lays out V views in one batch; returns (pixels, tiles, loss blocks).
// Supertiles of a batch whose views' st_base are assigned.
size_t batch_supertiles(const DevCam* d, int V) {
    if (V <= 0) return 0;
    const DevCam& c = d[V - 1];
    return (size_t)c.st_base + (size_t)c.st_x * ((c.tiles_y + ST_EDGE - 1) / ST_EDGE);
}

void assign_bases(DevCam* d, int V, size_t& px, size_t& tiles, size_t& lblocks) {
    px = tiles = lblocks = 0;
    size_t sts = 0;
    for (int v = 0; v < V; ++v) {
        d[v].st_base = (int)sts;
        sts += (size_t)d[v].st_x * ((d[v].tiles_y + ST_EDGE - 1) / ST_EDGE);
        d[v].tile_base = (int)tiles;
        d[v].pix_base = (int)px;
        d[v].loss_base = (int)lblocks;
        tiles += (size_t)d[v].tiles_x * d[v].tiles_y;
        px += (size_t)d[v].width * d[v].height;
        lblocks += (size_t)d[v].loss_bx * ((d[v].height + LOSS_TILE - 1) / LOSS_TILE);
    }
}

int bits_for(size_t n) {
    int b = 1;
    while (((size_t)1 << b) < n) ++b;
    return b;
}

void fill_lrs(const rgs_train_config& c, int compat, float lr[NPL * 4]) {
    for (int k = 0; k < NPL * 4; ++k) lr[k] = 0.0f;
    for (int f = 0; f < NP; ++f) {
        int p, l;
        record_to_plane(f, p, l);
        float v;
        if (f < 3) v = c.lr_position;
        else if (f == 3) v = c.lr_opacity;
        else if (f < 8) v = c.lr_rotation;
        else if (f < 11) v = c.lr_scale;
        else {
            int k = f - 11;  // sh index; flat gradient index is 11 + k
            bool dc = compat ? (k < 3) : (k == 0 || k == 16 || k == 32);
            v = dc ? c.lr_sh_dc : c.lr_sh_rest;
        }
        lr[p * 4 + l] = v;
    }
}

// compiler-rt __powisf2 (LLVM's lowering of f32::powi, optimizer.rs:125-126).
float powi_f(float a, int b) {
    bool recip = b < 0;
    float r = 1.0f;
    for (;;) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return recip ? 1.0f / r : r;
}

void adam_args(rgs_ctx* ctx, Scene& s, const rgs_train_config& cfg, AdamArgs& a) {
    a.params = s.params.as<float4>();
    a.m1 = s.m1.as<float4>();
    a.m2 = s.m2.as<float4>();
    a.grad_accum = s.accum.as<float>();
    a.grad_denom = s.denom.as<uint32_t>();
    fill_lrs(cfg, ctx->opt.reference_compat, a.lr);
    a.b1 = cfg.beta1;
    a.b2 = cfg.beta2;
    a.one_minus_b1 = 1.0f - cfg.beta1;
    a.one_minus_b2 = 1.0f - cfg.beta2;
    a.eps = cfg.eps;
    a.bc1 = 1.0f - powi_f(cfg.beta1, (int)s.t);
    a.bc2 = 1.0f - powi_f(cfg.beta2, (int)s.t);
    a.denom_inc = 1;
    a.skip_flag = nullptr;
    a.bc_dev = nullptr;
    a.mstride = s.mcap;
}

// Parameter buffers sized for n Gaussians; moments keep their contents.
int ensure_scene(rgs_ctx* ctx, Scene& s, int n, bool keep_params) {
    if (n <= s.cap && s.params.p) return RGS_OK;
    int cap = std::max(n + n / 8 + 64, 256);
    DBuf np;
    CK(np.ensure((size_t)cap * NPL * sizeof(float4)));
    if (keep_params && s.n > 0) {
        CK(cudaMemcpy2DAsync(np.p, (size_t)cap * sizeof(float4), s.params.p, (size_t)s.cap * sizeof(float4),
                             (size_t)s.n * sizeof(float4), NPL, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
    s.params.release();
    s.params = np;
    s.cap = cap;
    s.grads.release();
    CK(s.grads.ensure((size_t)cap * NPL * sizeof(float4)));
    return RGS_OK;
}

// Moment / statistics buffers hold at least `len` Gaussians (contents kept).
int ensure_moments(rgs_ctx* ctx, Scene& s, int len) {
    if (len <= s.mcap && s.m1.p) return RGS_OK;
    int mcap = std::max(len + len / 8 + 64, 256);
    DBuf n1, n2, na, nd;
    CK(n1.ensure((size_t)mcap * NPL * sizeof(float4)));
    CK(n2.ensure((size_t)mcap * NPL * sizeof(float4)));
    CK(na.ensure((size_t)mcap * sizeof(float)));
    CK(nd.ensure((size_t)mcap * sizeof(uint32_t)));
    CK(cudaMemsetAsync(n1.p, 0, (size_t)mcap * NPL * sizeof(float4), ctx->st));
    CK(cudaMemsetAsync(n2.p, 0, (size_t)mcap * NPL * sizeof(float4), ctx->st));
    CK(cudaMemsetAsync(na.p, 0, (size_t)mcap * sizeof(float), ctx->st));
    CK(cudaMemsetAsync(nd.p, 0, (size_t)mcap * sizeof(uint32_t), ctx->st));
    if (s.mcap > 0 && s.m1.p) {
        size_t keep = (size_t)s.mcap;
        CK(cudaMemcpy2DAsync(n1.p, (size_t)mcap * 16, s.m1.p, keep * 16, keep * 16, NPL, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpy2DAsync(n2.p, (size_t)mcap * 16, s.m2.p, keep * 16, keep * 16, NPL, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpyAsync(na.p, s.accum.p, keep * 4, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpyAsync(nd.p, s.denom.p, keep * 4, cudaMemcpyDeviceToDevice, ctx->st));
    }
    CK(cudaStreamSynchronize(ctx->st));
    s.m1.release(); s.m2.release(); s.accum.release(); s.denom.release();
    s.m1 = n1; s.m2 = n2; s.accum = na; s.denom = nd;
    s.mcap = mcap;
    return RGS_OK;
}

int upload_gaussians(rgs_ctx* ctx, Scene& s, const float* g, size_t n) {
    if (n > (size_t)0x3fffffff) return fail(ctx, RGS_ERR_INVALID_ARG, "too many Gaussians");
    int rc = ensure_scene(ctx, s, (int)n, false);
    if (rc) return rc;
    s.n = (int)n;
    if (n == 0) return RGS_OK;
    CK(ctx->stage_a.ensure(n * NP * sizeof(float)));
    CK(cudaMemcpyAsync(ctx->stage_a.p, g, n * NP * sizeof(float), cudaMemcpyHostToDevice, ctx->st));
    launch_aos_to_planes(ctx->stage_a.as<float>(), s.params.as<float4>(), (int)n, s.cap, ctx->st);
    CK(cudaGetLastError());
    return RGS_OK;
}

int check_finite(rgs_ctx* ctx, Scene& s) {
    if (s.n == 0) return RGS_OK;
    CK(ctx->scalars.ensure(SC_COUNT * 4));
    int* flag = ctx->scalars.as<int>() + SC_FINITE;
    CK(cudaMemsetAsync(flag, 0, 4, ctx->st));
    launch_check_finite(s.params.as<float4>(), s.n, s.cap, flag, ctx->st);
    int h = 0;
    CK(cudaMemcpyAsync(&h, flag, 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (h) return fail(ctx, RGS_ERR_NONFINITE, "a Gaussian parameter is NaN or infinite");
    return RGS_OK;
}

int ensure_work(rgs_ctx* ctx, size_t S, size_t px, size_t tiles, size_t lblocks, int V) {
    CK(ctx->rec.ensure(std::max<size_t>(S, 1) * 3 * sizeof(float4)));
    CK(ctx->acc.ensure(std::max<size_t>(S, 1) * 3 * sizeof(float4)));
    CK(ctx->gv.ensure(std::max<size_t>(S, 1) * 4 * sizeof(float4)));
    CK(ctx->cnt.ensure(std::max<size_t>(S, 1) * 4));
    CK(ctx->tdesc.ensure(std::max<size_t>(S, 1) * 8));
    CK(ctx->spans.ensure(std::max<size_t>(S, 1) * 32));
    CK(ctx->dkey.ensure(std::max<size_t>(S, 1) * 4));
    CK(ctx->ids.ensure(std::max<size_t>(S, 1) * 4));
    CK(ctx->ckey.ensure(std::max<size_t>(S, 1) * 4));
    CK(ctx->cslot.ensure(std::max<size_t>(S, 1) * 4));
    CK(ctx->chunk_counts.ensure(std::max<size_t>(compact_chunks(S), 1) * 8));
    CK(ctx->st_cnt.ensure(std::max<size_t>(S, 1) * 4));
    CK(ctx->st_desc.ensure(std::max<size_t>(S, 1) * 8));
    CK(ctx->st_planes.ensure(ST_TILES * 4));
    CK(ctx->st_block_sums.ensure((size_t)bin_grid_blocks() * 8 + 64));
    CK(ctx->ranges.ensure(std::max<size_t>(tiles, 1) * sizeof(uint2)));
    CK(ctx->rgb.ensure(px * 3 * 4));
    CK(ctx->final_t.ensure(px * 4));
    CK(ctx->last.ensure(px * 4));
    CK(ctx->dl.ensure(px * 3 * 4));
    CK(ctx->partials.ensure(std::max<size_t>(lblocks, 1) * 2 * 4));
    CK(ctx->scalars.ensure(SC_COUNT * 4));
    CK(ctx->block_sums.ensure((size_t)bin_grid_blocks() * 8 + 64));
    CK(ctx->view_pairs.ensure(MAX_VIEWS * 8));
    CK(ctx->hdr.ensure(sizeof(StepHdr)));
    CK(ctx->outd.ensure(sizeof(StepOut)));
    (void)V;
    // whatever runs next writes the pixel buffers
    ctx->batch_views = 0;
    return RGS_OK;
}

// The projection's per-Gaussian term cache for scene s (allocated outside
// any stream capture).
int ensure_gcache(rgs_ctx* ctx, const Scene& s) {
    CK(ctx->gcache.ensure((size_t)std::max(s.cap, 1) * 2 * sizeof(float4)));
    return RGS_OK;
}

int ensure_pairs(rgs_ctx* ctx, unsigned long long K) {
    if (K <= ctx->pair_cap && ctx->pkeys.p) return RGS_OK;
    if (K > 0xC0000000ull) return fail(ctx, RGS_ERR_CAPACITY, "more than 3 * 2^30 (Gaussian, tile) pairs in one view");
    unsigned long long cap = std::max<unsigned long long>(K + K / 4 + 1024, 1 << 16);
    cap = std::min<unsigned long long>(cap, 0xF0000000ull);
    ctx->pkeys.release();
    ctx->pvals.release();
    ctx->st_masks.release();
    ctx->st_chunks.release();
    CK(ctx->pkeys.ensure(cap * 4));
    CK(ctx->pvals.ensure(cap * 4));
    CK(ctx->st_masks.ensure(cap * 2));
    CK(ctx->st_chunks.ensure(supertile_chunks(cap) * ST_TILES * 4));
    ctx->pair_cap = (uint32_t)cap;
    return RGS_OK;
}

struct Binned {
    const uint32_t* keys;
    const uint32_t* vals;
};

// Projection + depth sort + pair emission + tile sort + ranges for one batch.
// `k_host` >= 0 means the pair count was read back (plain path).
// prune: tile lists hold only the (tile, splat) pairs the blend's own tile
// test keeps (exact: the blend drops the others from every batch anyway).
// Only valid with a zero background, where a pixel whose reference tile list
// is empty renders the same 0 as one whose splats all miss it.
int bin_batch(rgs_ctx* ctx, Scene& s, const DevCam* cams_dev, int V, size_t tiles, bool host_count, Binned& out,
              bool project = true, bool prune = false, size_t st_cap = 0) {
    // supertiles the buffers and scans cover: the batch's own unless the
    // caller (a captured graph replayed for other views) gives a bound
    if (!st_cap) st_cap = std::max<size_t>(ctx->hdr_h->total_st, 1);
    cudaStream_t st = ctx->st;
    const size_t S = (size_t)s.n * V;
    uint32_t* sc = ctx->scalars.as<uint32_t>();
    if (project) {
        cudaMemsetAsync(sc + SC_VISIBLE, 0, 4, st);
        launch_project(s.params.as<float4>(), s.n, s.cap, cams_dev, V, ctx->opt.tile_w, ctx->opt.tile_h,
                       ctx->rec.as<float4>(), ctx->cnt.as<uint32_t>(), ctx->tdesc.as<uint2>(), ctx->dkey.as<uint32_t>(),
                       ctx->ids.as<uint32_t>(), prune ? 1 : 0, sc + SC_VISIBLE, ctx->gcache.as<float4>(), ctx->spans.as<uint4>(), st);
    }
    mark(ctx, 1);
    // only the slots with tile pairs go through the depth sort, gathered in
    // slot order (the stable sort then still breaks depth ties by index);
    // the gather also writes each slot's supertile rectangle and count
    launch_compact_visible(ctx->cnt.as<uint32_t>(), ctx->dkey.as<uint32_t>(), (uint32_t)S,
                           ctx->chunk_counts.as<unsigned long long>(), ctx->ckey.as<uint32_t>(), ctx->cslot.as<uint32_t>(),
                           sc + SC_NVIS, (unsigned long long*)(sc + SC_NVIS64), ctx->tdesc.as<uint2>(), cams_dev,
                           (uint32_t)s.n, ctx->st_cnt.as<uint32_t>(), ctx->st_desc.as<uint2>(), st);
    const uint32_t* nvis = sc + SC_NVIS;
    cudaError_t e;
    int which = radix_sort_pairs(ctx->ckey.as<uint32_t>(), ctx->cslot.as<uint32_t>(), (uint32_t)S, nvis, 32, ctx->sort,
                                 ctx->sort_grid, st, &e);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "depth sort");
    mark(ctx, 2);
    const uint32_t* order = which ? ctx->sort.vals2.as<uint32_t>() : ctx->cslot.as<uint32_t>();
    // (tile, slot) pairs of the batch, and (supertile, slot) entries
    launch_count_scan(order, ctx->cnt.as<uint32_t>(), (uint32_t)S, nvis, ctx->block_sums.as<unsigned long long>(),
                      sc + SC_PAIRS, (unsigned long long*)(sc + SC_PAIRS64), bin_grid_blocks(), st);
    launch_count_scan(order, ctx->st_cnt.as<uint32_t>(), (uint32_t)S, nvis, ctx->st_block_sums.as<unsigned long long>(),
                      sc + SC_STPAIRS, (unsigned long long*)(sc + SC_STPAIRS64), bin_grid_blocks(), st);
    if (host_count) {
        unsigned long long K = 0, KS = 0;
        uint32_t vis = 0;
        int fault = 0;
        CK(cudaMemcpyAsync(&K, sc + SC_PAIRS64, 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&KS, sc + SC_STPAIRS64, 8, cudaMemcpyDeviceToHost, st));
        if (project) CK(cudaMemcpyAsync(&vis, sc + SC_VISIBLE, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&fault, sc + SC_FAULT, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (fault) return fail(ctx, RGS_ERR_CUDA, "a sort pass's staged copies timed out");
        ctx->stats.visible += vis;
        int rc = ensure_pairs(ctx, std::max(K, KS));
        if (rc) return rc;
        ctx->stats.pairs += K;
        ctx->stats.supertile_entries += KS;
        // the depth order may live in the sort scratch: size it for the
        // supertile sort now, while nothing is in flight, so that sort never
        // reallocates it
        size_t need = std::max<size_t>(S, ctx->pair_cap) * 4 + 16;
        if (ctx->sort.keys2.bytes < need || ctx->sort.vals2.bytes < need) {
            std::vector<uint32_t> tmp;
            if (order == ctx->sort.vals2.as<uint32_t>()) {
                tmp.resize(S);
                CK(cudaMemcpyAsync(tmp.data(), order, S * 4, cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
            }
            CK(ctx->sort.keys2.ensure(need));
            CK(ctx->sort.vals2.ensure(need));
            if (!tmp.empty()) {
                CK(cudaMemcpyAsync(ctx->sort.vals2.p, tmp.data(), S * 4, cudaMemcpyHostToDevice, st));
                CK(cudaStreamSynchronize(st));
                order = ctx->sort.vals2.as<uint32_t>();
            }
        }
    }
    CK(cudaMemsetAsync(sc + SC_OVERFLOW, 0, 4, st));
    launch_emit_supertiles(order, ctx->st_desc.as<uint2>(), (uint32_t)S, nvis, ctx->st_block_sums.as<unsigned long long>(),
                           ctx->pkeys.as<uint32_t>(), ctx->pvals.as<uint32_t>(), ctx->pair_cap, (int*)(sc + SC_OVERFLOW),
                           sc + SC_STPAIRS, sc + SC_STEFF, cams_dev, (uint32_t)s.n, bin_grid_blocks(), st);
    mark(ctx, 3);
    int which2 = radix_sort_pairs(ctx->pkeys.as<uint32_t>(), ctx->pvals.as<uint32_t>(), ctx->pair_cap, sc + SC_STEFF,
                                  bits_for(std::max<size_t>(st_cap, 2)), ctx->sort, ctx->sort_grid, st, &e);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "supertile sort");
    mark(ctx, 4);
    const uint32_t* ent_keys = which2 ? ctx->sort.keys2.as<uint32_t>() : ctx->pkeys.as<uint32_t>();
    const uint32_t* ent_slot = which2 ? ctx->sort.vals2.as<uint32_t>() : ctx->pvals.as<uint32_t>();
    uint32_t* lists = which2 ? ctx->pvals.as<uint32_t>() : ctx->sort.vals2.as<uint32_t>();
    // tiles no entry's supertile holds keep an empty range
    CK(cudaMemsetAsync(ctx->ranges.p, 0, std::max<size_t>(tiles, 1) * sizeof(uint2), st));
    SupertileArgs sa;
    sa.cams = cams_dev;
    sa.nviews = V;
    sa.ent_key = ent_keys;
    sa.ent_slot = ent_slot;
    sa.n_ent = sc + SC_STEFF;
    sa.tdesc = ctx->tdesc.as<uint2>();
    sa.spans = ctx->spans.as<uint4>();
    sa.rec = ctx->rec.as<float4>();
    sa.S = (uint32_t)S;
    sa.n_per_view = (uint32_t)s.n;
    sa.tile_w = ctx->opt.tile_w;
    sa.tile_h = ctx->opt.tile_h;
    sa.prune = prune ? 1 : 0;
    sa.masks = ctx->st_masks.as<uint16_t>();
    sa.chunk_cnt = ctx->st_chunks.as<uint32_t>();
    sa.chunk_stride = (uint32_t)supertile_chunks(ctx->pair_cap);
    sa.plane_tot = ctx->st_planes.as<uint32_t>();
    sa.vals_out = lists;
    sa.cap = ctx->pair_cap;
    sa.ranges = ctx->ranges.as<uint2>();
    sa.overflow = (int*)(sc + SC_OVERFLOW);
    launch_supertile_lists(sa, st);
    mark(ctx, 5);
    CK(cudaGetLastError());
    out.keys = nullptr;
    out.vals = lists;
    return RGS_OK;
}

BlendArgs blend_args(rgs_ctx* ctx, Scene& s, const DevCam* cams_dev, int V, const uint32_t* tiles_dev, size_t tiles,
                     const Binned& b, const float bg[3], bool fwd) {
    BlendArgs a;
    a.cams = cams_dev;
    a.nviews = V;
    a.total_tiles = tiles_dev;
    a.total_tiles_host = (int)tiles;
    a.ranges = ctx->ranges.as<uint2>();
    a.pair_vals = b.vals;
    a.rec = ctx->rec.as<float4>();
    a.n_per_view = (uint32_t)s.n;
    a.bg[0] = bg[0]; a.bg[1] = bg[1]; a.bg[2] = bg[2];
    a.rgb = ctx->rgb.as<float>();
    a.final_t = ctx->final_t.as<float>();
    a.last = ctx->last.as<int>();
    a.dl = ctx->dl.as<float>();
    a.acc = ctx->acc.as<float4>();
    a.work = ctx->scalars.as<uint32_t>() + (fwd ? SC_WORK_F : SC_WORK_B);
    a.rect_filter = 0;
    a.empty_tile_black = 1;
    a.pixels_per_thread = ctx->opt.pixels_per_thread;
    a.tstore = nullptr;
    a.bg_start = 0;
    a.one = 1.0f;
    return a;
}

bool zero_bg(const float bg[3]) { return bg[0] == 0.0f && bg[1] == 0.0f && bg[2] == 0.0f; }

// Uploads one view's camera header (plain path) and returns its device copy.
int upload_single_cam(rgs_ctx* ctx, const DevCam& d, DevCam** dev) {
    StepHdr* h = ctx->hdr_h;
    h->cams[0] = d;
    h->total_tiles = (uint32_t)(d.tiles_x * d.tiles_y);
    h->total_loss_blocks = (uint32_t)(d.loss_bx * ((d.height + LOSS_TILE - 1) / LOSS_TILE));
    h->total_st = (uint32_t)batch_supertiles(&d, 1);
    CK(cudaMemcpyAsync(ctx->hdr.p, h, sizeof(StepHdr), cudaMemcpyHostToDevice, ctx->st));
    *dev = (DevCam*)((char*)ctx->hdr.p + offsetof(StepHdr, cams));
    // the host header is reused by the next call: wait for the copy
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

// Differentiation study (rgs_render_and_backward_variant): which backward,
// and the blend-kernel times and blend-state bytes it measured.
struct BwdStudy {
    bool store_all = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t state_bytes = 0;
};

// Forward + loss + backward + geometry of one view (the plain path).
// grads: accumulate (v > 0) or overwrite into s.grads; loss_out may be null.
int run_view_plain(rgs_ctx* ctx, Scene& s, const DevCam& dc_in, const float* target_dev, const float bg[3], float lambda,
                   bool do_backward, bool accumulate, float* loss_out, float* rgb_host, BwdStudy* study = nullptr,
                   bool bg_start = false) {
    cudaStream_t st = ctx->st;
    DevCam dc = dc_in;
    dc.target = target_dev;
    size_t px, tiles, lb;
    assign_bases(&dc, 1, px, tiles, lb);
    int rc = ensure_work(ctx, (size_t)s.n, px, tiles, lb, 1);
    if (rc) return rc;
    DevCam* cams_dev;
    if ((rc = upload_single_cam(ctx, dc, &cams_dev))) return rc;
    if ((rc = ensure_gcache(ctx, s))) return rc;
    mark(ctx, 0);
    Binned b;
    if ((rc = bin_batch(ctx, s, cams_dev, 1, tiles, true, b, true, zero_bg(bg)))) return rc;
    BlendArgs fa = blend_args(ctx, s, cams_dev, 1, nullptr, tiles, b, bg, true);
    fa.bg_start = bg_start ? 1 : 0;
    if (study) {
        // blend state: final T + last contributor per pixel, plus (store-all)
        // T per (tile-list position, tile pixel)
        study->state_bytes = (uint64_t)px * 8;
        if (study->store_all) {
            const uint64_t need = (uint64_t)ctx->stats.pairs * (uint64_t)(REF_TILE * REF_TILE) * 4;
            CK(ctx->tstore.ensure(std::max<uint64_t>(need, 16)));
            study->state_bytes += need;
            fa.tstore = ctx->tstore.as<float>();
        }
        CK(cudaEventRecord(study->ev[0], st));
        if (study->store_all) launch_blend_store_all(fa, true, st);
        else launch_blend_forward(fa, ctx->opt.tile_w, ctx->opt.tile_h, ctx->opt.batch, st);
        CK(cudaEventRecord(study->ev[1], st));
    } else {
        launch_blend_forward(fa, ctx->opt.tile_w, ctx->opt.tile_h, ctx->opt.batch, st);
    }
    mark(ctx, 6);
    CK(cudaGetLastError());
    if (rgb_host) {
        int fault = 0;
        CK(cudaMemcpyAsync(rgb_host, ctx->rgb.p, px * 3 * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&fault, ctx->sort.fault, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (fault) return fail(ctx, RGS_ERR_CUDA, "a sort pass's staged copies timed out");
    }
    if (!do_backward) return RGS_OK;
    float* losses_dev = (float*)((char*)ctx->outd.p + offsetof(StepOut, losses));
    CK(launch_loss(cams_dev, 1, (int)lb, ctx->rgb.as<float>(), lambda, ctx->dl.as<float>(), ctx->partials.as<float>(),
                   losses_dev, nullptr, ctx->opt.exact_loss != 0, st));
    mark(ctx, 7);
    CK(cudaMemsetAsync(ctx->acc.p, 0, std::max<size_t>(s.n, 1) * 3 * sizeof(float4), st));
    BlendArgs ba = blend_args(ctx, s, cams_dev, 1, nullptr, tiles, b, bg, false);
    if (study) {
        ba.tstore = fa.tstore;
        CK(cudaEventRecord(study->ev[2], st));
        if (study->store_all) launch_blend_store_all(ba, false, st);
        else launch_blend_backward(ba, ctx->opt.tile_w, ctx->opt.tile_h, ctx->opt.batch, st);
        CK(cudaEventRecord(study->ev[3], st));
    } else {
        launch_blend_backward(ba, ctx->opt.tile_w, ctx->opt.tile_h, ctx->opt.batch, st);
    }
    mark(ctx, 8);
    launch_geometry(s.params.as<float4>(), s.n, s.cap, cams_dev, 1, ctx->cnt.as<uint32_t>(), ctx->acc.as<float4>(),
                    ctx->rec.as<float4>(), ctx->gcache.as<float4>(), ctx->gv.as<float4>(), s.grads.as<float4>(),
                    accumulate ? 1 : 0, st);
    mark(ctx, 9);
    CK(cudaGetLastError());
    if (loss_out) {
        int fault = 0;
        CK(cudaMemcpyAsync(loss_out, losses_dev, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&fault, ctx->sort.fault, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (fault) return fail(ctx, RGS_ERR_CUDA, "a sort pass's staged copies timed out");
        prof_collect(ctx);
    }
    return RGS_OK;
}

int check_ctx(rgs_ctx* ctx) {
    if (!ctx) return RGS_ERR_INVALID_ARG;
    t_mem = &ctx->mem;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
    return RGS_OK;
}

}  // namespace

// ===========================================================================
// context
// ===========================================================================
extern "C" {

void rgs_options_default(rgs_options* o) {
    if (!o) return;
    o->device = 0;
    o->tile_w = 16;
    o->tile_h = 16;
    o->batch = 256;
    o->reference_compat = 1;
    o->pixels_per_thread = 2;
    o->batch_pair_limit = 0;
    o->exact_loss = 0;
}

void rgs_train_config_default(rgs_train_config* c) {
    if (!c) return;
    c->num_iterations = 30000;
    c->lr_position = 0.00016f;
    c->lr_rotation = 0.001f;
    c->lr_scale = 0.005f;
    c->lr_opacity = 0.05f;
    c->lr_sh_dc = 0.0025f;
    c->lr_sh_rest = 0.000125f;
    c->beta1 = 0.9f;
    c->beta2 = 0.999f;
    c->eps = 1e-8f;
    c->densify_from_iter = 500;
    c->densify_until_iter = 15000;
    c->densify_grad_threshold = 0.0002f;
    c->opacity_reset_iter = 3000;
    c->prune_opacity_thresh = 0.005f;
    c->max_gaussians = 3000000;
}

int rgs_device_count(int* count) {
    if (!count) return RGS_ERR_INVALID_ARG;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    *count = e == cudaSuccess ? n : 0;
    return e == cudaSuccess ? RGS_OK : RGS_ERR_NO_DEVICE;
}

int rgs_create(const rgs_options* opts, rgs_ctx** out) {
    if (!out) return RGS_ERR_INVALID_ARG;
    *out = nullptr;
    rgs_options o;
    rgs_options_default(&o);
    if (opts) o = *opts;
    bool shape_ok = (o.tile_w == 16 && o.tile_h == 16) || (o.tile_w == 8 && o.tile_h == 32) || (o.tile_w == 32 && o.tile_h == 8);
    if (!shape_ok || (o.batch != 128 && o.batch != 256 && o.batch != 512)) return RGS_ERR_INVALID_ARG;
    if (o.pixels_per_thread != 1 && o.pixels_per_thread != 2) return RGS_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return RGS_ERR_NO_DEVICE;
    }
    if (o.device < 0 || o.device >= ndev) return RGS_ERR_INVALID_ARG;
    if (o.batch_pair_limit == 0) o.batch_pair_limit = BATCH_PAIR_LIMIT;
    rgs_ctx* ctx = new rgs_ctx();
    ctx->opt = o;
    ctx->device = o.device;
    t_mem = &ctx->mem;
    cudaError_t e = cudaSetDevice(o.device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, o.device);
    // one-time per-device kernel attributes, set here so that no later call
    // (possibly inside a stream capture) has to
    if (e == cudaSuccess) e = prepare_loss_kernel();
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    ctx->st = ctx->own_stream;
    if (e == cudaSuccess) e = cudaMallocHost((void**)&ctx->hdr_h, sizeof(StepHdr));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&ctx->out_h, sizeof(StepOut));
    // scalar words live for the context; SC_FAULT starts (and stays) clear
    // unless a sort pass's staged copies time out
    if (e == cudaSuccess) e = ctx->scalars.ensure(SC_COUNT * 4);
    if (e == cudaSuccess) e = cudaMemset(ctx->scalars.p, 0, SC_COUNT * 4);
    if (e != cudaSuccess) {
        cudaGetLastError();
        rgs_destroy(ctx);
        return e == cudaErrorMemoryAllocation ? RGS_ERR_OOM : RGS_ERR_CUDA;
    }
    std::memset(ctx->hdr_h, 0, sizeof(StepHdr));
    std::memset(ctx->out_h, 0, sizeof(StepOut));
    ctx->sort_grid = sort_grid_blocks();
    ctx->sort.fault = ctx->scalars.as<int>() + SC_FAULT;
    *out = ctx;
    return RGS_OK;
}

void rgs_destroy(rgs_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    t_mem = &ctx->mem;
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    Scene* ss[2] = {&ctx->tr, &ctx->sc};
    for (Scene* s : ss) {
        s->params.release(); s->grads.release(); s->m1.release(); s->m2.release(); s->accum.release(); s->denom.release();
    }
    for (auto& t : ctx->targets) t.release();
    DBuf* bufs[] = {&ctx->hdr, &ctx->outd, &ctx->rec, &ctx->cnt, &ctx->tdesc, &ctx->spans, &ctx->gcache, &ctx->dkey, &ctx->ids,
                    &ctx->ckey, &ctx->cslot, &ctx->chunk_counts, &ctx->st_cnt, &ctx->st_desc, &ctx->st_masks,
                    &ctx->st_chunks, &ctx->st_planes, &ctx->st_block_sums, &ctx->acc, &ctx->gv, &ctx->pkeys,
                    &ctx->pvals,
                    &ctx->ranges, &ctx->rgb, &ctx->final_t, &ctx->last, &ctx->dl, &ctx->partials, &ctx->scalars,
                    &ctx->block_sums, &ctx->view_pairs, &ctx->sort.hist, &ctx->sort.keys2, &ctx->sort.vals2, &ctx->dens_scratch,
                    &ctx->dens_out, &ctx->m_tmp, &ctx->stage_a, &ctx->stage_b, &ctx->stage_c, &ctx->stage_d,
                    &ctx->target_stage, &ctx->tstore};
    for (DBuf* b : bufs) b->release();
    ctx->sfm.release();
    if (ctx->hdr_h) cudaFreeHost(ctx->hdr_h);
    if (ctx->out_h) cudaFreeHost(ctx->out_h);
    for (int i = 0; i <= RGS_NUM_STAGES; ++i)
        if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
    if (ctx->copy_st) cudaStreamSynchronize(ctx->copy_st);
    ctx->target_batch.release();
    if (ctx->ev_copy) cudaEventDestroy(ctx->ev_copy);
    if (ctx->copy_st) cudaStreamDestroy(ctx->copy_st);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    t_mem = nullptr;
    delete ctx;
}

const char* rgs_last_error(const rgs_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int rgs_synchronize(rgs_ctx* ctx) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_set_stream(rgs_ctx* ctx, void* cuda_stream) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    ctx->st = cuda_stream ? (cudaStream_t)cuda_stream : ctx->own_stream;
    return RGS_OK;
}

int rgs_set_profiling(rgs_ctx* ctx, int on) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (on && !ctx->ev[0])
        for (int i = 0; i <= RGS_NUM_STAGES; ++i) CK(cudaEventCreate(&ctx->ev[i]));
    ctx->prof = on != 0;
    return RGS_OK;
}

int rgs_get_stage_times(rgs_ctx* ctx, float* ms_out, int reset) {
    if (!ctx) return RGS_ERR_INVALID_ARG;
    if (ms_out)
        for (int i = 0; i < RGS_NUM_STAGES; ++i) ms_out[i] = ctx->stage_ms[i];
    if (reset)
        for (int i = 0; i < RGS_NUM_STAGES; ++i) ctx->stage_ms[i] = 0.0f;
    return RGS_OK;
}

int rgs_get_memory(rgs_ctx* ctx, uint64_t* held_bytes, uint64_t* peak_bytes, int reset_peak) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (held_bytes) *held_bytes = ctx->mem.held;
    if (peak_bytes) *peak_bytes = ctx->mem.peak;
    if (reset_peak) ctx->mem.peak = ctx->mem.held;
    return RGS_OK;
}

int rgs_get_stats(rgs_ctx* ctx, rgs_stats* out) {
    if (!ctx || !out) return RGS_ERR_INVALID_ARG;
    *out = ctx->stats;
    out->pair_capacity = ctx->pair_cap;
    return RGS_OK;
}

// ===========================================================================
// stateless drop-ins
// ===========================================================================
int rgs_render_and_backward(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, const float* target_rgba,
                            const float bg[3], const rgs_loss_config* cfg, float* loss_out, float* grads_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!camera || !target_rgba || !bg || !cfg || (n && !gaussians)) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    DevCam dc;
    if ((rc = make_devcam(ctx, *camera, dc))) return rc;
    Scene& s = ctx->sc;
    if ((rc = upload_gaussians(ctx, s, gaussians, n))) return rc;
    if ((rc = check_finite(ctx, s))) return rc;
    size_t px = (size_t)camera->width * camera->height;
    CK(ctx->target_stage.ensure(px * 4 * 4));
    CK(cudaMemcpyAsync(ctx->target_stage.p, target_rgba, px * 16, cudaMemcpyHostToDevice, ctx->st));
    ctx->stats = rgs_stats{};
    float loss = 0.0f;
    if ((rc = run_view_plain(ctx, s, dc, ctx->target_stage.as<float>(), bg, cfg->lambda_dssim, true, false, &loss, nullptr)))
        return rc;
    if (loss_out) *loss_out = loss;
    if (grads_out && n) {
        CK(ctx->stage_b.ensure(n * NG * 4));
        launch_grads_to_aos(s.grads.as<float4>(), ctx->stage_b.as<float>(), (int)n, s.cap, NG, ctx->st);
        CK(cudaMemcpyAsync(grads_out, ctx->stage_b.p, n * NG * 4, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
    return RGS_OK;
}

int rgs_render_and_backward_variant(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera,
                                    const float* target_rgba, const float bg[3], const rgs_loss_config* cfg, int variant,
                                    float* loss_out, float* grads_out, rgs_backward_report* report) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!camera || !target_rgba || !bg || !cfg || (n && !gaussians)) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if (variant != RGS_BACKWARD_RECOMPUTE && variant != RGS_BACKWARD_STORE_ALL)
        return fail(ctx, RGS_ERR_INVALID_ARG, "unknown backward variant");
    if (variant == RGS_BACKWARD_STORE_ALL && !(ctx->opt.tile_w == REF_TILE && ctx->opt.tile_h == REF_TILE))
        return fail(ctx, RGS_ERR_INVALID_ARG, "the store-all backward needs 16x16 tiles");
    DevCam dc;
    if ((rc = make_devcam(ctx, *camera, dc))) return rc;
    Scene& s = ctx->sc;
    if ((rc = upload_gaussians(ctx, s, gaussians, n))) return rc;
    if ((rc = check_finite(ctx, s))) return rc;
    size_t px = (size_t)camera->width * camera->height;
    CK(ctx->target_stage.ensure(px * 4 * 4));
    CK(cudaMemcpyAsync(ctx->target_stage.p, target_rgba, px * 16, cudaMemcpyHostToDevice, ctx->st));
    ctx->stats = rgs_stats{};
    BwdStudy study;
    study.store_all = variant == RGS_BACKWARD_STORE_ALL;
    for (auto& e : study.ev) CK(cudaEventCreate(&e));
    float loss = 0.0f;
    rc = run_view_plain(ctx, s, dc, ctx->target_stage.as<float>(), bg, cfg->lambda_dssim, true, false, &loss, nullptr, &study);
    float fwd_ms = 0.0f, bwd_ms = 0.0f;
    if (rc == RGS_OK) {
        cudaError_t e = cudaEventElapsedTime(&fwd_ms, study.ev[0], study.ev[1]);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&bwd_ms, study.ev[2], study.ev[3]);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "variant timing");
    }
    for (auto& e : study.ev) cudaEventDestroy(e);
    if (rc) return rc;
    if (loss_out) *loss_out = loss;
    if (report) {
        report->forward_ms = fwd_ms;
        report->backward_ms = bwd_ms;
        report->state_bytes = study.state_bytes;
        report->pairs = ctx->stats.pairs;
    }
    if (grads_out && n) {
        CK(ctx->stage_b.ensure(n * NG * 4));
        launch_grads_to_aos(s.grads.as<float4>(), ctx->stage_b.as<float>(), (int)n, s.cap, NG, ctx->st);
        CK(cudaMemcpyAsync(grads_out, ctx->stage_b.p, n * NG * 4, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
    return RGS_OK;
}

int rgs_render_color(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, const float bg[3],
                     float* rgb_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!camera || !bg || !rgb_out || (n && !gaussians)) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    DevCam dc;
    if ((rc = make_devcam(ctx, *camera, dc))) return rc;
    Scene& s = ctx->sc;
    if ((rc = upload_gaussians(ctx, s, gaussians, n))) return rc;
    if ((rc = check_finite(ctx, s))) return rc;
    ctx->stats = rgs_stats{};
    return run_view_plain(ctx, s, dc, nullptr, bg, 0.0f, false, false, nullptr, rgb_out);
}

// cpu::rasterize of scene s for one camera into a host framebuffer.
int rasterize_scene(rgs_ctx* ctx, Scene& s, const rgs_camera* camera, const float bg[3], int format, void* out) {
    int rc;
    if (format != RGS_FB_RGBA_F32 && format != RGS_FB_RGBA8_SRGB) return fail(ctx, RGS_ERR_INVALID_ARG, "unknown framebuffer format");
    DevCam dc;
    if ((rc = make_devcam(ctx, *camera, dc))) return rc;
    ctx->stats = rgs_stats{};
    if ((rc = run_view_plain(ctx, s, dc, nullptr, bg, 0.0f, false, false, nullptr, nullptr, nullptr, true))) return rc;
    const size_t px = (size_t)camera->width * camera->height;
    const size_t bytes = px * (format == RGS_FB_RGBA8_SRGB ? 4 : 16);
    CK(ctx->stage_a.ensure(std::max<size_t>(bytes, 16)));
    launch_pack_framebuffer(ctx->rgb.as<float>(), ctx->final_t.as<float>(), px, format == RGS_FB_RGBA8_SRGB ? 1 : 0,
                            ctx->stage_a.p, ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, ctx->stage_a.p, bytes, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_rasterize(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, const float bg[3], int format,
                  void* out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!camera || !bg || !out || (n && !gaussians)) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    Scene& s = ctx->sc;
    if ((rc = upload_gaussians(ctx, s, gaussians, n))) return rc;
    if ((rc = check_finite(ctx, s))) return rc;
    return rasterize_scene(ctx, s, camera, bg, format, out);
}

int rgs_trainer_rasterize(rgs_ctx* ctx, uint32_t view, const float bg[3], int format, void* out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!bg || !out || view >= ctx->cams.size()) return fail(ctx, RGS_ERR_INVALID_ARG, "bad argument");
    return rasterize_scene(ctx, ctx->tr, &ctx->cams[view], bg, format, out);
}

int rgs_photometric_loss_grad(rgs_ctx* ctx, const float* rendered_rgb, const float* target_rgba, uint32_t width,
                              uint32_t height, float lambda, float* loss_out, float* dl_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!rendered_rgb || !target_rgba || !loss_out || !dl_out) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    rgs_camera cam{};
    cam.width = width;
    cam.height = height;
    cam.fx = cam.fy = 1.0f;
    for (int i = 0; i < 4; ++i) cam.c2w[i * 5] = 1.0f;
    DevCam dc;
    if ((rc = make_devcam(ctx, cam, dc))) return rc;
    size_t px, tiles, lb;
    assign_bases(&dc, 1, px, tiles, lb);
    if ((rc = ensure_work(ctx, 1, px, tiles, lb, 1))) return rc;
    CK(ctx->target_stage.ensure(px * 16));
    CK(cudaMemcpyAsync(ctx->target_stage.p, target_rgba, px * 16, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->rgb.p, rendered_rgb, px * 12, cudaMemcpyHostToDevice, ctx->st));
    dc.target = ctx->target_stage.as<float>();
    DevCam* cams_dev;
    if ((rc = upload_single_cam(ctx, dc, &cams_dev))) return rc;
    float* losses_dev = (float*)((char*)ctx->outd.p + offsetof(StepOut, losses));
    CK(launch_loss(cams_dev, 1, (int)lb, ctx->rgb.as<float>(), lambda, ctx->dl.as<float>(), ctx->partials.as<float>(),
                   losses_dev, nullptr, ctx->opt.exact_loss != 0, ctx->st));
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(loss_out, losses_dev, 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(dl_out, ctx->dl.p, px * 12, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_adam_step(rgs_ctx* ctx, float* gaussians, size_t n, const float* grads, rgs_adam_state* state,
                  const rgs_train_config* cfg) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!state || !cfg || (n && (!gaussians || !grads))) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if (state->len < n || (n && (!state->m1 || !state->m2 || !state->grad_accum || !state->grad_denom)))
        return fail(ctx, RGS_ERR_INVALID_ARG, "AdamState shorter than the Gaussian slice");
    Scene& s = ctx->sc;
    state->t += 1;
    if (n == 0) return RGS_OK;
    if ((rc = upload_gaussians(ctx, s, gaussians, n))) return rc;
    if ((rc = ensure_moments(ctx, s, (int)n))) return rc;
    cudaStream_t st = ctx->st;
    CK(ctx->stage_b.ensure(n * NG * 4));
    CK(cudaMemcpyAsync(ctx->stage_b.p, grads, n * NG * 4, cudaMemcpyHostToDevice, st));
    launch_aos_to_grad_planes(ctx->stage_b.as<float>(), s.grads.as<float4>(), (int)n, s.cap, NG, st);
    CK(ctx->stage_c.ensure(n * NP * 4));
    CK(ctx->stage_d.ensure(n * NP * 4));
    CK(cudaMemcpyAsync(ctx->stage_c.p, state->m1, n * NP * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->stage_d.p, state->m2, n * NP * 4, cudaMemcpyHostToDevice, st));
    launch_aos_to_grad_planes(ctx->stage_c.as<float>(), s.m1.as<float4>(), (int)n, s.mcap, NP, st);
    launch_aos_to_grad_planes(ctx->stage_d.as<float>(), s.m2.as<float4>(), (int)n, s.mcap, NP, st);
    CK(cudaMemcpyAsync(s.accum.p, state->grad_accum, n * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s.denom.p, state->grad_denom, n * 4, cudaMemcpyHostToDevice, st));
    s.t = state->t;
    AdamArgs a;
    adam_args(ctx, s, *cfg, a);
    a.denom_inc = 1;
    launch_adam((int)n, s.cap, s.grads.as<float4>(), a, st);
    CK(cudaGetLastError());
    launch_planes_to_aos(s.params.as<float4>(), ctx->stage_a.as<float>(), (int)n, s.cap, st);
    launch_grads_to_aos(s.m1.as<float4>(), ctx->stage_c.as<float>(), (int)n, s.mcap, NP, st);
    launch_grads_to_aos(s.m2.as<float4>(), ctx->stage_d.as<float>(), (int)n, s.mcap, NP, st);
    CK(cudaMemcpyAsync(gaussians, ctx->stage_a.p, n * NP * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(state->m1, ctx->stage_c.p, n * NP * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(state->m2, ctx->stage_d.p, n * NP * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(state->grad_accum, s.accum.p, n * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(state->grad_denom, s.denom.p, n * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return RGS_OK;
}

int rgs_densify_and_prune(rgs_ctx* ctx, const float* gaussians, size_t n, const float* grad_accum, const uint32_t* grad_denom,
                          const rgs_train_config* cfg, float scene_extent, float* out, size_t out_cap, size_t* n_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!cfg || !n_out || (n && (!gaussians || !grad_accum || !grad_denom))) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    *n_out = 0;
    if (n == 0) return RGS_OK;
    Scene& s = ctx->sc;
    if ((rc = upload_gaussians(ctx, s, gaussians, n))) return rc;
    if ((rc = ensure_moments(ctx, s, (int)n))) return rc;
    cudaStream_t st = ctx->st;
    CK(cudaMemcpyAsync(s.accum.p, grad_accum, n * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s.denom.p, grad_denom, n * 4, cudaMemcpyHostToDevice, st));
    DensifyArgs a;
    a.params = s.params.as<float4>();
    a.n = (int)n;
    a.cap = s.cap;
    a.grad_accum = s.accum.as<float>();
    a.grad_denom = s.denom.as<uint32_t>();
    a.prune_opacity = cfg->prune_opacity_thresh;
    a.grad_threshold = cfg->densify_grad_threshold;
    a.extent = scene_extent;
    a.max_gaussians = cfg->max_gaussians;
    int n_new = 0, ocap = 0;
    CK(densify_and_prune(a, ctx->dens_out, &ocap, ctx->dens_scratch, &n_new, st));
    *n_out = (size_t)n_new;
    if ((size_t)n_new > out_cap || (!out && n_new)) return fail(ctx, RGS_ERR_CAPACITY, "output buffer too small");
    CK(ctx->stage_a.ensure((size_t)n_new * NP * 4 + 4));
    launch_planes_to_aos(ctx->dens_out.as<float4>(), ctx->stage_a.as<float>(), n_new, ocap, st);
    CK(cudaMemcpyAsync(out, ctx->stage_a.p, (size_t)n_new * NP * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return RGS_OK;
}

int rgs_reset_opacities(rgs_ctx* ctx, float* gaussians, size_t n) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (n && !gaussians) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if (n == 0) return RGS_OK;
    Scene& s = ctx->sc;
    if ((rc = upload_gaussians(ctx, s, gaussians, n))) return rc;
    launch_reset_opacities(s.params.as<float4>(), (int)n, s.cap, ctx->st);
    launch_planes_to_aos(s.params.as<float4>(), ctx->stage_a.as<float>(), (int)n, s.cap, ctx->st);
    CK(cudaMemcpyAsync(gaussians, ctx->stage_a.p, n * NP * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_project(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, int mode, rgs_splat_info_2d* splats_out,
                uint32_t* keys_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!camera || (n && (!gaussians || !splats_out || !keys_out))) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if (mode != RGS_PROJECT_WGSL && mode != RGS_PROJECT_CPU_MATH) return fail(ctx, RGS_ERR_INVALID_ARG, "unknown mode");
    DevCam dc;
    if ((rc = make_devcam(ctx, *camera, dc))) return rc;
    if (n == 0) return RGS_OK;
    Scene& s = ctx->sc;
    if ((rc = upload_gaussians(ctx, s, gaussians, n))) return rc;
    if ((rc = ensure_work(ctx, 1, 1, 1, 1, 1))) return rc;
    DevCam* cams_dev;
    if ((rc = upload_single_cam(ctx, dc, &cams_dev))) return rc;
    CK(ctx->stage_b.ensure(n * 10 * 4));
    CK(ctx->stage_c.ensure(n * 4));
    launch_project_wgsl(s.params.as<float4>(), (int)n, s.cap, cams_dev, mode == RGS_PROJECT_CPU_MATH ? 1 : 0,
                        ctx->stage_b.as<float>(), ctx->stage_c.as<uint32_t>(), ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(splats_out, ctx->stage_b.p, n * 40, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(keys_out, ctx->stage_c.p, n * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_gpu_render(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, int mode, const float bg[3],
                   float* rgb_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!camera || !bg || !rgb_out || (n && !gaussians)) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if (mode != RGS_PROJECT_WGSL && mode != RGS_PROJECT_CPU_MATH) return fail(ctx, RGS_ERR_INVALID_ARG, "unknown mode");
    DevCam dc;
    if ((rc = make_devcam(ctx, *camera, dc))) return rc;
    Scene& s = ctx->sc;
    if ((rc = upload_gaussians(ctx, s, gaussians, n))) return rc;
    size_t px, tiles, lb;
    assign_bases(&dc, 1, px, tiles, lb);
    if ((rc = ensure_work(ctx, std::max<size_t>(n, 1), px, tiles, lb, 1))) return rc;
    DevCam* cams_dev;
    if ((rc = upload_single_cam(ctx, dc, &cams_dev))) return rc;
    CK(ctx->stage_b.ensure(std::max<size_t>(n, 1) * 40));
    CK(ctx->stage_c.ensure(std::max<size_t>(n, 1) * 4));
    launch_project_wgsl(s.params.as<float4>(), (int)n, s.cap, cams_dev, mode == RGS_PROJECT_CPU_MATH ? 1 : 0,
                        ctx->stage_b.as<float>(), ctx->stage_c.as<uint32_t>(), ctx->st);
    launch_composite_prepare(ctx->stage_b.as<float>(), (int)n, cams_dev, ctx->opt.tile_w, ctx->opt.tile_h,
                             ctx->rec.as<float4>(), ctx->cnt.as<uint32_t>(), ctx->tdesc.as<uint2>(), ctx->dkey.as<uint32_t>(),
                             ctx->ids.as<uint32_t>(),
                             ctx->st);
    Binned b;
    if ((rc = bin_batch(ctx, s, cams_dev, 1, tiles, true, b, false))) return rc;
    BlendArgs fa = blend_args(ctx, s, cams_dev, 1, nullptr, tiles, b, bg, true);
    fa.rect_filter = 1;
    fa.empty_tile_black = 0;
    launch_blend_forward(fa, ctx->opt.tile_w, ctx->opt.tile_h, ctx->opt.batch, ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(rgb_out, ctx->rgb.p, px * 12, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

// ===========================================================================
// device-resident trainer
// ===========================================================================
}  // extern "C"
namespace {
int fresh_adam_state(rgs_ctx* ctx, Scene& s);
}
extern "C" {

int rgs_trainer_set_gaussians(rgs_ctx* ctx, const float* gaussians, size_t n) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (n && !gaussians) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    Scene& s = ctx->tr;
    if ((rc = upload_gaussians(ctx, s, gaussians, n))) return rc;
    return fresh_adam_state(ctx, s);
}

int rgs_trainer_count(rgs_ctx* ctx, size_t* n) {
    if (!ctx || !n) return RGS_ERR_INVALID_ARG;
    *n = (size_t)ctx->tr.n;
    return RGS_OK;
}

int rgs_trainer_get_gaussians(rgs_ctx* ctx, float* out, size_t cap, size_t* n_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    Scene& s = ctx->tr;
    if (n_out) *n_out = (size_t)s.n;
    if ((size_t)s.n > cap || (s.n && !out)) return fail(ctx, RGS_ERR_CAPACITY, "output buffer too small");
    if (s.n == 0) return RGS_OK;
    CK(ctx->stage_a.ensure((size_t)s.n * NP * 4));
    launch_planes_to_aos(s.params.as<float4>(), ctx->stage_a.as<float>(), s.n, s.cap, ctx->st);
    CK(cudaMemcpyAsync(out, ctx->stage_a.p, (size_t)s.n * NP * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_trainer_set_cameras(rgs_ctx* ctx, const rgs_camera* cameras, size_t count) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (count && !cameras) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    for (size_t i = 0; i < count; ++i) {
        DevCam d;
        if ((rc = make_devcam(ctx, cameras[i], d))) return rc;
    }
    ctx->cams.assign(cameras, cameras + count);
    for (auto& t : ctx->targets) t.release();
    ctx->targets.clear();
    ctx->targets.resize(count);
    return RGS_OK;
}

int rgs_trainer_set_target(rgs_ctx* ctx, size_t index, const float* target_rgba) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (index >= ctx->cams.size() || !target_rgba) return fail(ctx, RGS_ERR_INVALID_ARG, "bad camera index or null target");
    size_t px = (size_t)ctx->cams[index].width * ctx->cams[index].height;
    CK(ctx->targets[index].ensure(px * 16));
    CK(cudaMemcpyAsync(ctx->targets[index].p, target_rgba, px * 16, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

}  // extern "C"

namespace {

// After new Gaussians arrived in s.params: reject non-finite ones and start
// from AdamState::new (zero moments, accumulators and step count).
int fresh_adam_state(rgs_ctx* ctx, Scene& s) {
    int rc = check_finite(ctx, s);
    if (rc) return rc;
    if ((rc = ensure_moments(ctx, s, std::max<int>(s.n, 1)))) return rc;
    CK(cudaMemsetAsync(s.m1.p, 0, (size_t)s.mcap * NPL * 16, ctx->st));
    CK(cudaMemsetAsync(s.m2.p, 0, (size_t)s.mcap * NPL * 16, ctx->st));
    CK(cudaMemsetAsync(s.accum.p, 0, (size_t)s.mcap * 4, ctx->st));
    CK(cudaMemsetAsync(s.denom.p, 0, (size_t)s.mcap * 4, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    s.mlen = s.n;
    s.t = 0;
    return RGS_OK;
}

// ---- io::ply (src/io/ply.rs): files <-> device planes -----------------------
int write_file(rgs_ctx* ctx, const char* path, const std::string& head, const void* body, size_t body_bytes) {
    // save_ply / save_splat create the parent directory first (ply.rs:36-38, 254-256)
    std::error_code ec;
    const std::filesystem::path fp(path);
    if (fp.has_parent_path()) std::filesystem::create_directories(fp.parent_path(), ec);
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(ctx, RGS_ERR_IO, std::string("creating ") + path);
    bool ok = head.empty() || std::fwrite(head.data(), 1, head.size(), f) == head.size();
    ok = ok && (body_bytes == 0 || std::fwrite(body, 1, body_bytes, f) == body_bytes);
    ok = (std::fclose(f) == 0) && ok;
    return ok ? RGS_OK : fail(ctx, RGS_ERR_IO, std::string("writing ") + path);
}

int read_file(rgs_ctx* ctx, const char* path, std::vector<uint8_t>& d) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(ctx, RGS_ERR_IO, std::string("opening ") + path);
    d.clear();
    uint8_t buf[1 << 16];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) d.insert(d.end(), buf, buf + got);
    const bool bad = std::ferror(f) != 0;
    std::fclose(f);
    return bad ? fail(ctx, RGS_ERR_IO, std::string("reading ") + path) : RGS_OK;
}

// The Gaussians of `s` -> the file of save_ply (ply == true) or save_splat.
int save_model(rgs_ctx* ctx, Scene& s, const char* path, bool ply) {
    const size_t n = (size_t)s.n;
    const size_t bytes = n * (ply ? 62 * 4 : 32);
    CK(ctx->stage_b.ensure(std::max<size_t>(bytes, 16)));
    if (ply) launch_pack_ply(s.params.as<float4>(), s.n, s.cap, ctx->stage_b.as<float>(), ctx->st);
    else launch_pack_splat(s.params.as<float4>(), s.n, s.cap, ctx->stage_b.p, ctx->st);
    CK(cudaGetLastError());
    std::vector<uint8_t> host(bytes);
    if (bytes) CK(cudaMemcpyAsync(host.data(), ctx->stage_b.p, bytes, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return write_file(ctx, path, ply ? ply_header(n) : std::string(), host.data(), bytes);
}

// A parsed PLY -> the planes of `s` (n = its vertex count).
int load_model(rgs_ctx* ctx, Scene& s, const std::vector<uint8_t>& d, const PlyLayout& L) {
    if (L.count > (size_t)0x3fffffff) return fail(ctx, RGS_ERR_INVALID_ARG, "too many vertices");
    if (L.format == 2) {
        std::vector<float> aos(std::max<size_t>(L.count, 1) * NP);
        decode_ply_ascii(d, L, aos.data());
        return upload_gaussians(ctx, s, aos.data(), L.count);
    }
    int rc = ensure_scene(ctx, s, (int)L.count, false);
    if (rc) return rc;
    s.n = (int)L.count;
    if (L.count == 0) return RGS_OK;
    const size_t body = L.count * L.stride;
    const size_t fbytes = L.fields.size() * sizeof(PlyField);
    CK(ctx->stage_c.ensure(std::max<size_t>(body, 16)));
    CK(ctx->stage_d.ensure(std::max<size_t>(fbytes, 16)));
    if (body) CK(cudaMemcpyAsync(ctx->stage_c.p, d.data() + L.body, body, cudaMemcpyHostToDevice, ctx->st));
    if (fbytes) CK(cudaMemcpyAsync(ctx->stage_d.p, L.fields.data(), fbytes, cudaMemcpyHostToDevice, ctx->st));
    launch_unpack_ply(ctx->stage_c.as<uint8_t>(), L.stride, (int)L.count, ctx->stage_d.as<PlyField>(), (int)L.fields.size(),
                      L.format == 1 ? 1 : 0, s.params.as<float4>(), s.cap, ctx->st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));  // the host file buffer is released by the caller
    return RGS_OK;
}

// gaussians_from_sfm into s.params (s.n = n).
int sfm_to_scene(rgs_ctx* ctx, Scene& s, const double* xyz, const uint8_t* rgb, size_t n) {
    if (n > (size_t)0x3fffffff) return fail(ctx, RGS_ERR_INVALID_ARG, "too many points");
    int rc = ensure_scene(ctx, s, (int)n, false);
    if (rc) return rc;
    s.n = (int)n;
    if (n == 0) return RGS_OK;
    SfmScratch& w = ctx->sfm;
    CK(w.xyz.ensure(n * 24));
    CK(w.rgb.ensure(n * 3 + 16));
    CK(cudaMemcpyAsync(w.xyz.p, xyz, n * 24, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(w.rgb.p, rgb, n * 3, cudaMemcpyHostToDevice, ctx->st));
    int bad = 0;
    cudaError_t e = cudaSuccess;
    sfm_init_planes(w.xyz.as<double>(), w.rgb.as<uint8_t>(), (int)n, s.params.as<float4>(), s.cap, w, sort_grid_blocks(),
                    ctx->st, &bad, &e);
    CK(e);
    if (bad) {
        s.n = 0;
        return fail(ctx, RGS_ERR_INVALID_ARG, "non-finite SfM point coordinate");
    }
    return RGS_OK;
}

// parse_points3d_bin (sfm.rs:147-183) over a file's bytes.
int parse_points3d(rgs_ctx* ctx, const std::vector<uint8_t>& d, std::vector<double>& xyz, std::vector<uint8_t>& rgb) {
    size_t at = 0;
    auto take = [&](void* dst, size_t k) {
        if (d.size() - at < k) return false;
        std::memcpy(dst, d.data() + at, k);
        at += k;
        return true;
    };
    uint64_t count = 0;
    if (!take(&count, 8)) return fail(ctx, RGS_ERR_FORMAT, "points3D.bin: no point count");
    xyz.clear();
    rgb.clear();
    for (uint64_t r = 0; r < count; ++r) {
        uint64_t id = 0, track = 0;
        double p[3], err = 0.0;
        uint8_t c[3];
        if (!take(&id, 8) || !take(p, 24) || !take(c, 3) || !take(&err, 8) || !take(&track, 8))
            return fail(ctx, RGS_ERR_FORMAT, "points3D.bin: record cut short");
        if (track > (d.size() - at) / 8) return fail(ctx, RGS_ERR_FORMAT, "points3D.bin: track cut short");
        at += (size_t)track * 8;
        xyz.insert(xyz.end(), p, p + 3);
        rgb.insert(rgb.end(), c, c + 3);
    }
    return RGS_OK;
}

int check_views(rgs_ctx* ctx, const uint32_t* views, size_t nviews, bool need_targets) {
    if (!views || nviews == 0) return fail(ctx, RGS_ERR_INVALID_ARG, "no views");
    if (nviews > (size_t)MAX_VIEWS) return fail(ctx, RGS_ERR_INVALID_ARG, "at most 64 views per step");
    for (size_t v = 0; v < nviews; ++v) {
        if (views[v] >= ctx->cams.size()) return fail(ctx, RGS_ERR_INVALID_ARG, "view index out of range");
        if (need_targets && !ctx->targets[views[v]].p) return fail(ctx, RGS_ERR_INVALID_ARG, "view has no target");
    }
    return RGS_OK;
}

// Plain path: per-view launch sequence with host-read pair counts; gradients
// of the views summed in ctx->tr.grads.
int plain_backward(rgs_ctx* ctx, const uint32_t* views, size_t nviews, const float bg[3], float lambda, float* losses) {
    Scene& s = ctx->tr;
    ctx->stats = rgs_stats{};
    for (size_t v = 0; v < nviews; ++v) {
        DevCam dc;
        int rc = make_devcam(ctx, ctx->cams[views[v]], dc);
        if (rc) return rc;
        float loss = 0.0f;
        rc = run_view_plain(ctx, s, dc, ctx->targets[views[v]].as<float>(), bg, lambda, true, v > 0, &loss, nullptr);
        if (rc) return rc;
        if (losses) losses[v] = loss;
    }
    return RGS_OK;
}

int apply_adam(rgs_ctx* ctx, const rgs_train_config& tc, uint32_t denom_inc) {
    Scene& s = ctx->tr;
    s.t += 1;
    if (s.n == 0) return RGS_OK;
    AdamArgs a;
    adam_args(ctx, s, tc, a);
    a.denom_inc = denom_inc;
    launch_adam(s.n, s.cap, s.grads.as<float4>(), a, ctx->st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

// Capacity of the batched buffers: every view at the largest camera size.
void batch_caps(rgs_ctx* ctx, int V, size_t& px, size_t& tiles, size_t& lb) {
    size_t mp = 0, mt = 0, ml = 0;
    for (const rgs_camera& c : ctx->cams) {
        size_t w = c.width, h = c.height;
        mp = std::max(mp, w * h);
        mt = std::max(mt, ((w + ctx->opt.tile_w - 1) / ctx->opt.tile_w) * ((h + ctx->opt.tile_h - 1) / ctx->opt.tile_h));
        ml = std::max(ml, ((w + LOSS_TILE - 1) / LOSS_TILE) * ((h + LOSS_TILE - 1) / LOSS_TILE));
    }
    px = mp * V;
    tiles = mt * V;
    lb = ml * V;
}

int capture_batched(rgs_ctx* ctx, int V, size_t tiles_cap, const float bg[3], float lambda, const rgs_train_config& tc,
                    bool fused, bool host_targets, int accumulate) {
    Scene& s = ctx->tr;
    cudaStream_t st = ctx->st;
    if (ctx->gexec) {
        cudaGraphExecDestroy(ctx->gexec);
        ctx->gexec = nullptr;
    }
    // size every scratch buffer before capture (no allocation inside it)
    size_t S = (size_t)s.n * V;
    CK(ctx->sort.keys2.ensure(std::max<size_t>(S, ctx->pair_cap) * 4 + 16));
    CK(ctx->sort.vals2.ensure(std::max<size_t>(S, ctx->pair_cap) * 4 + 16));
    CK(ctx->sort.hist.ensure(sort_hist_bytes(ctx->sort_grid)));
    StepHdr* hd = ctx->hdr.as<StepHdr>();
    const DevCam* cams_dev = (const DevCam*)((char*)ctx->hdr.p + offsetof(StepHdr, cams));
    float* losses_dev = (float*)((char*)ctx->outd.p + offsetof(StepOut, losses));
    uint32_t* sc = ctx->scalars.as<uint32_t>();
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(ctx->hdr.p, ctx->hdr_h, sizeof(StepHdr), cudaMemcpyHostToDevice, st);
    mark(ctx, 0);
    Binned b;
    // supertiles of any V views of this context (the graph is replayed for other view sets)
    size_t st_view_max = 1;
    for (const rgs_camera& cam : ctx->cams) {
        const size_t tx = (cam.width + ctx->opt.tile_w - 1) / ctx->opt.tile_w, ty = (cam.height + ctx->opt.tile_h - 1) / ctx->opt.tile_h;
        st_view_max = std::max(st_view_max, ((tx + ST_EDGE - 1) / ST_EDGE) * ((ty + ST_EDGE - 1) / ST_EDGE));
    }
    int rc = bin_batch(ctx, s, cams_dev, V, tiles_cap, false, b, true, zero_bg(bg), st_view_max * (size_t)V);
    if (!rc) {
        BlendArgs fa = blend_args(ctx, s, cams_dev, V, &hd->total_tiles, tiles_cap, b, bg, true);
        launch_blend_forward(fa, ctx->opt.tile_w, ctx->opt.tile_h, ctx->opt.batch, st);
        mark(ctx, 6);
        // the step's targets were copied from host memory on copy_st, issued
        // just before this graph's launch; only the loss waits for them
        if (host_targets) cudaStreamWaitEvent(st, ctx->ev_copy, cudaEventWaitExternal);
        cudaError_t le = launch_loss(cams_dev, V, 0, ctx->rgb.as<float>(), lambda, ctx->dl.as<float>(),
                                     ctx->partials.as<float>(), losses_dev, &hd->total_loss_blocks,
                                     ctx->opt.exact_loss != 0, st);
        if (le != cudaSuccess) rc = cuda_fail(ctx, le, "loss kernel launch");
        mark(ctx, 7);
        cudaMemsetAsync(ctx->acc.p, 0, std::max<size_t>(S, 1) * 3 * sizeof(float4), st);
        BlendArgs ba = blend_args(ctx, s, cams_dev, V, &hd->total_tiles, tiles_cap, b, bg, false);
        launch_blend_backward(ba, ctx->opt.tile_w, ctx->opt.tile_h, ctx->opt.batch, st);
        mark(ctx, 8);
        if (fused) {
            AdamArgs a;
            adam_args(ctx, s, tc, a);
            a.denom_inc = (uint32_t)V;
            a.skip_flag = (const int*)(sc + SC_OVERFLOW);
            a.bc_dev = hd->bc;
            launch_geometry_adam(cams_dev, V, s.n, s.cap, ctx->cnt.as<uint32_t>(), ctx->acc.as<float4>(),
                                 ctx->rec.as<float4>(), ctx->gcache.as<float4>(), ctx->gv.as<float4>(), a, st);
        } else {
            launch_geometry(s.params.as<float4>(), s.n, s.cap, cams_dev, V, ctx->cnt.as<uint32_t>(), ctx->acc.as<float4>(),
                            ctx->rec.as<float4>(), ctx->gcache.as<float4>(), ctx->gv.as<float4>(), s.grads.as<float4>(),
                            accumulate, st);
        }
        mark(ctx, 9);
        cudaMemcpyAsync(&ctx->out_h->pairs, sc + SC_PAIRS, 4, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&ctx->out_h->pairs64, sc + SC_PAIRS64, 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&ctx->out_h->st_pairs64, sc + SC_STPAIRS64, 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&ctx->out_h->sort_fault, sc + SC_FAULT, 4, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&ctx->out_h->overflow, sc + SC_OVERFLOW, 4, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&ctx->out_h->visible, sc + SC_VISIBLE, 4, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(ctx->out_h->losses, losses_dev, sizeof(float) * V, cudaMemcpyDeviceToHost, st);
    }
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "stream capture of the batched step");
    e = cudaGraphInstantiate(&ctx->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "graph instantiate");
    ctx->stats.graph_captures += 1;
    return RGS_OK;
}

// Batched path: one launch per stage over all views, replayed from a CUDA
// graph; the fused geometry-backward + Adam kernel ends the step.
int split_step(rgs_ctx* ctx, const uint32_t* views, int V, const float bg[3], float lambda, const rgs_train_config& tc,
               float* losses, bool fused, const float* const* host_targets);

int batched_step(rgs_ctx* ctx, const uint32_t* views, int V, const float bg[3], float lambda, const rgs_train_config& tc,
                 float* losses, bool fused, const float* const* host_targets = nullptr, int accumulate = 0,
                 bool allow_split = true) {
    Scene& s = ctx->tr;
    StepHdr* h = ctx->hdr_h;
    for (int v = 0; v < V; ++v) {
        int rc = make_devcam(ctx, ctx->cams[views[v]], h->cams[v]);
        if (rc) return rc;
        h->cams[v].target = ctx->targets[views[v]].as<float>();
    }
    size_t px, tiles, lb;
    assign_bases(h->cams, V, px, tiles, lb);
    h->total_tiles = (uint32_t)tiles;
    h->total_loss_blocks = (uint32_t)lb;
    h->total_st = (uint32_t)batch_supertiles(h->cams, V);
    size_t px_cap, tiles_cap, lb_cap;
    batch_caps(ctx, V, px_cap, tiles_cap, lb_cap);
    size_t S = (size_t)s.n * V;
    int rc = ensure_work(ctx, S, px_cap, tiles_cap, lb_cap, V);
    if (rc) return rc;
    if ((rc = ensure_gcache(ctx, s))) return rc;
    if (!ctx->pkeys.p && (rc = ensure_pairs(ctx, S * 4))) return rc;
    if ((rc = ensure_moments(ctx, s, s.n))) return rc;
    if (host_targets) {
        if (!ctx->copy_st) {
            CK(cudaStreamCreateWithFlags(&ctx->copy_st, cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&ctx->ev_copy, cudaEventDisableTiming));
        }
        // the previous step has finished (it synchronised), so the batch
        // target buffer is free to refill
        CK(ctx->target_batch.ensure(px_cap * 16));
        for (int v = 0; v < V; ++v) h->cams[v].target = ctx->target_batch.as<float>() + (size_t)h->cams[v].pix_base * 4;
    }
    if (ctx->split_hint && allow_split && V > 1) {
        // The last batched step ran as view groups: project this batch alone
        // first (no emission, no blend) and, if its pairs are again past the
        // budget, go to the groups directly instead of through a full attempt
        // that would overflow its pair buffer.
        const DevCam* cams_dev = (const DevCam*)((char*)ctx->hdr.p + offsetof(StepHdr, cams));
        uint32_t* sc = ctx->scalars.as<uint32_t>();
        CK(cudaMemcpyAsync(ctx->hdr.p, ctx->hdr_h, sizeof(StepHdr), cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemsetAsync(sc + SC_VISIBLE, 0, 4, ctx->st));
        launch_project(s.params.as<float4>(), s.n, s.cap, cams_dev, V, ctx->opt.tile_w, ctx->opt.tile_h, ctx->rec.as<float4>(),
                       ctx->cnt.as<uint32_t>(), ctx->tdesc.as<uint2>(), ctx->dkey.as<uint32_t>(), ctx->ids.as<uint32_t>(),
                       zero_bg(bg) ? 1 : 0, sc + SC_VISIBLE, ctx->gcache.as<float4>(), ctx->spans.as<uint4>(), ctx->st);
        launch_view_pairs(ctx->cnt.as<uint32_t>(), (uint32_t)s.n, V, ctx->view_pairs.as<unsigned long long>(), ctx->st);
        CK(cudaGetLastError());
        unsigned long long per[MAX_VIEWS], total = 0;
        CK(cudaMemcpyAsync(per, ctx->view_pairs.p, sizeof(unsigned long long) * V, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        for (int v = 0; v < V; ++v) total += per[v];
        if (total > ctx->opt.batch_pair_limit) return split_step(ctx, views, V, bg, lambda, tc, losses, fused, host_targets);
        ctx->split_hint = false;
    }
    const uint64_t tstep = fused ? 1 : 0;
    for (int attempt = 0; attempt < 4; ++attempt) {
        s.t += tstep;
        h->bc[0] = 1.0f - powi_f(tc.beta1, (int)s.t);
        h->bc[1] = 1.0f - powi_f(tc.beta2, (int)s.t);
        // Everything a captured graph bakes in: sizes, every buffer address, and
        // the loss weight, background and optimiser constants.
        const DBuf* bufs[] = {&s.params, &s.grads, &s.m1, &s.m2, &s.accum, &s.denom, &ctx->rec, &ctx->cnt, &ctx->tdesc, &ctx->spans, &ctx->gv, &ctx->gcache, &ctx->dkey,
                              &ctx->ids, &ctx->ckey, &ctx->cslot, &ctx->chunk_counts, &ctx->st_cnt, &ctx->st_desc,
                              &ctx->st_masks, &ctx->st_chunks, &ctx->st_planes, &ctx->st_block_sums,
                              &ctx->acc, &ctx->pkeys,
                              &ctx->pvals, &ctx->ranges, &ctx->rgb, &ctx->final_t,
                              &ctx->last, &ctx->dl, &ctx->partials, &ctx->scalars, &ctx->block_sums, &ctx->hdr, &ctx->outd,
                              &ctx->sort.hist, &ctx->sort.keys2, &ctx->sort.vals2};
        float fk[14] = {bg[0], bg[1], bg[2], lambda, tc.lr_position, tc.lr_rotation, tc.lr_scale, tc.lr_opacity,
                        tc.lr_sh_dc, tc.lr_sh_rest, tc.beta1, tc.beta2, tc.eps, (float)ctx->opt.reference_compat};
        auto make_key = [&]() {
            std::vector<uint64_t> key = {(uint64_t)s.n, (uint64_t)s.cap, (uint64_t)V, (uint64_t)s.mcap, ctx->pair_cap,
                                         px_cap, tiles_cap, lb_cap, (uint64_t)fused, (uint64_t)ctx->prof,
                                         (uint64_t)(uintptr_t)ctx->st, (uint64_t)ctx->opt.tile_w,
                                         (uint64_t)ctx->opt.tile_h, (uint64_t)ctx->opt.batch,
                                         (uint64_t)ctx->opt.pixels_per_thread, (uint64_t)(host_targets != nullptr),
                                         (uint64_t)accumulate};
            for (const DBuf* b : bufs) key.push_back((uint64_t)(uintptr_t)b->p);
            for (float f : fk) {
                uint32_t u;
                std::memcpy(&u, &f, 4);
                key.push_back(u);
            }
            return key;
        };
        std::vector<uint64_t> key = make_key();
        if (!ctx->gexec || key != ctx->g_key) {
            for (int i = 0; i <= RGS_NUM_STAGES; ++i) ctx->ev_marked[i] = false;
            if ((rc = capture_batched(ctx, V, tiles_cap, bg, lambda, tc, fused, host_targets != nullptr, accumulate))) {
                s.t -= tstep;
                return rc;
            }
            for (int i = 0; i <= RGS_NUM_STAGES; ++i) ctx->graph_marked[i] = ctx->ev_marked[i];
            ctx->g_key = make_key();  // capture may have grown scratch buffers
        }
        if (host_targets && attempt == 0) {
            for (int v = 0; v < V; ++v)
                CK(cudaMemcpyAsync((void*)h->cams[v].target, host_targets[v],
                                   (size_t)h->cams[v].width * h->cams[v].height * 16, cudaMemcpyHostToDevice, ctx->copy_st));
            CK(cudaEventRecord(ctx->ev_copy, ctx->copy_st));
        }
        CK(cudaGraphLaunch(ctx->gexec, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if (ctx->prof) {
            for (int i = 0; i <= RGS_NUM_STAGES; ++i) ctx->ev_marked[i] = ctx->graph_marked[i];
            prof_collect(ctx);
        }
        if (ctx->out_h->sort_fault) return fail(ctx, RGS_ERR_CUDA, "a sort pass's staged copies timed out");
        ctx->stats.pairs = ctx->out_h->pairs64;
        ctx->stats.supertile_entries = ctx->out_h->st_pairs64;
        ctx->stats.visible = ctx->out_h->visible;
        ctx->stats.view_groups = 1;
        if (!ctx->out_h->overflow) {
            if (losses)
                for (int v = 0; v < V; ++v) losses[v] = ctx->out_h->losses[v];
            if (fused) s.mlen = std::max(s.mlen, s.n);
            ctx->batch_views = allow_split ? V : 0;
            return RGS_OK;
        }
        // pair buffer too small: Adam was skipped on the device; grow and
        // redo, or run the batch as view groups when it is past the limit
        s.t -= tstep;
        ctx->stats.overflow_retries += 1;
        if (accumulate) return fail(ctx, RGS_ERR_CAPACITY, "a view group outgrew its pair buffer");
        const unsigned long long K = ctx->out_h->pairs64;
        if (K > ctx->opt.batch_pair_limit && allow_split && V > 1) return split_step(ctx, views, V, bg, lambda, tc, losses, fused, host_targets);
        // the supertile entries share the pair buffers: room for both
        if ((rc = ensure_pairs(ctx, std::max(K, (unsigned long long)ctx->out_h->st_pairs64)))) return rc;
    }
    return fail(ctx, RGS_ERR_CAPACITY, "pair buffer overflow persisted");
}

// The batch's views in consecutive groups whose pairs stay within the
// context's batch_pair_limit (per-view counts from the projection that just ran): each
// group runs the batched pipeline without Adam, gradients accumulating across
// groups, then one Adam step with denom += V -- the summed-gradient
// semantics of a single batch.
int split_step(rgs_ctx* ctx, const uint32_t* views, int V, const float bg[3], float lambda, const rgs_train_config& tc,
               float* losses, bool fused, const float* const* host_targets) {
    Scene& s = ctx->tr;
    ctx->split_hint = true;
    unsigned long long per[MAX_VIEWS];
    launch_view_pairs(ctx->cnt.as<uint32_t>(), (uint32_t)s.n, V, ctx->view_pairs.as<unsigned long long>(), ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(per, ctx->view_pairs.p, sizeof(unsigned long long) * V, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    int groups = 0;
    unsigned long long total = 0, total_st = 0;
    for (int v0 = 0; v0 < V;) {
        int v1 = v0 + 1;
        unsigned long long k = per[v0];
        while (v1 < V && k + per[v1] <= ctx->opt.batch_pair_limit) k += per[v1++];
        // size the pair buffer for the group first: a group that accumulates
        // into the gradients must not overflow and be redone
        int rc = ensure_pairs(ctx, k);
        if (rc) return rc;
        rc = batched_step(ctx, views + v0, v1 - v0, bg, lambda, tc, losses ? losses + v0 : nullptr, false,
                          host_targets ? host_targets + v0 : nullptr, groups > 0 ? 1 : 0, false);
        if (rc) return rc;
        total += ctx->stats.pairs;
        total_st += ctx->stats.supertile_entries;
        ++groups;
        v0 = v1;
    }
    ctx->stats.pairs = total;
    ctx->stats.supertile_entries = total_st;
    ctx->stats.view_groups = (uint32_t)groups;
    ctx->batch_views = 0;
    if (!fused) return RGS_OK;
    int rc = apply_adam(ctx, tc, (uint32_t)V);
    if (rc) return rc;
    s.mlen = std::max(s.mlen, s.n);
    return RGS_OK;
}

}  // namespace

extern "C" {

int rgs_save_ply(rgs_ctx* ctx, const float* gaussians, size_t n, const char* path) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!path || (n && !gaussians)) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if ((rc = upload_gaussians(ctx, ctx->sc, gaussians, n))) return rc;
    return save_model(ctx, ctx->sc, path, true);
}

int rgs_save_splat(rgs_ctx* ctx, const float* gaussians, size_t n, const char* path) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!path || (n && !gaussians)) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if ((rc = upload_gaussians(ctx, ctx->sc, gaussians, n))) return rc;
    return save_model(ctx, ctx->sc, path, false);
}

int rgs_load_ply(rgs_ctx* ctx, const char* path, float* out, size_t cap, size_t* n_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!path || !n_out) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    std::vector<uint8_t> d;
    if ((rc = read_file(ctx, path, d))) return rc;
    PlyLayout L;
    std::string err;
    if (parse_ply(d, L, err)) return fail(ctx, RGS_ERR_FORMAT, err + ": " + path);
    *n_out = L.count;
    if (!out || cap < L.count) return fail(ctx, RGS_ERR_CAPACITY, "output holds fewer records than the file's vertices");
    if (L.format == 2) {
        decode_ply_ascii(d, L, out);
        return RGS_OK;
    }
    Scene& s = ctx->sc;
    if ((rc = load_model(ctx, s, d, L))) return rc;
    if (L.count == 0) return RGS_OK;
    CK(ctx->stage_a.ensure(L.count * NP * sizeof(float)));
    launch_planes_to_aos(s.params.as<float4>(), ctx->stage_a.as<float>(), s.n, s.cap, ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, ctx->stage_a.p, L.count * NP * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_gaussians_from_sfm(rgs_ctx* ctx, const double* xyz, const uint8_t* rgb, size_t n, float* out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (n && (!xyz || !rgb || !out)) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    Scene& s = ctx->sc;
    if ((rc = sfm_to_scene(ctx, s, xyz, rgb, n))) return rc;
    if (n == 0) return RGS_OK;
    CK(ctx->stage_a.ensure(n * NP * sizeof(float)));
    launch_planes_to_aos(s.params.as<float4>(), ctx->stage_a.as<float>(), s.n, s.cap, ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, ctx->stage_a.p, n * NP * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_trainer_init_from_sfm(rgs_ctx* ctx, const double* xyz, const uint8_t* rgb, size_t n) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (n && (!xyz || !rgb)) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    Scene& s = ctx->tr;
    if ((rc = sfm_to_scene(ctx, s, xyz, rgb, n))) return rc;
    return fresh_adam_state(ctx, s);
}

int rgs_read_points3d_bin(rgs_ctx* ctx, const char* path, double* xyz, uint8_t* rgb, size_t cap, size_t* n_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!path || !n_out) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    std::vector<uint8_t> d;
    if ((rc = read_file(ctx, path, d))) return rc;
    std::vector<double> px;
    std::vector<uint8_t> pc;
    if ((rc = parse_points3d(ctx, d, px, pc))) return rc;
    const size_t n = pc.size() / 3;
    *n_out = n;
    if (!xyz || !rgb || cap < n) return fail(ctx, RGS_ERR_CAPACITY, "output holds fewer points than the file");
    if (n) {
        std::memcpy(xyz, px.data(), n * 24);
        std::memcpy(rgb, pc.data(), n * 3);
    }
    return RGS_OK;
}

int rgs_srgb8_to_linear(rgs_ctx* ctx, const uint8_t* rgba8, size_t npix, float* out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (npix && (!rgba8 || !out)) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if (npix == 0) return RGS_OK;
    CK(ctx->stage_a.ensure(npix * 4));
    CK(ctx->stage_b.ensure(npix * 16));
    CK(cudaMemcpyAsync(ctx->stage_a.p, rgba8, npix * 4, cudaMemcpyHostToDevice, ctx->st));
    launch_srgb8_to_linear(ctx->stage_a.p, npix, ctx->stage_b.as<float>(), ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, ctx->stage_b.p, npix * 16, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_trainer_set_target_rgba8(rgs_ctx* ctx, size_t index, const uint8_t* rgba8) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (index >= ctx->cams.size() || !rgba8) return fail(ctx, RGS_ERR_INVALID_ARG, "bad camera index or null target");
    const size_t px = (size_t)ctx->cams[index].width * ctx->cams[index].height;
    CK(ctx->targets[index].ensure(px * 16));
    CK(ctx->stage_a.ensure(std::max<size_t>(px * 4, 16)));
    CK(cudaMemcpyAsync(ctx->stage_a.p, rgba8, px * 4, cudaMemcpyHostToDevice, ctx->st));
    launch_srgb8_to_linear(ctx->stage_a.p, px, ctx->targets[index].as<float>(), ctx->st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_trainer_save_ply(rgs_ctx* ctx, const char* path) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!path) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    return save_model(ctx, ctx->tr, path, true);
}

int rgs_trainer_save_splat(rgs_ctx* ctx, const char* path) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!path) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    return save_model(ctx, ctx->tr, path, false);
}

int rgs_trainer_load_ply(rgs_ctx* ctx, const char* path, size_t* n_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!path) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    std::vector<uint8_t> d;
    if ((rc = read_file(ctx, path, d))) return rc;
    PlyLayout L;
    std::string err;
    if (parse_ply(d, L, err)) return fail(ctx, RGS_ERR_FORMAT, err + ": " + path);
    Scene& s = ctx->tr;
    if ((rc = load_model(ctx, s, d, L))) return rc;
    if ((rc = fresh_adam_state(ctx, s))) return rc;
    if (n_out) *n_out = L.count;
    return RGS_OK;
}

int rgs_trainer_step(rgs_ctx* ctx, const uint32_t* views, size_t nviews, const float bg[3], const rgs_loss_config* loss_cfg,
                     const rgs_train_config* train_cfg, int mode, float* losses_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!bg || !loss_cfg || !train_cfg) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if ((rc = check_views(ctx, views, nviews, true))) return rc;
    if (mode == RGS_STEP_BATCHED)
        return batched_step(ctx, views, (int)nviews, bg, loss_cfg->lambda_dssim, *train_cfg, losses_out, true);
    if (mode != RGS_STEP_PLAIN) return fail(ctx, RGS_ERR_INVALID_ARG, "unknown step mode");
    if ((rc = ensure_moments(ctx, ctx->tr, ctx->tr.n))) return rc;
    if ((rc = plain_backward(ctx, views, nviews, bg, loss_cfg->lambda_dssim, losses_out))) return rc;
    if ((rc = apply_adam(ctx, *train_cfg, (uint32_t)nviews))) return rc;
    ctx->tr.mlen = std::max(ctx->tr.mlen, ctx->tr.n);
    return RGS_OK;
}

int rgs_trainer_step_host_targets(rgs_ctx* ctx, const uint32_t* views, size_t nviews, const float* const* targets_rgba,
                                  const float bg[3], const rgs_loss_config* loss_cfg, const rgs_train_config* train_cfg,
                                  float* losses_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!bg || !loss_cfg || !train_cfg || !targets_rgba) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if ((rc = check_views(ctx, views, nviews, false))) return rc;
    for (size_t v = 0; v < nviews; ++v)
        if (!targets_rgba[v]) return fail(ctx, RGS_ERR_INVALID_ARG, "null target pointer");
    return batched_step(ctx, views, (int)nviews, bg, loss_cfg->lambda_dssim, *train_cfg, losses_out, true, targets_rgba);
}

int rgs_trainer_backward(rgs_ctx* ctx, const uint32_t* views, size_t nviews, const float bg[3], const rgs_loss_config* loss_cfg,
                         int mode, float* losses_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!bg || !loss_cfg) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if ((rc = check_views(ctx, views, nviews, true))) return rc;
    if (mode == RGS_STEP_BATCHED) {
        rgs_train_config tc;
        rgs_train_config_default(&tc);
        return batched_step(ctx, views, (int)nviews, bg, loss_cfg->lambda_dssim, tc, losses_out, false);
    }
    if (mode != RGS_STEP_PLAIN) return fail(ctx, RGS_ERR_INVALID_ARG, "unknown step mode");
    return plain_backward(ctx, views, nviews, bg, loss_cfg->lambda_dssim, losses_out);
}

int rgs_get_options(rgs_ctx* ctx, rgs_options* out) {
    if (!ctx || !out) return RGS_ERR_INVALID_ARG;
    *out = ctx->opt;
    return RGS_OK;
}

int rgs_set_tiling(rgs_ctx* ctx, int tile_w, int tile_h, int batch, int pixels_per_thread) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    bool shape_ok = (tile_w == 16 && tile_h == 16) || (tile_w == 8 && tile_h == 32) || (tile_w == 32 && tile_h == 8);
    if (!shape_ok) return fail(ctx, RGS_ERR_INVALID_ARG, "tile shape must be 16x16, 8x32 or 32x8");
    if (batch != 128 && batch != 256 && batch != 512) return fail(ctx, RGS_ERR_INVALID_ARG, "batch must be 128, 256 or 512");
    if (pixels_per_thread != 1 && pixels_per_thread != 2)
        return fail(ctx, RGS_ERR_INVALID_ARG, "pixels_per_thread must be 1 or 2");
    // the graph key holds the layout, so the next batched step recaptures
    ctx->opt.tile_w = tile_w;
    ctx->opt.tile_h = tile_h;
    ctx->opt.batch = batch;
    ctx->opt.pixels_per_thread = pixels_per_thread;
    return RGS_OK;
}

// Autotuner: every layout is timed on the same views with CUDA events on the
// context's stream around `reps` batched render + backward passes (after one
// untimed pass that captures the layout's graph and warms it), and the fastest
// one is kept. Gradients are overwritten; parameters, moments, grad_accum /
// grad_denom and the Adam step count are untouched (MODE 0 of the geometry
// pass writes gradients only).
int rgs_trainer_autotune(rgs_ctx* ctx, const uint32_t* views, size_t nviews, const float bg[3], const rgs_loss_config* loss_cfg,
                         int reps, rgs_tune_entry* results, rgs_options* chosen) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!bg || !loss_cfg) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if (reps < 1) return fail(ctx, RGS_ERR_INVALID_ARG, "reps must be >= 1");
    if ((rc = check_views(ctx, views, nviews, true))) return rc;
    static const int shapes[3][2] = {{16, 16}, {8, 32}, {32, 8}};
    static const int batches[3] = {128, 256, 512};
    rgs_train_config tc;
    rgs_train_config_default(&tc);
    const rgs_options saved = ctx->opt;
    const bool prof = ctx->prof;
    ctx->prof = false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t ce = cudaEventCreate(&e0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
    if (ce != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        ctx->prof = prof;
        return cuda_fail(ctx, ce, "autotune events");
    }
    float best = 0.0f;
    rgs_options best_opt = saved;
    int k = 0;
    for (int si = 0; si < 3 && rc == RGS_OK; ++si)
        for (int bi = 0; bi < 3 && rc == RGS_OK; ++bi)
            for (int ppt = 1; ppt <= 2 && rc == RGS_OK; ++ppt, ++k) {
                ctx->opt.tile_w = shapes[si][0];
                ctx->opt.tile_h = shapes[si][1];
                ctx->opt.batch = batches[bi];
                ctx->opt.pixels_per_thread = ppt;
                rc = batched_step(ctx, views, (int)nviews, bg, loss_cfg->lambda_dssim, tc, nullptr, false);
                float ms = 0.0f;
                if (rc == RGS_OK && (ce = cudaEventRecord(e0, ctx->st)) != cudaSuccess) rc = cuda_fail(ctx, ce, "autotune");
                for (int r = 0; r < reps && rc == RGS_OK; ++r)
                    rc = batched_step(ctx, views, (int)nviews, bg, loss_cfg->lambda_dssim, tc, nullptr, false);
                if (rc == RGS_OK && (ce = cudaEventRecord(e1, ctx->st)) != cudaSuccess) rc = cuda_fail(ctx, ce, "autotune");
                if (rc == RGS_OK && (ce = cudaEventSynchronize(e1)) != cudaSuccess) rc = cuda_fail(ctx, ce, "autotune");
                if (rc == RGS_OK && (ce = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) rc = cuda_fail(ctx, ce, "autotune");
                ms /= (float)reps;
                if (results) results[k] = rgs_tune_entry{shapes[si][0], shapes[si][1], batches[bi], ppt, ms};
                if (rc == RGS_OK && (k == 0 || ms < best)) {
                    best = ms;
                    best_opt = ctx->opt;
                }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->prof = prof;
    ctx->opt = rc == RGS_OK ? best_opt : saved;
    if (rc == RGS_OK && chosen) *chosen = ctx->opt;
    return rc;
}

int rgs_trainer_get_grads(rgs_ctx* ctx, float* out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    Scene& s = ctx->tr;
    if (s.n == 0) return RGS_OK;
    if (!out) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    CK(ctx->stage_b.ensure((size_t)s.n * NG * 4));
    launch_grads_to_aos(s.grads.as<float4>(), ctx->stage_b.as<float>(), s.n, s.cap, NG, ctx->st);
    CK(cudaMemcpyAsync(out, ctx->stage_b.p, (size_t)s.n * NG * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_trainer_grad_buffer(rgs_ctx* ctx, void** device_ptr, size_t* bytes, size_t* plane_stride) {
    if (!ctx || !device_ptr || !bytes || !plane_stride) return RGS_ERR_INVALID_ARG;
    *device_ptr = ctx->tr.grads.p;
    *bytes = (size_t)ctx->tr.cap * NPL * sizeof(float4);
    *plane_stride = (size_t)ctx->tr.cap;
    return RGS_OK;
}

int rgs_trainer_apply_adam(rgs_ctx* ctx, const rgs_train_config* cfg, uint32_t denom_increment) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!cfg) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if ((rc = ensure_moments(ctx, ctx->tr, ctx->tr.n))) return rc;
    if ((rc = apply_adam(ctx, *cfg, denom_increment))) return rc;
    ctx->tr.mlen = std::max(ctx->tr.mlen, ctx->tr.n);
    return RGS_OK;
}

int rgs_trainer_render(rgs_ctx* ctx, uint32_t view, const float bg[3], float* rgb_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!bg || !rgb_out || view >= ctx->cams.size()) return fail(ctx, RGS_ERR_INVALID_ARG, "bad argument");
    DevCam dc;
    if ((rc = make_devcam(ctx, ctx->cams[view], dc))) return rc;
    return run_view_plain(ctx, ctx->tr, dc, nullptr, bg, 0.0f, false, false, nullptr, rgb_out);
}

int rgs_trainer_densify_and_prune(rgs_ctx* ctx, const rgs_train_config* cfg, float scene_extent, size_t* n_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!cfg) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    Scene& s = ctx->tr;
    if ((rc = ensure_moments(ctx, s, std::max(s.n, 1)))) return rc;
    DensifyArgs a;
    a.params = s.params.as<float4>();
    a.n = s.n;
    a.cap = s.cap;
    a.grad_accum = s.accum.as<float>();
    a.grad_denom = s.denom.as<uint32_t>();
    a.prune_opacity = cfg->prune_opacity_thresh;
    a.grad_threshold = cfg->densify_grad_threshold;
    a.extent = scene_extent;
    a.max_gaussians = cfg->max_gaussians;
    int n_new = 0, ocap = 0;
    CK(densify_and_prune(a, ctx->dens_out, &ocap, ctx->dens_scratch, &n_new, ctx->st));
    if (s.n > 0) {
        std::swap(s.params, ctx->dens_out);
        s.cap = ocap;
        s.n = n_new;
        s.grads.release();
        CK(s.grads.ensure((size_t)s.cap * NPL * sizeof(float4)));
    }
    // AdamState::resize grows the moments (zero-filled) and never shrinks them;
    // the statistics are zeroed (optimizer.rs:262-266).
    if ((rc = ensure_moments(ctx, s, std::max(s.n, 1)))) return rc;
    s.mlen = std::max(s.mlen, s.n);
    CK(cudaMemsetAsync(s.accum.p, 0, (size_t)s.mcap * 4, ctx->st));
    CK(cudaMemsetAsync(s.denom.p, 0, (size_t)s.mcap * 4, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (n_out) *n_out = (size_t)s.n;
    return RGS_OK;
}

int rgs_trainer_reset_opacities(rgs_ctx* ctx) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    launch_reset_opacities(ctx->tr.params.as<float4>(), ctx->tr.n, ctx->tr.cap, ctx->st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_trainer_get_adam_state(rgs_ctx* ctx, rgs_adam_state* state) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    Scene& s = ctx->tr;
    if (!state) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    size_t len = std::min<size_t>(state->len, (size_t)s.mcap);
    state->t = s.t;
    if (len == 0) return RGS_OK;
    if (!state->m1 || !state->m2 || !state->grad_accum || !state->grad_denom) return fail(ctx, RGS_ERR_INVALID_ARG, "null array");
    CK(ctx->stage_c.ensure(len * NP * 4));
    CK(ctx->stage_d.ensure(len * NP * 4));
    launch_grads_to_aos(s.m1.as<float4>(), ctx->stage_c.as<float>(), (int)len, s.mcap, NP, ctx->st);
    launch_grads_to_aos(s.m2.as<float4>(), ctx->stage_d.as<float>(), (int)len, s.mcap, NP, ctx->st);
    CK(cudaMemcpyAsync(state->m1, ctx->stage_c.p, len * NP * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(state->m2, ctx->stage_d.p, len * NP * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(state->grad_accum, s.accum.p, len * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(state->grad_denom, s.denom.p, len * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_trainer_set_adam_state(rgs_ctx* ctx, const rgs_adam_state* state) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    Scene& s = ctx->tr;
    if (!state) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    size_t len = state->len;
    if ((rc = ensure_moments(ctx, s, (int)std::max<size_t>(len, 1)))) return rc;
    s.t = state->t;
    s.mlen = (int)len;
    if (len == 0) return RGS_OK;
    if (!state->m1 || !state->m2 || !state->grad_accum || !state->grad_denom) return fail(ctx, RGS_ERR_INVALID_ARG, "null array");
    CK(ctx->stage_c.ensure(len * NP * 4));
    CK(ctx->stage_d.ensure(len * NP * 4));
    CK(cudaMemcpyAsync(ctx->stage_c.p, state->m1, len * NP * 4, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->stage_d.p, state->m2, len * NP * 4, cudaMemcpyHostToDevice, ctx->st));
    launch_aos_to_grad_planes(ctx->stage_c.as<float>(), s.m1.as<float4>(), (int)len, s.mcap, NP, ctx->st);
    launch_aos_to_grad_planes(ctx->stage_d.as<float>(), s.m2.as<float4>(), (int)len, s.mcap, NP, ctx->st);
    CK(cudaMemcpyAsync(s.accum.p, state->grad_accum, len * 4, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(s.denom.p, state->grad_denom, len * 4, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

}  // extern "C"

// ===========================================================================
// introspection (include/rgsplat_debug.h)
// ===========================================================================
namespace {

// Uploads gaussians + camera into the scratch scene and bins one view.
int debug_bin(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, DevCam& dc, DevCam** cams_dev,
              Binned& b, size_t& px, size_t& tiles, size_t& lb, bool prune = false) {
    if (!camera || (n && !gaussians)) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    int rc = make_devcam(ctx, *camera, dc);
    if (rc) return rc;
    Scene& s = ctx->sc;
    if ((rc = upload_gaussians(ctx, s, gaussians, n))) return rc;
    if ((rc = check_finite(ctx, s))) return rc;
    assign_bases(&dc, 1, px, tiles, lb);
    if ((rc = ensure_work(ctx, std::max<size_t>(n, 1), px, tiles, lb, 1))) return rc;
    if ((rc = upload_single_cam(ctx, dc, cams_dev))) return rc;
    if ((rc = ensure_gcache(ctx, s))) return rc;
    return bin_batch(ctx, s, *cams_dev, 1, tiles, true, b, true, prune);
}

}  // namespace

extern "C" {

int rgs_debug_project(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, int32_t* visible, float* rec10,
                      int32_t* rect4) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (n && (!visible || !rec10 || !rect4)) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    DevCam dc, *cams_dev;
    Binned b;
    size_t px, tiles, lb;
    if ((rc = debug_bin(ctx, gaussians, n, camera, dc, &cams_dev, b, px, tiles, lb))) return rc;
    if (n == 0) return RGS_OK;
    std::vector<float4> rec(3 * n);
    std::vector<uint32_t> cnt(n);
    CK(cudaMemcpyAsync(rec.data(), ctx->rec.p, 3 * n * sizeof(float4), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(cnt.data(), ctx->cnt.p, n * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    for (size_t i = 0; i < n; ++i) {
        visible[i] = cnt[i] > 0;
        float* r = rec10 + i * 10;
        int32_t* q = rect4 + i * 4;
        if (!cnt[i]) {
            for (int k = 0; k < 10; ++k) r[k] = 0.0f;
            q[0] = q[1] = q[2] = q[3] = 0;
            continue;
        }
        float4 a = rec[i], c = rec[n + i], k = rec[2 * n + i];
        r[0] = a.x; r[1] = a.y; r[2] = c.x; r[3] = c.y; r[4] = c.z; r[5] = k.x; r[6] = k.y; r[7] = k.z; r[8] = a.z; r[9] = a.w;
        uint32_t rx, ry;
        std::memcpy(&rx, &c.w, 4);
        std::memcpy(&ry, &k.w, 4);
        q[0] = (int32_t)(rx & 0xffffu) / REF_TILE;
        q[1] = (int32_t)(ry & 0xffffu) / REF_TILE;
        q[2] = ((int32_t)(rx >> 16) + REF_TILE - 1) / REF_TILE;
        q[3] = ((int32_t)(ry >> 16) + REF_TILE - 1) / REF_TILE;
    }
    return RGS_OK;
}

namespace {
int debug_tile_lists(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, uint64_t* n_pairs,
                     int32_t* offsets, int32_t* entries, size_t cap, bool prune) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!n_pairs) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    DevCam dc, *cams_dev;
    Binned b;
    size_t px, tiles, lb;
    if ((rc = debug_bin(ctx, gaussians, n, camera, dc, &cams_dev, b, px, tiles, lb, prune))) return rc;
    uint32_t K = 0;
    CK(cudaMemcpyAsync(&K, ctx->scalars.as<uint32_t>() + SC_PAIRS, 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    *n_pairs = K;
    if (!entries) return RGS_OK;
    if (!offsets || cap < K) return fail(ctx, RGS_ERR_CAPACITY, "entries buffer too small");
    // each tile's list is ranges[t] in the list buffer (lists are grouped by
    // supertile there): concatenate them in tile order
    std::vector<uint2> rg(std::max<size_t>(tiles, 1));
    std::vector<uint32_t> vals(std::max<uint32_t>(K, 1));
    CK(cudaMemcpyAsync(rg.data(), ctx->ranges.p, tiles * sizeof(uint2), cudaMemcpyDeviceToHost, ctx->st));
    if (K) CK(cudaMemcpyAsync(vals.data(), b.vals, (size_t)K * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    size_t k = 0;
    for (size_t t = 0; t < tiles; ++t) {
        offsets[t] = (int32_t)k;
        if (rg[t].y < rg[t].x || rg[t].y > K || k + (rg[t].y - rg[t].x) > K)
            return fail(ctx, RGS_ERR_CUDA, "internal: tile ranges out of bounds");
        for (uint32_t p = rg[t].x; p < rg[t].y; ++p) entries[k++] = (int32_t)vals[p];
    }
    offsets[tiles] = (int32_t)k;
    if (k != K) return fail(ctx, RGS_ERR_CUDA, "internal: tile lists do not hold every pair");
    return RGS_OK;
}
}  // namespace

int rgs_debug_tile_lists(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, uint64_t* n_pairs,
                         int32_t* offsets, int32_t* entries, size_t cap) {
    return debug_tile_lists(ctx, gaussians, n, camera, n_pairs, offsets, entries, cap, false);
}

int rgs_debug_pruned_tile_lists(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera,
                                uint64_t* n_pairs, int32_t* offsets, int32_t* entries, size_t cap) {
    return debug_tile_lists(ctx, gaussians, n, camera, n_pairs, offsets, entries, cap, true);
}

int rgs_debug_forward(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, const float bg[3], float* rgb,
                      float* final_t, int32_t* last) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!bg || !rgb || !final_t || !last) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    DevCam dc, *cams_dev;
    Binned b;
    size_t px, tiles, lb;
    if ((rc = debug_bin(ctx, gaussians, n, camera, dc, &cams_dev, b, px, tiles, lb))) return rc;
    BlendArgs fa = blend_args(ctx, ctx->sc, cams_dev, 1, nullptr, tiles, b, bg, true);
    launch_blend_forward(fa, ctx->opt.tile_w, ctx->opt.tile_h, ctx->opt.batch, ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(rgb, ctx->rgb.p, px * 12, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(final_t, ctx->final_t.p, px * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(last, ctx->last.p, px * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

int rgs_debug_backward(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, const float* target_rgba,
                       const float bg[3], float lambda, float* acc9, float* dl_dpix) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!bg || !target_rgba || (n && !acc9)) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    DevCam dc, *cams_dev;
    Binned b;
    size_t px, tiles, lb;
    if ((rc = debug_bin(ctx, gaussians, n, camera, dc, &cams_dev, b, px, tiles, lb))) return rc;
    CK(ctx->target_stage.ensure(px * 16));
    CK(cudaMemcpyAsync(ctx->target_stage.p, target_rgba, px * 16, cudaMemcpyHostToDevice, ctx->st));
    dc.target = ctx->target_stage.as<float>();
    if ((rc = upload_single_cam(ctx, dc, &cams_dev))) return rc;
    BlendArgs fa = blend_args(ctx, ctx->sc, cams_dev, 1, nullptr, tiles, b, bg, true);
    launch_blend_forward(fa, ctx->opt.tile_w, ctx->opt.tile_h, ctx->opt.batch, ctx->st);
    float* losses_dev = (float*)((char*)ctx->outd.p + offsetof(StepOut, losses));
    CK(launch_loss(cams_dev, 1, (int)lb, ctx->rgb.as<float>(), lambda, ctx->dl.as<float>(), ctx->partials.as<float>(),
                   losses_dev, nullptr, ctx->opt.exact_loss != 0, ctx->st));
    CK(cudaMemsetAsync(ctx->acc.p, 0, std::max<size_t>(n, 1) * 3 * sizeof(float4), ctx->st));
    BlendArgs ba = blend_args(ctx, ctx->sc, cams_dev, 1, nullptr, tiles, b, bg, false);
    launch_blend_backward(ba, ctx->opt.tile_w, ctx->opt.tile_h, ctx->opt.batch, ctx->st);
    CK(cudaGetLastError());
    if (n) {
        std::vector<float4> acc(3 * n);
        CK(cudaMemcpyAsync(acc.data(), ctx->acc.p, 3 * n * sizeof(float4), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        for (size_t i = 0; i < n; ++i) {
            float4 a = acc[i], c = acc[n + i], d = acc[2 * n + i];
            float* o = acc9 + i * 9;
            o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w; o[4] = c.x; o[5] = c.y; o[6] = c.z; o[7] = c.w; o[8] = d.x;
        }
    }
    if (dl_dpix) {
        CK(cudaMemcpyAsync(dl_dpix, ctx->dl.p, px * 12, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
    return RGS_OK;
}

int rgs_trainer_evaluated_pairs(rgs_ctx* ctx, uint64_t* forward_pairs, uint64_t* backward_pairs) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!forward_pairs || !backward_pairs) return fail(ctx, RGS_ERR_INVALID_ARG, "null argument");
    if (ctx->batch_views <= 0) return fail(ctx, RGS_ERR_INVALID_ARG, "no batched pass holds the pixel buffers");
    const DevCam* cams_dev = (const DevCam*)((char*)ctx->hdr.p + offsetof(StepHdr, cams));
    unsigned long long* out = ctx->view_pairs.as<unsigned long long>();
    unsigned long long h[2] = {0, 0};
    CK(cudaMemsetAsync(out, 0, 16, ctx->st));
    launch_evaluated_pairs(cams_dev, ctx->batch_views, ctx->ranges.as<uint2>(), ctx->final_t.as<float>(), ctx->last.as<int>(),
                           ctx->opt.tile_w, ctx->opt.tile_h, out, ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h, out, 16, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    *forward_pairs = h[0];
    *backward_pairs = h[1];
    return RGS_OK;
}

int rgs_debug_exp_sfu_error(rgs_ctx* ctx, float lo, float hi, uint32_t n, float* max_rel) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!max_rel || n == 0 || !(lo <= hi) || !(hi <= 0.0f) || !(lo >= -8.0f))
        return fail(ctx, RGS_ERR_INVALID_ARG, "need -8 <= lo <= hi <= 0, n > 0");
    CK(ctx->view_pairs.ensure(MAX_VIEWS * 8));
    unsigned int* out = ctx->view_pairs.as<unsigned int>();
    unsigned int h = 0;
    CK(cudaMemsetAsync(out, 0, 4, ctx->st));
    launch_exp_sfu_error(lo, hi, n, out, ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&h, out, 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    std::memcpy(max_rel, &h, 4);
    return RGS_OK;
}

int rgs_debug_trainer_batch_pixels(rgs_ctx* ctx, size_t k, float* rgb, float* final_t, float* dl_dpix) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (ctx->batch_views <= 0) return fail(ctx, RGS_ERR_INVALID_ARG, "no batched pass holds the pixel buffers");
    if (k >= (size_t)ctx->batch_views) return fail(ctx, RGS_ERR_INVALID_ARG, "view position out of range");
    const DevCam& c = ctx->hdr_h->cams[k];
    const size_t px = (size_t)c.width * c.height, base = (size_t)c.pix_base;
    if (rgb) CK(cudaMemcpyAsync(rgb, ctx->rgb.as<float>() + base * 3, px * 12, cudaMemcpyDeviceToHost, ctx->st));
    if (final_t) CK(cudaMemcpyAsync(final_t, ctx->final_t.as<float>() + base, px * 4, cudaMemcpyDeviceToHost, ctx->st));
    if (dl_dpix) CK(cudaMemcpyAsync(dl_dpix, ctx->dl.as<float>() + base * 3, px * 12, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return RGS_OK;
}

}  // extern "C"
