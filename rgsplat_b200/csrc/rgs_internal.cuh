// rgs_internal.cuh -- layouts and kernel launchers shared by the library's .cu files.
//
// HBM layout (all device-resident, SoA "planes" of float4 so every load of a
// Gaussian's state is a coalesced 16-byte access):
//   params  [NPL][cap] float4   plane 0: position.xyz, opacity_logit
//                               plane 1: rotation wxyz
//                               plane 2: log_scale.xyz, pad
//                               planes 3..14: sh[0..47] (channel-major as in
//                               Gaussian3D::sh_coeffs, src/math/mod.rs:45)
//   i.e. the reference's 59-float Gaussian3D record with one pad after
//   log_scale, transposed. Gradients and both Adam moments use the same planes;
//   the gradient pad lane carries screen_grad_norm (backward.rs:40).
// Per step, for V views and N Gaussians, a "slot" s = v*N + i names Gaussian i
// as seen by view v:
//   rec     [3][S] float4  projected splat: (sx, sy, opacity, depth),
//                          (conic a, b, c, pixel rect x0|x1<<16),
//                          (r, g, b, pixel rect y0|y1<<16)
//   cnt     [S] u32        number of CTA tiles the splat touches (0 = culled)
//   acc     [3][S] float4  blend-backward accumulators (color3, opacity,
//                          conic3, sx, sy) of backward.rs:92-99
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace rgs {

constexpr int NPL = 15;        // float4 planes per Gaussian
constexpr int NP = 59;         // trainable floats (optimizer.rs:71)
constexpr int NG = 60;         // GaussianGrad floats (backward.rs:33-41)
constexpr int REF_TILE = 16;   // TILE_SIZE of backward.rs:21

// One view of a batch, prepared on the host.
struct DevCam {
    float view[12];            // rows 0..2 of inverse(c2w), row-major
    float fx, fy, cx, cy;
    float pos[3];              // camera centre (Camera::position, mod.rs:163-165)
    int width, height;
    int ref_tiles_x, ref_tiles_y;  // 16x16 reference tiles
    int tiles_x, tiles_y;      // CTA tiles of the configured shape
    int tile_base;             // first global CTA tile of this view
    int pix_base;              // first pixel of this view in the batch buffers
    int loss_base;             // first loss block of this view
    int loss_bx;               // loss blocks per row
    int st_x;                  // supertiles (4x4 CTA tiles) per row
    int st_base;               // first global supertile of this view
    const float* target;       // RGBA float target (w*h*4), device
};

// Tile lists are built through supertiles of ST_EDGE x ST_EDGE CTA tiles: the
// slots are first sorted by supertile, then the sorted entries are expanded
// into the lists of the supertiles' tiles (supertile.cu).
constexpr int ST_EDGE = 4;
constexpr int ST_TILES = ST_EDGE * ST_EDGE;

// Reference record (Gaussian3D) float index -> (plane, lane).
__host__ __device__ inline void record_to_plane(int f, int& p, int& l) {
    if (f < 4) { p = 0; l = f; }
    else if (f < 8) { p = 1; l = f - 4; }
    else if (f < 11) { p = 2; l = f - 8; }
    else { p = 3 + (f - 11) / 4; l = (f - 11) % 4; }
}

// GaussianGrad flat index j (0..59) -> record float index (optimizer.rs:165-173,
// 186-195); 59 (screen_grad_norm) -> the pad lane (plane 2, lane 3) = 11.
__host__ __device__ inline int grad_to_record(int j) {
    if (j < 3) return j;
    if (j < 7) return 4 + (j - 3);
    if (j < 10) return 8 + (j - 7);
    if (j == 10) return 3;
    if (j < 59) return j;
    return -1;
}

enum Status {
    RGS_OK_ = 0,
    E_INVALID = -1,
    E_OOM = -2,
    E_CUDA = -3,
    E_NONFINITE = -4,
    E_SINGULAR = -5,
    E_CAPACITY = -6,
    E_NODEVICE = -7,
};

// Device bytes a context holds through its buffers, and the most it has held
// since its last reset. Each entry point sets the calling thread's counter to
// its context's (contexts are used by one host thread at a time).
struct MemCounter {
    size_t held = 0, peak = 0;
};
extern thread_local MemCounter* t_mem;
inline void mem_add(size_t b) {
    if (!t_mem) return;
    t_mem->held += b;
    if (t_mem->held > t_mem->peak) t_mem->peak = t_mem->held;
}
inline void mem_sub(size_t b) {
    if (t_mem) t_mem->held -= b < t_mem->held ? b : t_mem->held;
}

// Grow-only device allocation.
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t need) {
        if (need <= bytes) return cudaSuccess;
        release();
        size_t want = need + need / 4 + 256;
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) {
            bytes = want;
            mem_add(want);
        } else {
            p = nullptr;
        }
        return e;
    }
    void release() {
        if (p) {
            cudaFree(p);
            mem_sub(bytes);
        }
        p = nullptr;
        bytes = 0;
    }
    template <class T> T* as() const { return (T*)p; }
};

struct SortScratch {
    DBuf hist;   // [G][R] u32
    DBuf keys2, vals2;
    int* fault = nullptr;  // device word the owner provides: set (and left set)
                           // when a pass's staged copies time out
};

// Device scratch of the SfM initialisation (sfm.cu): its own sort buffers, so
// the trainer's captured step never sees them change.
struct SfmScratch {
    DBuf xyz, rgb;           // the points as uploaded
    DBuf u32, f64, scales, flag;
    SortScratch sort;
    void release() {
        for (DBuf* b : {&xyz, &rgb, &u32, &f64, &scales, &flag, &sort.hist, &sort.keys2, &sort.vals2}) b->release();
    }
};

// ---- launchers (each defined in the .cu file named in the comment) --------

// device.cu: SM count of the current device, cached per device ordinal.
int device_sm_count();

// layout.cu
void launch_aos_to_planes(const float* aos, float4* planes, int n, int cap, cudaStream_t st);
void launch_planes_to_aos(const float4* planes, float* aos, int n, int cap, cudaStream_t st);
void launch_grads_to_aos(const float4* gplanes, float* aos, int n, int cap, int stride, cudaStream_t st);
void launch_aos_to_grad_planes(const float* aos, float4* planes, int n, int cap, int stride, cudaStream_t st);
void launch_check_finite(const float4* planes, int n, int cap, int* flag, cudaStream_t st);

// project.cu
// tdesc[s] = (global id of the splat's first CTA tile, width | height << 16 of
// its CTA-tile rectangle), cnt[s] = its number of CTA tiles, or with prune = 1
// the number inside the rows' kept spans (tiles.cuh); zero for culled slots.
// *visible (zeroed by the caller) gains the number of slots with cnt > 0.
// With prune, spans[2 slot] holds the kept spans of rectangles up to SPAN_ROWS
// rows and 15 columns, byte r of the 16 (x holds rows 0-3, y 4-7, ...): first
// kept column - first rectangle column | kept count << 4. Larger rectangles
// get SPANS_NONE in every word (a byte 0xff never occurs in a packed record:
// the first column and the count add up to at most 15).
constexpr int SPAN_ROWS = 16;
constexpr uint32_t SPANS_NONE = 0xffffffffu;
void launch_project(const float4* params, int n, int cap, const DevCam* cams, int nviews,
                    int tile_w, int tile_h, float4* rec, uint32_t* cnt, uint2* tdesc, uint32_t* dkey,
                    uint32_t* ids, int prune, uint32_t* visible, float4* gcache, uint4* spans, cudaStream_t st);
// Per-Gaussian view-independent projection terms ([2][cap] float4: opacity
// and the 3D covariance's six entries), computed by launch_project first and
// read by the geometry of the same step.
void launch_gauss_cache(const float4* params, int n, int cap, float4* gcache, cudaStream_t st);
void launch_project_wgsl(const float4* params, int n, int cap, const DevCam* cam, int cpu_math,
                         float* splats10, uint32_t* keys, cudaStream_t st);
void launch_composite_prepare(const float* splats10, int n, const DevCam* cam, int tile_w, int tile_h,
                              float4* rec, uint32_t* cnt, uint2* tdesc, uint32_t* dkey, uint32_t* ids,
                              cudaStream_t st);

// sort.cu: stable LSD radix sort of (key, value) u32 pairs on bits [0, bits).
// n_dev may be null (then n_host is used). Returns which buffer holds the
// result: 0 = (keys, vals), 1 = (keys2, vals2) in the scratch.
int radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n_host, const uint32_t* n_dev, int bits,
                     SortScratch& sc, int grid, cudaStream_t st, cudaError_t* err);
int sort_grid_blocks();
// scratch of one radix pass: a [256][grid] digit histogram plus 256 digit totals
inline size_t sort_hist_bytes(int grid) { return ((size_t)grid * 256 + 256) * 4; }

// bin.cu
// Exclusive scan of the per-slot counts cnt[order[r]] in depth order (pruned
// tile pairs, or supertile entries). block_sums: one u64 per CTA of `grid`;
// *total is the count saturated at 2^32 - 1, *total64 the exact count.
// S_dev (may be null) holds the number of order entries on the device.
void launch_count_scan(const uint32_t* order, const uint32_t* cnt, uint32_t S, const uint32_t* S_dev,
                       unsigned long long* block_sums, uint32_t* total, unsigned long long* total64, int grid, cudaStream_t st);
// Per-view pair totals (slot = view * n + Gaussian) into out[0, V).
void launch_view_pairs(const uint32_t* cnt, uint32_t n, int V, unsigned long long* out, cudaStream_t st);
int bin_grid_blocks();
// The slots with at least one tile pair (cnt != 0), gathered in slot order:
// their keys into ckey, their slot indices into cslot, the count into *n_out
// (and *n_out64). chunk_counts holds compact_chunks(S) u64.
size_t compact_chunks(size_t S);
void launch_compact_visible(const uint32_t* cnt, const uint32_t* key, uint32_t S, unsigned long long* chunk_counts,
                            uint32_t* ckey, uint32_t* cslot, uint32_t* n_out, unsigned long long* n_out64,
                            const uint2* tdesc, const DevCam* cams, uint32_t n_per_view, uint32_t* st_cnt, uint2* st_desc,
                            cudaStream_t st);
// Supertile rectangles expanded into (supertile id, slot) entries in the
// order's (depth) order: the rectangle emitter with the view's supertile
// stride (st_desc holds the first supertile id and width | height << 16).
void launch_emit_supertiles(const uint32_t* order, const uint2* st_desc, uint32_t S, const uint32_t* S_dev,
                            const unsigned long long* block_sums, uint32_t* keys, uint32_t* vals, uint32_t cap, int* overflow,
                            const uint32_t* total, uint32_t* eff, const DevCam* cams, uint32_t n_per_view, int grid,
                            cudaStream_t st);

// supertile.cu: the tile lists from the supertile-sorted entries.
struct SupertileArgs {
    const DevCam* cams;
    int nviews;
    const uint32_t* ent_key;       // sorted entries: supertile id
    const uint32_t* ent_slot;      // sorted entries: slot
    const uint32_t* n_ent;         // device count of the sorted entries
    const uint2* tdesc;            // per slot: first CTA tile, rect width | height << 16
    const uint4* spans;            // per slot (with prune), 32 B: packed kept spans (or SPANS_NONE), then tdesc
    const float4* rec;             // splat records (three planes of S)
    uint32_t S;
    uint32_t n_per_view;           // slot = view * n_per_view + Gaussian
    int tile_w, tile_h, prune;
    uint16_t* masks;               // per entry: the supertile's tiles it keeps (bit = row * 4 + col)
    uint32_t* chunk_cnt;           // [tile position][chunk_stride] entries per chunk, scanned in place
    uint32_t chunk_stride;         // supertile_chunks(cap)
    uint32_t* plane_tot;           // [tile position] entries with that bit
    uint32_t* vals_out;            // tile lists: slots
    uint32_t cap;                  // capacity of vals_out (and of the entries)
    uint2* ranges;                 // [global CTA tile] list range in vals_out; zeroed by the caller
    int* overflow;
};
// chunk_cnt's row length for up to `entries` entries.
size_t supertile_chunks(size_t entries);
// Per entry the 16-tile mask, the per-chunk counts and their scans, then the
// tile lists and the ranges of every tile that some entry's supertile holds.
void launch_supertile_lists(const SupertileArgs& a, cudaStream_t st);

// blend.cu
struct BlendArgs {
    const DevCam* cams;
    int nviews;
    const uint32_t* total_tiles;   // device scalar (or null -> total_tiles_host)
    int total_tiles_host;
    const uint2* ranges;
    const uint32_t* pair_vals;
    const float4* rec;
    uint32_t n_per_view;
    float bg[3];
    float* rgb;
    float* final_t;
    int* last;
    const float* dl;
    float4* acc;
    uint32_t* work;                // dynamic tile counter (zeroed by the launcher)
    int rect_filter;               // per-pixel reference-tile membership test
    int empty_tile_black;          // pixels of empty reference tiles render 0, not bg
    int pixels_per_thread;         // 1 or 2 vertically adjacent pixels per thread
    float* tstore;                 // store-all variant only: T per (list position, tile pixel)
    int bg_start;                  // preview compositing (rasterizer.rs:133): colour starts at bg and
                                   // the output is that sum, bg not scaled by the final T
    float one;                     // 1.0f, read at run time: the packed-lane kernels add
                                   // products as fma(product, one, acc) so that the code
                                   // generator cannot fuse the multiply into the add
};
void launch_blend_forward(const BlendArgs& a, int tile_w, int tile_h, int batch, cudaStream_t st);
void launch_blend_backward(const BlendArgs& a, int tile_w, int tile_h, int batch, cudaStream_t st);
void launch_blend_store_all(const BlendArgs& a, bool fwd, cudaStream_t st);
// Largest relative difference of the backward's SFU exponential from the
// forward's exp over n points on [lo, hi] (float bits, atomicMax into *out).
void launch_exp_sfu_error(float lo, float hi, uint32_t n, unsigned int* out, cudaStream_t st);
// (pixel, splat) pairs the forward and backward blends of a pass evaluated,
// from its final T, last contributors and tile ranges: out[0] forward,
// out[1] backward (added to; u64).
void launch_evaluated_pairs(const DevCam* cams, int nviews, const uint2* ranges, const float* final_t, const int* last,
                            int tile_w, int tile_h, unsigned long long* out, cudaStream_t st);

// raster.cu: preview framebuffer (colour, 1 - T) as RGBA f32 or sRGB RGBA8.
void launch_pack_framebuffer(const float* rgb, const float* final_t, size_t npix, int srgb8, void* out, cudaStream_t st);
// sfm.cu: gaussians_from_sfm (sfm.rs:365-450) from device-resident points
// (xyz n*3 f64, rgb n*3 u8) into parameter planes [NPL][cap]. *bad_host is set
// when a coordinate is not finite (the planes then hold no defined values).
int sfm_init_planes(const double* xyz, const uint8_t* rgb, int n, float4* planes, int cap, SfmScratch& w, int grid,
                    cudaStream_t st, int* bad_host, cudaError_t* err);
// 8-bit sRGB RGBA -> linear RGBA f32 (images.rs:67-72).
void launch_srgb8_to_linear(const void* rgba8, size_t npix, float* out, cudaStream_t st);

// ply.cu: io::ply codecs (src/io/ply.rs) on device-resident planes.
struct PlyField {
    uint32_t offset;   // byte offset in the vertex record
    uint8_t width;     // 1, 2, 4 or 8 bytes
    int16_t target;    // Gaussian3D record index, -1 = skipped
};
struct PlyLayout {
    int format = 2;    // 0 binary LE, 1 binary BE, 2 ascii
    size_t count = 0;  // vertices
    size_t stride = 0; // bytes per binary vertex record
    size_t body = 0;   // byte offset of the body
    std::vector<PlyField> fields;
};
std::string ply_header(size_t n);
int parse_ply(const std::vector<uint8_t>& data, PlyLayout& layout, std::string& err);
void decode_ply_ascii(const std::vector<uint8_t>& data, const PlyLayout& layout, float* out /* count * 59 */);
void launch_pack_ply(const float4* params, int n, int cap, float* out /* n * 62 */, cudaStream_t st);
void launch_pack_splat(const float4* params, int n, int cap, void* out /* n * 32 bytes */, cudaStream_t st);
void launch_unpack_ply(const uint8_t* body, size_t stride, int n, const PlyField* fields, int nfields, int big_endian,
                       float4* params, int cap, cudaStream_t st);

// loss.cu
// The loss kernel needs more dynamic shared memory than the default limit; the
// limit is a per-device function attribute, set on the current device the
// first time this is called there (under a mutex; later calls return at once).
cudaError_t prepare_loss_kernel();
// Prepares the current device (above), then enqueues the loss kernels; exact:
// the reference's separate multiply and add in the blurs (else fused).
cudaError_t launch_loss(const DevCam* cams, int nviews, int total_blocks, const float* rgb, float lambda,
                        float* dl, float* partials, float* losses, const uint32_t* total_dev,
                        bool exact, cudaStream_t st);

// geom.cu
struct AdamArgs {
    float4* params;
    float4* m1;
    float4* m2;
    float* grad_accum;
    uint32_t* grad_denom;
    float lr[NPL * 4];
    float b1, b2, one_minus_b1, one_minus_b2, bc1, bc2, eps;
    uint32_t denom_inc;
    const int* skip_flag;   // when non-null and *skip_flag != 0 the update is skipped
    const float* bc_dev;    // when non-null, (bc1, bc2) are read from device memory
    int mstride;            // plane stride (Gaussians) of m1 / m2
};
// gv: per-slot scratch of 4 float4 planes (S = n * nviews slots).
void launch_geometry(const float4* params, int n, int cap, const DevCam* cams, int nviews,
                     const uint32_t* cnt, const float4* acc, const float4* rec, const float4* gcache, float4* gv,
                     float4* grads, int accumulate, cudaStream_t st);
void launch_geometry_adam(const DevCam* cams, int nviews, int n, int cap, const uint32_t* cnt,
                          const float4* acc, const float4* rec, const float4* gcache, float4* gv, const AdamArgs& a,
                          cudaStream_t st);
void launch_adam(int n, int cap, const float4* grads, const AdamArgs& a, cudaStream_t st);
void launch_reset_opacities(float4* params, int n, int cap, cudaStream_t st);

// densify.cu
struct DensifyArgs {
    const float4* params;
    int n, cap;
    const float* grad_accum;
    const uint32_t* grad_denom;
    float prune_opacity, grad_threshold, extent;
    uint64_t max_gaussians;
};
// Writes the new Gaussians into `out` (grown as needed; its plane stride is
// returned in *out_cap) and the new count in *n_out. Synchronises `st`.
cudaError_t densify_and_prune(const DensifyArgs& a, DBuf& out, int* out_cap, DBuf& scratch,
                              int* n_out, cudaStream_t st);

}  // namespace rgs
