// oracle/capi.cpp -- C entry points of the CPU oracle (TEST INFRASTRUCTURE ONLY).
//
// Called through ctypes by tests/ and by bench.py's CPU-baseline leg. Gaussians
// are the reference's AoS record (Gaussian3D, src/math/mod.rs:27-46: 59 floats),
// gradients the GaussianGrad record (src/cpu/backward.rs:33-41: 60 floats).
#include <omp.h>

#include "oracle.hpp"
#include "ply.hpp"
#include "sfm.hpp"

namespace orc {
int g_libm_math = 0;
}

using namespace orc;
typedef orc::CameraIn orc_camera;
typedef orc::TrainCfgIn orc_train_config;

template <class T> static int rab(const T* g, size_t n, const orc_camera* cam, const T* target, const T* bg, T lambda, T* loss, T* grads, T* rendered, T* final_t, int32_t* last, T* dl, T* acc) {
    if (!cam || (!g && n)) return ORC_EINVAL;
    Cam<T> c;
    if (!make_cam(*cam, c)) return ORC_EINVAL;
    DebugOut<T> d{rendered, final_t, last, dl, acc};
    return render_and_backward((const Gaussian<T>*)g, n, c, target, bg, lambda, loss, (Grad<T>*)grads, &d);
}

extern "C" {

int orc_set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
}
void orc_set_libm_math(int on) { g_libm_math = on ? 1 : 0; }
float orc_expf(float x) { return t_exp(x); }
float orc_logf(float x) { return t_log(x); }
void orc_expf_array(const float* x, float* y, size_t n) {
    for (size_t i = 0; i < n; ++i) y[i] = t_exp(x[i]);
}
void orc_expf_fast_array(const float* x, float* y, size_t n) {
    for (size_t i = 0; i < n; ++i) y[i] = t_expa(x[i]);
}
void orc_logf_array(const float* x, float* y, size_t n) {
    for (size_t i = 0; i < n; ++i) y[i] = t_log(x[i]);
}
float orc_sigmoid_f(float x) { return sigmoid(x); }
float orc_logit_f(float x) { return logit(x); }

int orc_render_and_backward_f(const float* g, size_t n, const orc_camera* cam, const float* target, const float* bg, float lambda, float* loss, float* grads, float* rendered, float* final_t, int32_t* last, float* dl, float* acc) {
    return rab<float>(g, n, cam, target, bg, lambda, loss, grads, rendered, final_t, last, dl, acc);
}
int orc_render_and_backward_d(const double* g, size_t n, const orc_camera* cam, const double* target, const double* bg, double lambda, double* loss, double* grads, double* rendered, double* final_t, int32_t* last, double* dl, double* acc) {
    return rab<double>(g, n, cam, target, bg, lambda, loss, grads, rendered, final_t, last, dl, acc);
}

int orc_render_color_f(const float* g, size_t n, const orc_camera* cam, const float* bg, float* rgb, float* final_t, int32_t* last) {
    Cam<float> c;
    if (!cam || !make_cam(*cam, c)) return ORC_EINVAL;
    return render_color((const Gaussian<float>*)g, n, c, bg, rgb, final_t, last);
}

int orc_rasterize_f(const float* g, size_t n, const orc_camera* cam, const float* bg, float* rgba) {
    Cam<float> c;
    if (!cam || !make_cam(*cam, c)) return ORC_EINVAL;
    return rasterize((const Gaussian<float>*)g, n, c, bg, rgba);
}

int orc_linear_to_srgb(const float* x, size_t n, float* out) {
    for (size_t i = 0; i < n; ++i) out[i] = fm::linear_to_srgb(x[i]);
    return ORC_OK;
}

// images.rs:67-72: RGBA8 -> linear RGBA f32 (alpha linear)
// sfm.rs:365-450
int orc_gaussians_from_sfm(const double* xyz, const uint8_t* rgb, size_t n, float* out) {
    if (n && (!xyz || !rgb || !out)) return ORC_EINVAL;
    for (size_t i = 0; i < 3 * n; ++i)
        if (!std::isfinite(xyz[i])) return ORC_EINVAL;
    sfm::gaussians_from_sfm(xyz, rgb, n, out);
    return ORC_OK;
}
int orc_sfm_scales(const double* xyz, size_t n, float* out) {
    if (n && (!xyz || !out)) return ORC_EINVAL;
    sfm::estimate_initial_scales(xyz, n, out);
    return ORC_OK;
}
long orc_rust_binary_search(const double* xs, size_t n, double t, int* ok) {
    bool b = false;
    const size_t r = sfm::rust_binary_search(xs, n, t, &b);
    *ok = b ? 1 : 0;
    return (long)r;
}
// sfm.rs:147-183; *n_out = point count, records copied when cap holds them
int orc_parse_points3d_bin(const uint8_t* data, size_t size, double* xyz, uint8_t* rgb, size_t cap, size_t* n_out) {
    std::vector<sfm::Point> pts;
    if (sfm::parse_points3d_bin(data, size, pts)) return ORC_EINVAL;
    *n_out = pts.size();
    if (xyz && rgb && cap >= pts.size())
        for (size_t i = 0; i < pts.size(); ++i) {
            std::memcpy(xyz + 3 * i, pts[i].xyz, 24);
            std::memcpy(rgb + 3 * i, pts[i].rgb, 3);
        }
    return ORC_OK;
}

int orc_srgb8_to_linear(const uint8_t* rgba8, size_t npix, float* out) {
    for (size_t i = 0; i < npix * 4; ++i) {
        const float x = (float)rgba8[i] / 255.0f;
        out[i] = i % 4 == 3 ? x : fm::srgb_to_linear(x);
    }
    return ORC_OK;
}

int orc_to_u8_srgb(const float* rgba, size_t n_values, uint8_t* out) {
    to_u8_srgb(rgba, n_values, out);
    return ORC_OK;
}

// io::ply (src/io/ply.rs): encoders return the byte count and fill `out` when
// it holds at least that many bytes; the decoder fills up to `cap` records.
long orc_save_ply(const float* g, size_t n, uint8_t* out, size_t cap) {
    auto b = ply::save_ply(g, n);
    if (out && cap >= b.size()) std::memcpy(out, b.data(), b.size());
    return (long)b.size();
}
long orc_save_splat(const float* g, size_t n, uint8_t* out, size_t cap) {
    auto b = ply::save_splat(g, n);
    if (out && cap >= b.size()) std::memcpy(out, b.data(), b.size());
    return (long)b.size();
}
int orc_load_ply(const uint8_t* data, size_t size, float* out, size_t cap, size_t* n_out) {
    std::vector<float> v;
    int rc = ply::load_ply(data, size, v);
    if (rc) return rc;
    const size_t n = v.size() / 59;
    *n_out = n;
    if (out && cap >= n) std::memcpy(out, v.data(), v.size() * 4);
    return ORC_OK;
}

int orc_photometric_loss_grad_f(const float* rendered, const float* target, int w, int h, float lambda, float* loss, float* dl) {
    if (w <= 0 || h <= 0) return ORC_EINVAL;
    *loss = photometric_loss_grad(rendered, target, w, h, lambda, dl);
    return ORC_OK;
}
int orc_photometric_loss_grad_d(const double* rendered, const double* target, int w, int h, double lambda, double* loss, double* dl) {
    if (w <= 0 || h <= 0) return ORC_EINVAL;
    *loss = photometric_loss_grad(rendered, target, w, h, lambda, dl);
    return ORC_OK;
}

// Per-Gaussian projection (backward.rs:210-280). rec: 16 floats per Gaussian
// (sx, sy, conic3, cov2d3, color3, raw_color3, opacity, depth); rect: tile rect.
int orc_project_f(const float* g, size_t n, const orc_camera* cam, int32_t* visible, float* rec, int32_t* rect) {
    Cam<float> c;
    if (!cam || !make_cam(*cam, c)) return ORC_EINVAL;
    const Gaussian<float>* gs = (const Gaussian<float>*)g;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) {
        Splat<float> s;
        bool v = project(gs[i], (int)i, c, s);
        visible[i] = v ? 1 : 0;
        float* r = rec + (size_t)i * 16;
        int32_t* q = rect + (size_t)i * 4;
        if (!v) {
            for (int k = 0; k < 16; ++k) r[k] = 0.0f;
            q[0] = q[1] = q[2] = q[3] = 0;
            continue;
        }
        r[0] = s.sx; r[1] = s.sy;
        r[2] = s.conic[0]; r[3] = s.conic[1]; r[4] = s.conic[2];
        r[5] = s.cov2d[0]; r[6] = s.cov2d[1]; r[7] = s.cov2d[2];
        r[8] = s.color[0]; r[9] = s.color[1]; r[10] = s.color[2];
        r[11] = s.raw_color[0]; r[12] = s.raw_color[1]; r[13] = s.raw_color[2];
        r[14] = s.opacity; r[15] = s.depth;
        q[0] = s.tx0; q[1] = s.ty0; q[2] = s.tx1; q[3] = s.ty1;
    }
    return ORC_OK;
}

// Tile lists (backward.rs:172-208) as CSR over Gaussian indices. Call with
// entries == NULL to size; *n_pairs receives the total.
int orc_bin_f(const float* g, size_t n, const orc_camera* cam, int64_t* n_pairs, int32_t* tile_offsets, int32_t* entries, int64_t cap) {
    Cam<float> c;
    if (!cam || !make_cam(*cam, c)) return ORC_EINVAL;
    Binned<float> B;
    int rc = project_and_bin((const Gaussian<float>*)g, n, c, B);
    if (rc) return rc;
    int64_t total = 0;
    for (auto& L : B.tile_lists) total += (int64_t)L.size();
    *n_pairs = total;
    if (!entries) return ORC_OK;
    if (cap < total) return ORC_ESIZE;
    int64_t k = 0;
    for (size_t t = 0; t < B.tile_lists.size(); ++t) {
        tile_offsets[t] = (int32_t)k;
        for (int si : B.tile_lists[t]) entries[k++] = B.splats[si].gi;
    }
    tile_offsets[B.tile_lists.size()] = (int32_t)k;
    return ORC_OK;
}

int orc_adam_step_f(float* g, size_t n, const float* grads, float* m1, float* m2, float* grad_accum, uint32_t* grad_denom, uint64_t* t, const orc_train_config* cfg) {
    adam_step((Gaussian<float>*)g, n, (const Grad<float>*)grads, m1, m2, grad_accum, grad_denom, t, *cfg);
    return ORC_OK;
}

int64_t orc_densify_and_prune_f(const float* g, size_t n, float* out, const float* grad_accum, const uint32_t* grad_denom, const orc_train_config* cfg, float extent) {
    return (int64_t)densify_and_prune((const Gaussian<float>*)g, n, (Gaussian<float>*)out, grad_accum, grad_denom, *cfg, extent);
}

void orc_reset_opacities_f(float* g, size_t n) { reset_opacities((Gaussian<float>*)g, n); }
float orc_estimate_scene_extent_f(const float* g, size_t n) { return estimate_scene_extent((const Gaussian<float>*)g, n); }

int orc_project_wgsl_f(const float* g, size_t n, const orc_camera* cam, float* splats10, uint32_t* keys) {
    Cam<float> c;
    if (!cam || !make_cam(*cam, c)) return ORC_EINVAL;
    const Gaussian<float>* gs = (const Gaussian<float>*)g;
    for (size_t i = 0; i < n; ++i) project_wgsl(gs[i], c, ((SplatInfo2D*)splats10)[i], keys[i]);
    return ORC_OK;
}
void orc_composite_f(const float* splats10, size_t n, int w, int h, const float* bg, float* rgb) {
    composite((const SplatInfo2D*)splats10, n, w, h, bg, rgb);
}

// Small math kernels, exposed for the reference's inline unit tests.
void orc_mat_from_quat_f(const float* q, float* m9) {
    M3<float> r = mat_from_quat(q);
    std::memcpy(m9, r.m, 36);
}
void orc_to_rotation_matrix_f(const float* q, float* m9) {
    M3<float> r = to_rotation_matrix(q);
    std::memcpy(m9, r.m, 36);
}
void orc_quat_normalize_f(const float* q, float* o) { qnormalize(q, o); }
void orc_rotation_jacobian_f(const float* q, float* m36) {
    M3<float> d[4];
    rotation_jacobian(q, d);
    for (int k = 0; k < 4; ++k) std::memcpy(m36 + 9 * k, d[k].m, 36);
}
void orc_build_cov3d_f(const float* s, const float* q, float* m9) {
    M3<float> r = build_cov3d(s, q);
    std::memcpy(m9, r.m, 36);
}
void orc_backprop_cov3d_f(const float* s, const float* q, const float* g9, float* dls, float* dq) {
    M3<float> g;
    std::memcpy(g.m, g9, 36);
    backprop_cov3d(s, q, g, dls, dq);
}
void orc_sh_basis_f(const float* d, float* b16) { sh_basis(d, b16); }
void orc_sh_basis_grad_f(const float* d, float* g48) {
    float g[16][3];
    sh_basis_grad(d, g);
    std::memcpy(g48, g, sizeof(g));
}
void orc_eval_sh_deg3_f(const float* coeffs, const float* dir, float* rgb) {
    float b[16], raw[3];
    sh_basis(dir, b);
    eval_sh_raw(coeffs, b, raw);
    for (int i = 0; i < 3; ++i) rgb[i] = rclamp(raw[i], 0.0f, 1.0f);
}
// SSIM of one channel (backward.rs:697-756): returns the sum, writes its gradient.
float orc_ssim_channel_f(const float* x, const float* y, int w, int h, float* grad) {
    std::vector<float> k = gaussian_kernel_1d<float>(5, 1.5f);
    return ssim_channel(x, y, w, h, k, grad);
}
void orc_gaussian_kernel_1d_f(int radius, float sigma, float* out) {
    std::vector<float> k = gaussian_kernel_1d<float>(radius, sigma);
    std::memcpy(out, k.data(), k.size() * sizeof(float));
}

}  // extern "C"
