/*
 * rgsplat_debug.h -- introspection entry points of librgsplat_b200.
 *
 * These expose the intermediate state of one view of the training step (the
 * reference's private `project_and_bin`, `forward_pass` and `backward_pass`
 * caches, src/cpu/backward.rs:172-512) so parity tests can compare them with a
 * CPU restatement element by element. They are not needed to train.
 */
#ifndef RGSPLAT_DEBUG_H
#define RGSPLAT_DEBUG_H

#include "rgsplat.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-Gaussian projection (backward.rs:210-280). rec10: n * 10 floats
 * (sx, sy, conic a, b, c, r, g, b, opacity, depth); rect4: n * 4 ints, the
 * reference tile rectangle [tx0, ty0, tx1, ty1) (backward.rs:275-278);
 * visible[i] = 0 when culled. */
int rgs_debug_project(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, int32_t* visible,
                      float* rec10, int32_t* rect4);

/* Tile lists of project_and_bin (backward.rs:172-208) over the context's CTA
 * tiles (16x16 by default), as CSR: tile t holds entries[offsets[t] ..
 * offsets[t+1]) (Gaussian indices, front to back). offsets: tiles + 1 ints.
 * Call with entries == NULL to get *n_pairs. */
int rgs_debug_tile_lists(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, uint64_t* n_pairs,
                         int32_t* offsets, int32_t* entries, size_t cap);

/* The same lists pruned as the zero-background render and training paths bin
 * them: each splat only in the tiles of its rows' kept spans (a conservative
 * superset of the tiles whose pixels its alpha can reach). *n_pairs is the
 * pair count the projection made, which the lists must hold exactly. */
int rgs_debug_pruned_tile_lists(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera,
                                uint64_t* n_pairs, int32_t* offsets, int32_t* entries, size_t cap);

/* forward_pass caches (backward.rs:296-385): rgb w*h*3, final T w*h, last
 * contributor (index into the pixel's tile list, -1 if none) w*h. */
int rgs_debug_forward(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, const float bg[3],
                      float* rgb, float* final_t, int32_t* last);

/* backward_pass output (backward.rs:391-512) merged per Gaussian: n * 9 floats
 * (d color[3], d opacity, d conic[3], d sx, d sy), plus dL/dpixel (w*h*3). */
int rgs_debug_backward(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, const float* target_rgba,
                       const float bg[3], float lambda, float* acc9, float* dl_dpix);

/* Largest relative difference between the backward blend's SFU exponential
 * and the forward's exact exp (the one the oracle restates) over n points on
 * [lo, hi], -8 <= lo <= hi <= 0: the bound behind the backward's rule of
 * deciding alpha >= 1/255 and alpha > 0.99 with the exact exp whenever the
 * SFU value lies within 4e-6 relative of either threshold. */
int rgs_debug_exp_sfu_error(rgs_ctx* ctx, float lo, float hi, uint32_t n, float* max_rel);

/* Pixels of the view at position k of the trainer's most recent batched pass
 * (rgs_trainer_step or rgs_trainer_backward with RGS_STEP_BATCHED that ran as
 * one view group), read from the batch's own buffers: rgb w*h*3, final T w*h
 * and dL/dpixel w*h*3, each may be NULL. This is forward_pass's output and
 * photometric_loss_grad's gradient (backward.rs:296-385, 646-693) for every
 * view of a batch, for comparison with per-view reference renders.
 * RGS_ERR_INVALID_ARG when no such pass holds the buffers (another call has
 * written them since, or the batch ran as several view groups) or k is out of
 * range. */
int rgs_debug_trainer_batch_pixels(rgs_ctx* ctx, size_t k, float* rgb, float* final_t, float* dl_dpix);

#ifdef __cplusplus
}
#endif
#endif /* RGSPLAT_DEBUG_H */
