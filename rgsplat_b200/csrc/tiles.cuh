// tiles.cuh -- the conservative (tile, splat) rejection test shared by the
// projection (pruned tile counts), the pair emission and the blend kernels.
// All three evaluate it on the same stored floats, so they agree exactly on
// which (tile, splat) pairs are dropped.
#pragma once
#include "rgs_internal.cuh"

namespace rgs {

// Power below which alpha = min(op * e^power, 0.99) < 1/255 for this opacity
// (op <= 1 and op >= 1/255 for every projected splat), with a 1 % margin in
// alpha that covers the rounding of op * exp and of this logarithm.
__device__ __forceinline__ float power_floor(float op) { return -__logf(255.0f * op) - 0.01f; }

// Conservative tile test: rejects only if every pixel centre of the box has
// power = -q/2 < thr, where q = a dx^2 + 2 b dx dy + c dy^2 (the reference's
// expression, backward.rs:340). The box minimum of the convex q lies on an
// edge unless the splat centre is inside; on each edge the minimiser of the
// 1-D quadratic is clamped to the edge. Only well-conditioned conics
// (ac - b^2 >= ac / 100, so the float evaluation of q here and per pixel is
// accurate to ~1e-4 relative) are tested, with a 1e-3 margin; anything else
// (including NaN) is kept. The per-splat part (the edge minimisers' slopes
// b/c, b/a) is formed once by tile_test_setup.
struct TileTest {
    float sx, sy, a, b, c, rb, ra, thr;
    bool testable;
};

__device__ __forceinline__ TileTest tile_test_setup(float sx, float sy, float a, float b, float c, float thr) {
    TileTest t;
    t.sx = sx; t.sy = sy; t.a = a; t.b = b; t.c = c; t.thr = thr;
    t.testable = a > 0.0f && c > 0.0f && (a * c - b * b) >= 0.01f * (a * c);
    t.rb = t.testable ? b / c : 0.0f;
    t.ra = t.testable ? b / a : 0.0f;
    return t;
}

__device__ __forceinline__ bool tile_rejects(const TileTest& t, float x0c, float x1c, float y0c, float y1c) {
    if (!t.testable) return false;
    const float lx = x0c - t.sx, hx = x1c - t.sx, ly = y0c - t.sy, hy = y1c - t.sy;
    if (lx <= 0.0f && hx >= 0.0f && ly <= 0.0f && hy >= 0.0f) return false;
    float best = __int_as_float(0x7f800000);
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const float dx = e ? hx : lx;
        const float dy = fminf(fmaxf(-t.rb * dx, ly), hy);
        best = fminf(best, t.a * dx * dx + 2.0f * t.b * dx * dy + t.c * dy * dy);
        const float ey = e ? hy : ly;
        const float ex = fminf(fmaxf(-t.ra * ey, lx), hx);
        best = fminf(best, t.a * ex * ex + 2.0f * t.b * ex * ey + t.c * ey * ey);
    }
    return best * 0.999f > -2.0f * t.thr;
}

// Pixel-centre box of CTA tile (tx, ty), clipped to the image.
__device__ __forceinline__ void cta_tile_box(int tx, int ty, int tw, int th, int width, int height, float& x0c, float& x1c,
                                             float& y0c, float& y1c) {
    x0c = (float)(tx * tw) + 0.5f;
    x1c = (float)(min(tx * tw + tw, width) - 1) + 0.5f;
    y0c = (float)(ty * th) + 0.5f;
    y1c = (float)(min(ty * th + th, height) - 1) + 0.5f;
}

// ---- per-row kept spans (pair pruning) -----------------------------------
// The tiles of one CTA-tile row that the test above can keep are those whose
// pixel-centre box meets the ellipse E = {q <= T}, T = -2 thr / 0.999: for
// the row's band of pixel-centre rows [ly, hy] (relative to the centre), the
// x-extent of E within the band is [xl, xr], where xr is E's rightmost point
// if its y lies in the band, else the larger root of q(x, y_edge) = T at the
// band edge nearest to it (E's right boundary is concave in y), and likewise
// for xl (the roots are formed with 1/a, within an ulp of the quotient). The
// span is computed with T enlarged by 2 % and widened by half a pixel, so it
// contains every tile the per-tile test keeps with a margin far above float
// rounding; the blend still applies the per-tile test.
struct SpanSetup {
    float sx, sy, a, b, c, T, xr, yr, ia;  // ia = 1 / a
    bool testable;
};

__device__ __forceinline__ SpanSetup span_setup(float sx, float sy, float a, float b, float c, float thr) {
    SpanSetup u;
    u.sx = sx; u.sy = sy; u.a = a; u.b = b; u.c = c;
    u.testable = a > 0.0f && c > 0.0f && (a * c - b * b) >= 0.01f * (a * c);
    u.T = -2.0f * thr / 0.999f * 1.02f;
    const float det = a * c - b * b;
    u.xr = u.testable ? sqrtf(u.T * c / det) : 0.0f;
    u.yr = u.testable ? -b / c * u.xr : 0.0f;
    u.ia = u.testable ? 1.0f / a : 0.0f;
    return u;
}

// Kept CTA-tile columns [c0, c1) of tile row ty, clipped to [cx0, cx1).
__device__ __forceinline__ void kept_cols(const SpanSetup& u, int ty, int tw, int th, int height, int cx0, int cx1, int& c0,
                                          int& c1) {
    c0 = cx0;
    c1 = cx1;
    if (!u.testable) return;
    const float ly = ((float)(ty * th) + 0.5f) - u.sy;
    const float hy = ((float)(min(ty * th + th, height) - 1) + 0.5f) - u.sy;
    float xr, xl;
    const float er = fminf(fmaxf(u.yr, ly), hy);
    if (er == u.yr) {
        xr = u.xr;
    } else {
        const float disc = u.b * u.b * er * er - u.a * (u.c * er * er - u.T);
        if (!(disc >= 0.0f)) {
            c1 = c0;
            return;
        }
        xr = (-u.b * er + sqrtf(disc)) * u.ia;
    }
    const float el = fminf(fmaxf(-u.yr, ly), hy);
    if (el == -u.yr) {
        xl = -u.xr;
    } else {
        const float disc = u.b * u.b * el * el - u.a * (u.c * el * el - u.T);
        if (!(disc >= 0.0f)) {
            c1 = c0;
            return;
        }
        xl = (-u.b * el - sqrtf(disc)) * u.ia;
    }
    // pixel-space interval, widened by half a pixel; a tile's pixel centres
    // span [tx * tw + 0.5, tx * tw + tw - 0.5]
    const float X0 = u.sx + xl - 0.5f, X1 = u.sx + xr + 0.5f;
    // tile widths are powers of two, so multiplying by 1 / tw is exact
    const float itw = 1.0f / (float)tw;
    const float f0 = floorf((X0 + 0.5f) * itw - 1.0f);
    const float f1 = floorf((X1 - 0.5f) * itw) + 1.0f;
    c0 = (int)fminf(fmaxf(f0, (float)cx0), (float)cx1);
    c1 = (int)fminf(fmaxf(f1, (float)cx0), (float)cx1);
    if (c1 < c0) c1 = c0;
}

}  // namespace rgs
