/*
 * tileink_b200 differentiable rendering: dL/d(control points, colours, blur
 * sigma) for closed cubic paths drawn into one Gaussian blur group over an
 * opaque background, with L the mean squared error against a target image.
 *
 * Reference: the `backward()` entry the tileink Rust host would bind beside
 * NativeRenderer::render_to_image (src/native/renderer.rs:177-190); the
 * forward is the scene Canvas::push_blur_group (src/canvas/layers.rs:205-212)
 * + Canvas::push_path (src/canvas/paths.rs:65-156) records.
 *
 * The differentiable forward is the same scan / coarse path as tk_render
 * (identical segments and PTCL), followed by fine raster, blur and the group
 * composite in f32 without the RGBA8 rounding between stages, so that the
 * rendered image is a smooth function of the parameters:
 *   coverage  exact signed area A per pixel, c = min(|A|, 1) (nonzero)
 *   layer     premultiplied src-over of the paths in order onto transparent
 *   blur      separable Gaussian, taps exp(-k^2 / 2 sigma^2) normalised over
 *             |k| <= r, r = ceil(3 sigma) fixed by the forward, zero outside
 *             the canvas
 *   image     blurred layer src-over `background`
 *   loss      mean over pixels and the four channels of (image - target)^2
 * The flattening (how many lines, at which curve parameters) is fixed by the
 * forward; gradients are those of the function with that subdivision held
 * fixed, as in any differentiable rasterizer.
 */
#ifndef TILEINK_B200_DIFF_H
#define TILEINK_B200_DIFF_H

#include "tileink.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tk_diff_scene {
    uint32_t width, height;
    uint32_t path_count;
    uint32_t cubics_per_path;  /* points per path: 1 + 3 * cubics_per_path */
    const float* points;       /* [path][point][x, y], canvas pixels; path p is
                                  move_to(pt 0), cubic_to(pts 3k+1..3k+3) for
                                  k < cubics_per_path, close */
    const float* colors;       /* [path][r, g, b, a] straight, in [0, 1] */
    float sigma;               /* blur group sigma (> 0), or 0 for no blur group */
    float tolerance;           /* flattening tolerance, pixels */
    float background[4];       /* premultiplied RGBA under the group */
    /* Pixel rows [loss_row0, loss_row1) of the loss (loss_row1 == 0: every
     * row). The mean still divides by all W * H * 4 values, so losses and
     * gradients of row ranges that partition the image sum to the whole
     * image's: ranks of a row-split objective all-reduce (sum) them. */
    uint32_t loss_row0, loss_row1;
} tk_diff_scene;

/* Renders `scene`, returns the loss against `target` ([height][width][4]
 * premultiplied f32, host) and optionally the image (same layout). Keeps what
 * tk_diff_backward needs on the device. */
int32_t tk_diff_forward(tk_ctx* ctx, const tk_diff_scene* scene, const float* target, double* loss,
                        float* image);

/* Gradients of the last tk_diff_forward's loss: d_points like `points`,
 * d_colors like `colors`, d_sigma one value (0 without a blur group). Host
 * outputs; any may be NULL. Coverage is recomputed per tile, nothing per
 * pixel and record is kept from the forward. */
int32_t tk_diff_backward(tk_ctx* ctx, float* d_points, float* d_colors, float* d_sigma);

/* The forward's flattening with the weights of every line endpoint over the
 * control points: endpoint e of line l is
 *   sum_i endpoint_weights[8 l + 4 e + i] * point[endpoint_point[2 l + e] + i]
 * (global point indices across paths). Returns the line count; writes at most
 * `capacity` lines. Lines are those tk_canvas_push_path produces for the same
 * paths. */
uint64_t tk_diff_flatten(const tk_diff_scene* scene, tk_line* lines, uint32_t* endpoint_point,
                         float* endpoint_weights, uint64_t capacity);

#ifdef __cplusplus
}
#endif

#endif /* TILEINK_B200_DIFF_H */
