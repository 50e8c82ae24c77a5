// Layout table of every struct the C ABI passes (include/tileink.h,
// tileink_canvas.h, tileink_diff.h), so that a binding can check its own
// declarations against the compiled library field by field.
#include <cstddef>

#include "../../include/tileink.h"
#include "../../include/tileink_canvas.h"
#include "../../include/tileink_diff.h"

namespace {

#define S(T) tk_abi_field{#T, "", 0u, uint32_t(sizeof(T))}
#define F(T, m) tk_abi_field{#T, #m, uint32_t(offsetof(T, m)), uint32_t(sizeof(static_cast<T*>(nullptr)->m))}

const tk_abi_field kLayout[] = {
    S(tk_abi_field),
    F(tk_abi_field, type), F(tk_abi_field, field), F(tk_abi_field, offset), F(tk_abi_field, size),
    S(tk_image_desc),
    F(tk_image_desc, premul_rgba8), F(tk_image_desc, width), F(tk_image_desc, height),
    S(tk_affine),
    F(tk_affine, a), F(tk_affine, b), F(tk_affine, c), F(tk_affine, d), F(tk_affine, e), F(tk_affine, f),
    S(tk_line),
    F(tk_line, path_id), F(tk_line, pad), F(tk_line, p0), F(tk_line, p1),
    S(tk_path_record),
    F(tk_path_record, path_id), F(tk_path_record, line_count), F(tk_path_record, line_start),
    F(tk_path_record, flags), F(tk_path_record, data_offset), F(tk_path_record, data_len),
    F(tk_path_record, tile_x0), F(tk_path_record, tile_y0), F(tk_path_record, tile_x1), F(tk_path_record, tile_y1),
    F(tk_path_record, segment_start), F(tk_path_record, segment_capacity), F(tk_path_record, segment_count),
    F(tk_path_record, transform),
    S(tk_pixel_bounds),
    F(tk_pixel_bounds, x0), F(tk_pixel_bounds, y0), F(tk_pixel_bounds, x1), F(tk_pixel_bounds, y1),
    S(tk_draw_record),
    F(tk_draw_record, path_id), F(tk_draw_record, glyph_run_id), F(tk_draw_record, sdf_offset),
    F(tk_draw_record, sdf_len), F(tk_draw_record, sdf_shadow_offset), F(tk_draw_record, sdf_shadow_len),
    F(tk_draw_record, brush_offset), F(tk_draw_record, brush_len), F(tk_draw_record, tag),
    F(tk_draw_record, fill_rule), F(tk_draw_record, pixel_bounds), F(tk_draw_record, local_pixel_bounds),
    F(tk_draw_record, solid_rect), F(tk_draw_record, transform), F(tk_draw_record, inverse_transform),
    S(tk_layer_record),
    F(tk_layer_record, tag), F(tk_layer_record, draw), F(tk_layer_record, payload),
    S(tk_ptcl_record),
    F(tk_ptcl_record, tag), F(tk_ptcl_record, backdrop), F(tk_ptcl_record, fill_rule),
    F(tk_ptcl_record, segment_start), F(tk_ptcl_record, segment_end), F(tk_ptcl_record, color),
    S(tk_line_segment),
    F(tk_line_segment, p0x), F(tk_line_segment, p0y), F(tk_line_segment, p1x), F(tk_line_segment, p1y),
    F(tk_line_segment, y_edge),
    S(tk_segment_range),
    F(tk_segment_range, start), F(tk_segment_range, end),
    S(tk_tile_record),
    F(tk_tile_record, ptcl_count), F(tk_tile_record, ptcl_start), F(tk_tile_record, ptcl_end),
    F(tk_tile_record, glyph_count), F(tk_tile_record, glyph_start), F(tk_tile_record, glyph_end),
    S(tk_op),
    F(tk_op, kind), F(tk_op, batch_id), F(tk_op, layer_start), F(tk_op, layer_end), F(tk_op, sigma),
    F(tk_op, bounds),
    S(tk_scene_desc),
    F(tk_scene_desc, width), F(tk_scene_desc, height), F(tk_scene_desc, clear_color), F(tk_scene_desc, flags),
    F(tk_scene_desc, lines), F(tk_scene_desc, line_count), F(tk_scene_desc, paths), F(tk_scene_desc, path_count),
    F(tk_scene_desc, draw_count), F(tk_scene_desc, draws), F(tk_scene_desc, brush_blob),
    F(tk_scene_desc, brush_word_count), F(tk_scene_desc, layers), F(tk_scene_desc, layer_count),
    F(tk_scene_desc, draw_order_count), F(tk_scene_desc, draw_order), F(tk_scene_desc, draw_batch_ids),
    F(tk_scene_desc, ops), F(tk_scene_desc, op_count), F(tk_scene_desc, reserved), F(tk_scene_desc, sdf_blob),
    F(tk_scene_desc, sdf_word_count), F(tk_scene_desc, sdf_shadow_blob), F(tk_scene_desc, sdf_shadow_word_count),
    F(tk_scene_desc, images), F(tk_scene_desc, image_count), F(tk_scene_desc, image_reserved),
    S(tk_stats),
    F(tk_stats, lines), F(tk_stats, backdrop_len), F(tk_stats, segments), F(tk_stats, ptcl_records),
    F(tk_stats, tile_draw_refs), F(tk_stats, fill_particles), F(tk_stats, segment_visits), F(tk_stats, passes),
    F(tk_stats, tiles),
    S(tk_flatten_el),
    F(tk_flatten_el, verb), F(tk_flatten_el, path), F(tk_flatten_el, tolerance), F(tk_flatten_el, p),
    S(tk_stroke_polyline),
    F(tk_stroke_polyline, stroke), F(tk_stroke_polyline, element0), F(tk_stroke_polyline, element_count),
    F(tk_stroke_polyline, closed),
    S(tk_stroke_desc),
    F(tk_stroke_desc, path), F(tk_stroke_desc, polyline0), F(tk_stroke_desc, polyline_count),
    F(tk_stroke_desc, reserved), F(tk_stroke_desc, half_width), F(tk_stroke_desc, tolerance),
    F(tk_stroke_desc, transform),
    S(tk_flatten_desc),
    F(tk_flatten_desc, elements), F(tk_flatten_desc, element_count), F(tk_flatten_desc, path_elements),
    F(tk_flatten_desc, stroke_elements), F(tk_flatten_desc, stroke_element_count), F(tk_flatten_desc, polylines),
    F(tk_flatten_desc, polyline_count), F(tk_flatten_desc, stroke_count), F(tk_flatten_desc, strokes),
    S(tk_damage),
    F(tk_damage, full), F(tk_damage, rect_count), F(tk_damage, rects),
    S(tk_incremental_stats),
    F(tk_incremental_stats, total_tiles), F(tk_incremental_stats, dirty_tiles),
    F(tk_incremental_stats, full_redraw), F(tk_incremental_stats, reason),
    F(tk_incremental_stats, scan_reused), F(tk_incremental_stats, scanned_paths),
    S(tk_batch_info),
    F(tk_batch_info, width), F(tk_batch_info, height), F(tk_batch_info, tile_base), F(tk_batch_info, tile_count),
    F(tk_batch_info, path_base), F(tk_batch_info, draw_base), F(tk_batch_info, batch_base),
    F(tk_batch_info, line_base), F(tk_batch_info, layer_base), F(tk_batch_info, reserved),
    F(tk_batch_info, segment_base), F(tk_batch_info, pool_base), F(tk_batch_info, image_offset),
    S(tk_tune_result),
    F(tk_tune_result, scan_item_elems), F(tk_tune_result, tile_width), F(tk_tune_result, tile_height),
    F(tk_tune_result, candidates), F(tk_tune_result, candidate_elems), F(tk_tune_result, candidate_ms),
    S(tk_gradient_stop),
    F(tk_gradient_stop, offset), F(tk_gradient_stop, rgba),
    S(tk_brush_desc),
    F(tk_brush_desc, kind), F(tk_brush_desc, extend), F(tk_brush_desc, rgba), F(tk_brush_desc, p0),
    F(tk_brush_desc, p1), F(tk_brush_desc, r0), F(tk_brush_desc, r1), F(tk_brush_desc, stop_count),
    F(tk_brush_desc, stops),
    S(tk_sdf_shape),
    F(tk_sdf_shape, kind), F(tk_sdf_shape, cap), F(tk_sdf_shape, p0), F(tk_sdf_shape, p1), F(tk_sdf_shape, p2),
    F(tk_sdf_shape, radius), F(tk_sdf_shape, width), F(tk_sdf_shape, radii), F(tk_sdf_shape, widths),
    F(tk_sdf_shape, shadow), F(tk_sdf_shape, dash), F(tk_sdf_shape, flags), F(tk_sdf_shape, angle),
    S(tk_gen_params),
    F(tk_gen_params, width), F(tk_gen_params, height), F(tk_gen_params, paths), F(tk_gen_params, variant),
    F(tk_gen_params, sigma), F(tk_gen_params, jitter), F(tk_gen_params, flags), F(tk_gen_params, reserved),
    S(tk_diff_scene),
    F(tk_diff_scene, width), F(tk_diff_scene, height), F(tk_diff_scene, path_count),
    F(tk_diff_scene, cubics_per_path), F(tk_diff_scene, points), F(tk_diff_scene, colors), F(tk_diff_scene, sigma),
    F(tk_diff_scene, tolerance), F(tk_diff_scene, background),
    F(tk_diff_scene, loss_row0), F(tk_diff_scene, loss_row1),
};

#undef S
#undef F

}  // namespace

extern "C" uint32_t tk_abi_layout(const tk_abi_field** table) {
    if (table) *table = kLayout;
    return uint32_t(sizeof(kLayout) / sizeof(kLayout[0]));
}
