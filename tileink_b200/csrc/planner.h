// Host scan-line planner: tiles a line visits inside a path's tile bbox
// (src/shared/scan_line.rs:17-151). The Canvas sums it per path into the
// path's segment capacity (src/canvas/storage.rs:131-142).
#pragma once
#include <stdint.h>

#include "../../include/tileink.h"

#ifdef __cplusplus
extern "C" {
#endif

uint32_t tk_plan_line_tile_count(const tk_line* line, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1);

#ifdef __cplusplus
}
#endif
