// Host helpers shared between the library's translation units (not part of
// the C ABI).
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/tileink.h"
#include "../../include/tileink_diff.h"

// The differentiable flattening of every path of `scene` (the lines
// tk_diff_flatten returns, with their endpoint control points and weights),
// paths flattened on host threads and concatenated in path order.
void tk_diff_flatten_all(const tk_diff_scene* scene, std::vector<tk_line>& lines, std::vector<uint32_t>& ep_point,
                         std::vector<float>& ep_w);
