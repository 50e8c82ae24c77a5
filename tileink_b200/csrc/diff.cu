// Differentiable rendering: a float forward of fine raster, Gaussian blur and
// the group composite, and their hand-written adjoint.
//
// Model (the reference's fine + blur + composite path, fine/interpreter.hlsli,
// shared/coverage.hlsli:7-51, filter/blur.hlsli, without the RGBA8
// quantization between stages so that it is differentiable):
//   coverage  A = signed exact area of the path in the pixel (fill_alpha_at),
//             c = min(|A|, 1) (nonzero)
//   layer     L_i = s_i + L_{i-1} (1 - a_i),  s_i = colp_i c_i,  a_i = alpha_i c_i
//   blur      T1 = Gx L, B = Gy T1, taps w_k = e_k / sum e, e_k = exp(-k^2 / 2 sigma^2),
//             |k| <= r, zero outside the canvas
//   composite I = B + bg (1 - B.a)
//   loss      mean over pixels and channels of (I - target)^2
// Backward: dB from dI; the blur adjoint is the same symmetric blur; the sigma
// gradient uses the tap derivatives w'_k. Fine recomputes coverage per tile
// (forward replay storing A_i and P_i = g . L_{i-1} per pixel), then walks the
// records in reverse with the transmittance T_i = prod_{j>i} (1 - a_j):
//   dL/dc_i = T_i (g . colp_i - alpha_i P_i)
// and turns dL/dA per pixel into line-endpoint gradients by the boundary
// integral of the exact area: for a line P0 -> P1 (d = P1 - P0) and a pixel P,
//   dA_P/dP0 = (int_{u in U_P} (1 - u) du) (d.y, -d.x),
//   dA_P/dP1 = (int_{u in U_P} u du) (d.y, -d.x),
// U_P = the parameters u of the line's points inside P.
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.h"

namespace tk {
namespace {

using namespace tkd;

constexpr int kDiffThreads = 256;
constexpr uint32_t kDiffSegStage = 256;

struct DiffSmem {
    float4 sgp[kDiffSegStage];
    float sgy[kDiffSegStage];
    float gA[TK_TILE_SIZE * TK_TILE_SIZE];
    float red[kDiffThreads / 32][5];
};

// Signed area A of one fill record at tile pixel (lx, ly): fill_alpha_at over
// the record's segments, staged through shared memory in slices.
__device__ float record_area(DiffSmem& S, const SegmentRec* __restrict__ segments, uint32_t s0, uint32_t s1,
                             int32_t backdrop, uint32_t lx, uint32_t ly) {
    float base = float(backdrop), running = 0.0f, partial = 0.0f;
    for (uint32_t c0 = s0; c0 < s1; c0 += kDiffSegStage) {
        const uint32_t m = min(kDiffSegStage, s1 - c0);
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < m; j += kDiffThreads) {
            S.sgp[j] = __ldg(reinterpret_cast<const float4*>(segments + c0 + j));
            S.sgy[j] = __ldg(&segments[c0 + j].y_edge);
        }
        __syncthreads();
        for (uint32_t j = 0; j < m; ++j) {
            const float4 g = S.sgp[j];
            const RowParts q = segment_row_parts(g.x, g.y, g.z, g.w, S.sgy[j], ly);
            base += q.edge;
            if (q.dy != 0.0f) {
                const int32_t hi = min(max(f2i(ceilf(q.xmax)), 0), int32_t(TK_TILE_SIZE));
                if (hi < int32_t(TK_TILE_SIZE) && int32_t(lx) >= hi) running += q.dy;
                const int32_t lo = min(max(f2i(floorf(q.xmin)), 0), int32_t(TK_TILE_SIZE));
                if (int32_t(lx) >= lo && int32_t(lx) < hi) partial += segment_area_at(q.xmin, q.xmax, lx) * q.dy;
            }
        }
    }
    return base + running + partial;
}

__device__ __forceinline__ float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

// Forward: the float layer image of one target pass.
__global__ void __launch_bounds__(kDiffThreads)
    k_diff_fine_fwd(const tk_tile_record* __restrict__ tiles, const tk_ptcl_record* __restrict__ ptcl,
                    const SegmentRec* __restrict__ segments, const float4* __restrict__ colp, float4* layer,
                    uint32_t width, uint32_t height, uint32_t tw, uint32_t* error) {
    __shared__ DiffSmem S;
    const uint32_t tile = blockIdx.x;
    const tk_tile_record rec = tiles[tile];
    const uint32_t lx = threadIdx.x & 15u, ly = threadIdx.x >> 4;
    const uint32_t gx = (tile % tw) * TK_TILE_SIZE + lx, gy = (tile / tw) * TK_TILE_SIZE + ly;
    float4 L = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint64_t r = rec.ptcl_start; r < rec.ptcl_end; ++r) {
        const tk_ptcl_record q = ptcl[r];
        if (q.tag == TK_PTCL_END) break;
        if (q.tag == TK_PTCL_BATCH_BEGIN) {
            if ((q.color >> TK_TILE_PREFIX_SHIFT) && threadIdx.x == 0) atomicOr(error, ERR_UNSUPPORTED);
            continue;
        }
        if (q.tag != TK_PTCL_FILL) {
            if (threadIdx.x == 0) atomicOr(error, ERR_UNSUPPORTED);
            continue;
        }
        const float A = record_area(S, segments, q.segment_start, q.segment_end, q.backdrop, lx, ly);
        const float c = fminf(fabsf(A), 1.0f);
        const float4 p = colp[q.color];
        const float k = 1.0f - p.w * c;
        L = make_float4(p.x * c + L.x * k, p.y * c + L.y * k, p.z * c + L.z * k, p.w * c + L.w * k);
    }
    if (gx < width && gy < height) layer[uint64_t(gy) * width + gx] = L;
}

// out[p] = sum_k w[k + r] in[p + k * step]; zero outside the canvas.
__device__ __forceinline__ float4 blur_tap(const float4* __restrict__ img, const float* __restrict__ w, int32_t r,
                                           uint32_t width, uint32_t height, int32_t x, int32_t y, int32_t axis) {
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int32_t k = -r; k <= r; ++k) {
        const int32_t sx = axis == 0 ? x + k : x, sy = axis == 0 ? y : y + k;
        if (sx < 0 || sy < 0 || sx >= int32_t(width) || sy >= int32_t(height)) continue;
        const float4 v = img[uint64_t(sy) * width + sx];
        const float wk = w[k + r];
        acc.x += wk * v.x;
        acc.y += wk * v.y;
        acc.z += wk * v.z;
        acc.w += wk * v.w;
    }
    return acc;
}

__global__ void k_diff_blur(const float4* __restrict__ in, float4* out, const float* __restrict__ w, int32_t r,
                            uint32_t width, uint32_t height, int32_t axis) {
    const int32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= int32_t(width)) return;
    out[uint64_t(y) * width + x] = blur_tap(in, w, r, width, height, x, y, axis);
}

// I = B + bg (1 - B.a); gI = 2 (I - target) / (4 W H); loss partial sums.
// Only pixels [lo, hi) enter the loss (a row range of a split objective);
// the mean still divides by every pixel, so the row ranges' losses and
// gradients sum to the whole frame's.
__global__ void k_diff_composite(const float4* __restrict__ B, const float4* __restrict__ target, float4 bg,
                                 uint64_t n, uint64_t lo, uint64_t hi, float4* image, float4* gI, double* loss) {
    double acc = 0.0;
    const double inv = 1.0 / (4.0 * double(n));
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const float4 b = B[i];
        const float k = 1.0f - b.w;
        const float4 I = make_float4(b.x + bg.x * k, b.y + bg.y * k, b.z + bg.z * k, b.w + bg.w * k);
        const float4 t = target[i];
        const float4 d = make_float4(I.x - t.x, I.y - t.y, I.z - t.z, I.w - t.w);
        if (image) image[i] = I;
        if (i < lo || i >= hi) {
            gI[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            continue;
        }
        const float s = float(2.0 * inv);
        gI[i] = make_float4(s * d.x, s * d.y, s * d.z, s * d.w);
        acc += double(d.x) * d.x + double(d.y) * d.y + double(d.z) * d.z + double(d.w) * d.w;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31u) == 0) atomicAdd(loss, acc * inv);
}

__device__ __forceinline__ float4 composite_adjoint(float4 g, float4 bg) {
    // dI/dB: identity per channel, and -bg on the alpha channel's column.
    return make_float4(g.x, g.y, g.z, g.w - dot4(g, bg));
}

// Blur adjoint along `axis` plus the sigma term <dout, G' in_fwd>:
//   din[p] = sum_k w_k dout[p + k]   (symmetric taps, zero outside)
//   sig   += dout[p] . sum_k w'_k fwd_in[p + k]
// With `from_gI`, dout is the composite adjoint of gI.
__global__ void k_diff_blur_bwd(const float4* __restrict__ dout_src, const float4* __restrict__ fwd_in, float4* din,
                                const float* __restrict__ w, const float* __restrict__ wd, int32_t r, uint32_t width,
                                uint32_t height, int32_t axis, int32_t from_gI, float4 bg, double* sig) {
    const int32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    double part = 0.0;
    if (x < int32_t(width)) {
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f), dacc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int32_t k = -r; k <= r; ++k) {
            const int32_t sx = axis == 0 ? x + k : x, sy = axis == 0 ? y : y + k;
            if (sx < 0 || sy < 0 || sx >= int32_t(width) || sy >= int32_t(height)) continue;
            const uint64_t q = uint64_t(sy) * width + sx;
            float4 g = dout_src[q];
            if (from_gI) g = composite_adjoint(g, bg);
            const float wk = w[k + r], dk = wd[k + r];
            acc.x += wk * g.x;
            acc.y += wk * g.y;
            acc.z += wk * g.z;
            acc.w += wk * g.w;
            const float4 v = fwd_in[q];
            dacc.x += dk * v.x;
            dacc.y += dk * v.y;
            dacc.z += dk * v.z;
            dacc.w += dk * v.w;
        }
        const uint64_t p = uint64_t(y) * width + x;
        din[p] = acc;
        float4 g = dout_src[p];
        if (from_gI) g = composite_adjoint(g, bg);
        part = double(dot4(g, dacc));
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31u) == 0 && part != 0.0) atomicAdd(sig, part);
}

// Without blur the layer adjoint is the composite adjoint of gI.
__global__ void k_diff_composite_bwd(const float4* __restrict__ gI, float4 bg, uint64_t n, float4* dL) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        dL[i] = composite_adjoint(gI[i], bg);
}

// Boundary-integral weights of a tile segment q0 -> q1 (tile-local), part of
// line P0 -> P1 (tile-local), against the per-pixel adjoint gA: returns
// (sum gA int (1-u) du, sum gA int u du) over the cells the segment crosses.
__device__ float2 segment_boundary_sums(const float* __restrict__ gA, float4 q, float2 P0, float2 d) {
    const float dd = d.x * d.x + d.y * d.y;
    if (!(dd > 0.0f)) return make_float2(0.f, 0.f);
    const float u0 = ((q.x - P0.x) * d.x + (q.y - P0.y) * d.y) / dd;
    const float u1 = ((q.z - P0.x) * d.x + (q.w - P0.y) * d.y) / dd;
    const float ex = q.z - q.x, ey = q.w - q.y;
    float vx = 2.0f, vy = 2.0f, stx = 2.0f, sty = 2.0f;
    if (ex > 0.0f) { vx = (floorf(q.x) + 1.0f - q.x) / ex; stx = 1.0f / ex; }
    else if (ex < 0.0f) { vx = (ceilf(q.x) - 1.0f - q.x) / ex; stx = -1.0f / ex; }
    if (ey > 0.0f) { vy = (floorf(q.y) + 1.0f - q.y) / ey; sty = 1.0f / ey; }
    else if (ey < 0.0f) { vy = (ceilf(q.y) - 1.0f - q.y) / ey; sty = -1.0f / ey; }
    float v = 0.0f, s0 = 0.0f, s1 = 0.0f;
    for (int it = 0; it < 2 * int(TK_TILE_SIZE) + 4 && v < 1.0f; ++it) {
        const float vn = fminf(fminf(vx, vy), 1.0f);
        if (vn > v) {
            const float vm = 0.5f * (v + vn);
            const int32_t cx = min(max(int32_t(floorf(q.x + vm * ex)), 0), int32_t(TK_TILE_SIZE) - 1);
            const int32_t cy = min(max(int32_t(floorf(q.y + vm * ey)), 0), int32_t(TK_TILE_SIZE) - 1);
            const float ua = u0 + v * (u1 - u0), ub = u0 + vn * (u1 - u0);
            const float ul = fminf(ua, ub), uh = fmaxf(ua, ub);
            const float sq = 0.5f * (uh * uh - ul * ul);
            const float g = gA[cy * TK_TILE_SIZE + cx];
            s0 += g * ((uh - ul) - sq);
            s1 += g * sq;
        }
        if (vx <= vn) vx += stx;
        if (vy <= vn) vy += sty;
        v = vn;
    }
    return make_float2(s0, s1);
}

// Backward of fine: per tile, forward replay (A_i, P_i per pixel into
// `scratch`), then the records in reverse.
__global__ void __launch_bounds__(kDiffThreads)
    k_diff_fine_bwd(const tk_tile_record* __restrict__ tiles, const tk_ptcl_record* __restrict__ ptcl,
                    const SegmentRec* __restrict__ segments, const uint32_t* __restrict__ seg_line,
                    const tk_line* __restrict__ lines, const float4* __restrict__ colp,
                    const float4* __restrict__ dlayer, float2* scratch, float2* line_acc, float* color_acc,
                    uint32_t width, uint32_t height, uint32_t tw, uint32_t* error) {
    __shared__ DiffSmem S;
    const uint32_t tile = blockIdx.x;
    const tk_tile_record rec = tiles[tile];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t lx = tid & 15u, ly = tid >> 4;
    const uint32_t ox = (tile % tw) * TK_TILE_SIZE, oy = (tile / tw) * TK_TILE_SIZE;
    const uint32_t gx = ox + lx, gy = oy + ly;
    const bool inside = gx < width && gy < height;
    const float4 g = inside ? dlayer[uint64_t(gy) * width + gx] : make_float4(0.f, 0.f, 0.f, 0.f);
    // pass A: forward replay
    float4 L = make_float4(0.f, 0.f, 0.f, 0.f);
    uint64_t last = rec.ptcl_start;
    for (uint64_t r = rec.ptcl_start; r < rec.ptcl_end; ++r) {
        const tk_ptcl_record q = ptcl[r];
        last = r;
        if (q.tag == TK_PTCL_END) break;
        if (q.tag == TK_PTCL_BATCH_BEGIN) {
            // occlusion skips come only from opaque solid-rect records, which
            // differentiable scenes do not contain
            if ((q.color >> TK_TILE_PREFIX_SHIFT) && tid == 0) atomicOr(error, ERR_UNSUPPORTED);
            continue;
        }
        if (q.tag != TK_PTCL_FILL) continue;
        const float A = record_area(S, segments, q.segment_start, q.segment_end, q.backdrop, lx, ly);
        const float c = fminf(fabsf(A), 1.0f);
        const float4 p = colp[q.color];
        scratch[r * kDiffThreads + tid] = make_float2(A, dot4(g, L));
        const float k = 1.0f - p.w * c;
        L = make_float4(p.x * c + L.x * k, p.y * c + L.y * k, p.z * c + L.z * k, p.w * c + L.w * k);
    }
    // pass B: the FILL records in reverse
    float T = 1.0f;
    for (uint64_t r = last + 1; r-- > rec.ptcl_start;) {
        const tk_ptcl_record q = ptcl[r];
        if (q.tag != TK_PTCL_FILL) continue;
        const float2 ap = scratch[r * kDiffThreads + tid];
        const float A = ap.x, P = ap.y;
        const float c = inside ? fminf(fabsf(A), 1.0f) : 0.0f;
        const float4 p = colp[q.color];
        const float dc = T * (dot4(g, p) - p.w * P);
        // colour partials: T g c (4 channels) and -T P c (alpha through 1 - a)
        float v[5] = {T * g.x * c, T * g.y * c, T * g.z * c, T * g.w * c, -T * P * c};
#pragma unroll
        for (int k = 0; k < 5; ++k)
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < 5; ++k) S.red[warp][k] = v[k];
        S.gA[tid] = (inside && c < 1.0f && A != 0.0f) ? (A > 0.0f ? dc : -dc) : 0.0f;
        __syncthreads();
        if (tid < 5) {
            float s = 0.0f;
            for (int w = 0; w < kDiffThreads / 32; ++w) s += S.red[w][tid];
            if (s != 0.0f) atomicAdd(color_acc + uint64_t(q.color) * 5u + tid, s);
        }
        for (uint32_t j = q.segment_start + tid; j < q.segment_end; j += kDiffThreads) {
            const float4 seg = __ldg(reinterpret_cast<const float4*>(segments + j));
            const uint32_t li = seg_line[j];
            const tk_line ln = lines[li];
            const float2 P0 = make_float2(ln.p0[0] - float(ox), ln.p0[1] - float(oy));
            const float2 d = make_float2(ln.p1[0] - ln.p0[0], ln.p1[1] - ln.p0[1]);
            const float2 s = segment_boundary_sums(S.gA, seg, P0, d);
            if (s.x != 0.0f) atomicAdd(&line_acc[li].x, s.x);
            if (s.y != 0.0f) atomicAdd(&line_acc[li].y, s.y);
        }
        __syncthreads();
        T *= 1.0f - p.w * c;
    }
}

// Line-endpoint gradients to control points: each endpoint is
// sum_i w_i C[base + i] (frozen flattening weights).
__global__ void k_diff_lines_to_points(const tk_line* __restrict__ lines, const float2* __restrict__ line_acc,
                                       const uint32_t* __restrict__ ep_base, const float* __restrict__ ep_w,
                                       uint64_t n, float* dpoints) {
    for (uint64_t l = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; l < n; l += uint64_t(gridDim.x) * blockDim.x) {
        const tk_line ln = lines[l];
        const float dx = ln.p1[0] - ln.p0[0], dy = ln.p1[1] - ln.p0[1];
        const float2 s = line_acc[l];
        const float g[2][2] = {{s.x * dy, -s.x * dx}, {s.y * dy, -s.y * dx}};
        for (int e = 0; e < 2; ++e) {
            const uint32_t b = ep_base[2 * l + e];
            for (int i = 0; i < 4; ++i) {
                const float wi = ep_w[8 * l + 4 * e + i];
                if (wi == 0.0f) continue;
                atomicAdd(dpoints + 2u * (b + i), wi * g[e][0]);
                atomicAdd(dpoints + 2u * (b + i) + 1u, wi * g[e][1]);
            }
        }
    }
}

}  // namespace

void launch_diff_fine_fwd(const SceneView& s, const PassView& p, const float4* colp, float4* layer, cudaStream_t st) {
    const uint32_t T = s.tw * s.th;
    if (T == 0) return;
    k_diff_fine_fwd<<<T, kDiffThreads, 0, st>>>(p.tiles, p.ptcl, s.segments, colp, layer, s.width, s.height, s.tw,
                                               s.error);
}

void launch_diff_blur(const float4* in, float4* out, const float* w, int32_t r, uint32_t width, uint32_t height,
                      int32_t axis, cudaStream_t st) {
    dim3 grid((width + 255) / 256, height);
    k_diff_blur<<<grid, 256, 0, st>>>(in, out, w, r, width, height, axis);
}

void launch_diff_composite(const float4* B, const float4* target, float4 bg, uint64_t n, uint64_t lo, uint64_t hi,
                           float4* image, float4* gI, double* loss, cudaStream_t st) {
    k_diff_composite<<<148 * 8, 256, 0, st>>>(B, target, bg, n, lo, hi, image, gI, loss);
}

void launch_diff_blur_bwd(const float4* dout_src, const float4* fwd_in, float4* din, const float* w, const float* wd,
                          int32_t r, uint32_t width, uint32_t height, int32_t axis, bool from_gI, float4 bg,
                          double* sig, cudaStream_t st) {
    dim3 grid((width + 255) / 256, height);
    k_diff_blur_bwd<<<grid, 256, 0, st>>>(dout_src, fwd_in, din, w, wd, r, width, height, axis, from_gI ? 1 : 0, bg,
                                          sig);
}

void launch_diff_composite_bwd(const float4* gI, float4 bg, uint64_t n, float4* dL, cudaStream_t st) {
    k_diff_composite_bwd<<<148 * 8, 256, 0, st>>>(gI, bg, n, dL);
}

void launch_diff_fine_bwd(const SceneView& s, const PassView& p, const uint32_t* seg_line, const float4* colp,
                          const float4* dlayer, float2* scratch, float2* line_acc, float* color_acc, cudaStream_t st) {
    const uint32_t T = s.tw * s.th;
    if (T == 0) return;
    k_diff_fine_bwd<<<T, kDiffThreads, 0, st>>>(p.tiles, p.ptcl, s.segments, seg_line, s.lines, colp, dlayer, scratch,
                                               line_acc, color_acc, s.width, s.height, s.tw, s.error);
}

void launch_diff_lines_to_points(const tk_line* lines, const float2* line_acc, const uint32_t* ep_base,
                                 const float* ep_w, uint64_t n, float* dpoints, cudaStream_t st) {
    if (n == 0) return;
    k_diff_lines_to_points<<<148 * 4, 256, 0, st>>>(lines, line_acc, ep_base, ep_w, n, dpoints);
}

}  // namespace tk
