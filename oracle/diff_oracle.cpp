// FP64 restatement of the differentiable model (include/tileink_diff.h), the
// reference point of the finite-difference gradient checks.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// Coverage is the exact signed area of the path in every pixel, computed with
// the area/cover accumulation of a scanline rasterizer in double precision:
// each line is cut at integer rows and columns; a piece of signed height h in
// column X adds -h (X + 1 - xmid) to cell X and -h (xmid - X) to cell X + 1,
// and the prefix sum along the row gives A. The sign matches fill_alpha_at
// (shared/coverage.hlsli:34-51): pixels to the right of an edge running from
// p0 to p1 gain p0.y - p1.y per unit of row height. Then c = min(|A|, 1),
// premultiplied src-over of the paths in order, the separable Gaussian with
// taps exp(-k^2 / 2 sigma^2) normalised over |k| <= radius and zero outside
// the canvas, src-over onto the background, and the mean squared error.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "oracle.h"

namespace {

struct Piece {
    double xa, ya, xb, yb;  // within one row band
};

// Adds one row-band piece to the row's accumulation buffer (width + 2 cells,
// cell 0 collects everything left of the canvas).
void accumulate(std::vector<double>& acc, uint32_t width, double xa, double ya, double xb, double yb) {
    const double h = yb - ya;
    if (h == 0.0) return;
    auto add_column = [&](double xs, double ys, double xe, double ye) {
        const double hh = ye - ys;
        if (hh == 0.0) return;
        const double mid = 0.5 * (xs + xe);
        const double X = std::floor(std::min(xs, xe) + 0.5 * std::fabs(xe - xs));  // column of the sub-piece
        if (X < 0.0) {
            acc[0] += -hh;  // every pixel of the row lies to the right
            return;
        }
        if (X >= double(width)) return;
        const size_t xi = size_t(X);
        acc[xi] += -hh * (X + 1.0 - mid);
        acc[xi + 1] += -hh * (mid - X);
    };
    if (xa == xb) {
        add_column(xa, ya, xb, yb);
        return;
    }
    // cut at integer x between xa and xb
    const double dxdy = (xb - xa) / (yb - ya);
    double xs = xa, ys = ya;
    if (xb > xa) {
        for (double X = std::floor(xa) + 1.0; X < xb; X += 1.0) {
            const double y = ya + (X - xa) / dxdy;
            add_column(xs, ys, X, y);
            xs = X;
            ys = y;
        }
    } else {
        for (double X = std::ceil(xa) - 1.0; X > xb; X -= 1.0) {
            const double y = ya + (X - xa) / dxdy;
            add_column(xs, ys, X, y);
            xs = X;
            ys = y;
        }
    }
    add_column(xs, ys, xb, yb);
}

template <class F>
void parallel_rows(uint32_t rows, int threads, F&& f) {
    threads = std::max(1, std::min<int>(threads, int(rows)));
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            for (uint32_t y = uint32_t(t); y < rows; y += uint32_t(threads)) f(y);
        });
    for (auto& th : pool) th.join();
}

}  // namespace

extern "C" double or_diff_loss(uint32_t width, uint32_t height, uint32_t path_count, uint64_t line_count,
                               const tk_line* lines, const uint32_t* endpoint_point, const float* endpoint_weights,
                               const double* points, const double* colors, double sigma, int32_t radius,
                               const double* background, const float* target, double* image, int32_t threads) {
    const size_t n = size_t(width) * height;
    std::vector<double> layer(4 * n, 0.0);
    // line endpoints from the frozen weights
    std::vector<double> ep(4 * line_count);
    for (uint64_t l = 0; l < line_count; ++l)
        for (int e = 0; e < 2; ++e) {
            double x = 0.0, y = 0.0;
            const uint32_t b = endpoint_point[2 * l + e];
            for (int i = 0; i < 4; ++i) {
                const double w = double(endpoint_weights[8 * l + 4 * e + i]);
                if (w == 0.0) continue;
                x += w * points[2 * (b + i)];
                y += w * points[2 * (b + i) + 1];
            }
            ep[4 * l + 2 * e] = x;
            ep[4 * l + 2 * e + 1] = y;
        }
    uint64_t l0 = 0;
    for (uint32_t p = 0; p < path_count; ++p) {
        uint64_t l1 = l0;
        while (l1 < line_count && lines[l1].path_id == p) ++l1;
        // pieces per row band
        std::vector<std::vector<Piece>> rows(height);
        double xmax = 0.0;
        for (uint64_t l = l0; l < l1; ++l) {
            const double x0 = ep[4 * l], y0 = ep[4 * l + 1], x1 = ep[4 * l + 2], y1 = ep[4 * l + 3];
            xmax = std::max(xmax, std::max(x0, x1));
            if (y0 == y1) continue;
            const double ylo = std::min(y0, y1), yhi = std::max(y0, y1);
            const double ry0 = std::max(0.0, std::floor(ylo)), ry1 = std::min(double(height), std::ceil(yhi));
            for (double Y = ry0; Y < ry1; Y += 1.0) {
                const double ta = (std::max(ylo, Y) - y0) / (y1 - y0), tb = (std::min(yhi, Y + 1.0) - y0) / (y1 - y0);
                const double ua = std::min(ta, tb), ub = std::max(ta, tb);
                Piece pc{x0 + ua * (x1 - x0), y0 + ua * (y1 - y0), x0 + ub * (x1 - x0), y0 + ub * (y1 - y0)};
                if (pc.ya == pc.yb) continue;
                rows[size_t(Y)].push_back(pc);
            }
        }
        const double* col = colors + 4 * p;
        const double cp[4] = {col[0] * col[3], col[1] * col[3], col[2] * col[3], col[3]};
        const uint32_t xend = uint32_t(std::min<double>(width, std::max(0.0, std::ceil(xmax) + 1.0)));
        parallel_rows(height, threads, [&](uint32_t y) {
            if (rows[y].empty()) return;
            std::vector<double> acc(width + 2, 0.0);
            for (const Piece& pc : rows[y]) accumulate(acc, width, pc.xa, pc.ya - y, pc.xb, pc.yb - y);
            double A = 0.0;
            for (uint32_t x = 0; x < xend; ++x) {
                A += acc[x];
                const double c = std::min(std::fabs(A), 1.0);
                if (c == 0.0) continue;
                double* L = layer.data() + 4 * (size_t(y) * width + x);
                const double k = 1.0 - cp[3] * c;
                for (int ch = 0; ch < 4; ++ch) L[ch] = cp[ch] * c + L[ch] * k;
            }
        });
        l0 = l1;
    }
    // blur
    std::vector<double> B = layer;
    if (radius > 0) {
        std::vector<double> w(2 * radius + 1);
        double S = 0.0;
        for (int32_t k = -radius; k <= radius; ++k) S += (w[k + radius] = std::exp(-double(k) * k / (2.0 * sigma * sigma)));
        for (double& v : w) v /= S;
        std::vector<double> T1(4 * n, 0.0);
        parallel_rows(height, threads, [&](uint32_t y) {
            for (uint32_t x = 0; x < width; ++x)
                for (int32_t k = -radius; k <= radius; ++k) {
                    const int64_t sx = int64_t(x) + k;
                    if (sx < 0 || sx >= int64_t(width)) continue;
                    for (int ch = 0; ch < 4; ++ch)
                        T1[4 * (size_t(y) * width + x) + ch] += w[k + radius] * layer[4 * (size_t(y) * width + sx) + ch];
                }
        });
        std::fill(B.begin(), B.end(), 0.0);
        parallel_rows(height, threads, [&](uint32_t y) {
            for (int32_t k = -radius; k <= radius; ++k) {
                const int64_t sy = int64_t(y) + k;
                if (sy < 0 || sy >= int64_t(height)) continue;
                for (uint32_t x = 0; x < width; ++x)
                    for (int ch = 0; ch < 4; ++ch)
                        B[4 * (size_t(y) * width + x) + ch] += w[k + radius] * T1[4 * (size_t(sy) * width + x) + ch];
            }
        });
    }
    // composite and loss
    double loss = 0.0;
    for (size_t i = 0; i < n; ++i) {
        const double* b = B.data() + 4 * i;
        const double k = 1.0 - b[3];
        for (int ch = 0; ch < 4; ++ch) {
            const double I = b[ch] + background[ch] * k;
            if (image) image[4 * i + ch] = I;
            const double d = I - double(target[4 * i + ch]);
            loss += d * d;
        }
    }
    return loss / (4.0 * double(n));
}
