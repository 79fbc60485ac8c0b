// distortion.cu — per-edge displacement integrals on the device.
//
// squared_integral (src/distortion.rs:137-168): for one edge, the exact
// integral over normalised arc length t of |original(t) - current(t)|^2 on the
// merged breakpoints of both polylines, f64 throughout. One thread per edge
// walks both curves; the equal-edge Kahan aggregation (distortion.rs:172-216)
// runs on the host over the per-edge results in point-offset order.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace bt {
namespace {

__device__ __forceinline__ double seg_length(const float2* p, size_t i) {
    return hypot(static_cast<double>(p[i + 1].x) - p[i].x, static_cast<double>(p[i + 1].y) - p[i].y);
}

struct DevCursor {
    const float2* pts;
    uint32_t n, next;
    double total, traversed;
    double sx, sy, ex, ey, st, et;
    __device__ void init(const float2* p, uint32_t count, double length) {
        pts = p;
        n = count;
        next = 0;
        total = length;
        traversed = 0.0;
        sx = ex = p[0].x;
        sy = ey = p[0].y;
        st = et = 0.0;
    }
    __device__ uint32_t left() const { return (n >= 2 ? n - 1 : 0) - next; }
    __device__ void advance(double t) {
        while (et <= t && et < 1.0) {
            if (left() == 0) {
                sx = ex; sy = ey; st = et; et = 1.0;
                return;
            }
            const uint32_t i = next++;
            const double length = seg_length(pts, i);
            if (length == 0.0) continue;
            sx = pts[i].x; sy = pts[i].y;
            ex = pts[i + 1].x; ey = pts[i + 1].y;
            st = et;
            traversed += length;
            et = left() == 0 ? 1.0 : traversed / total;
        }
    }
    __device__ void position(double t, double* x, double* y) const {
        if (t >= et) { *x = ex; *y = ey; return; }
        if (t <= st) { *x = sx; *y = sy; return; }
        const double f = (t - st) / (et - st);
        *x = fma(f, ex - sx, sx);
        *y = fma(f, ey - sy, sy);
    }
};

__device__ bool curve_length(const float2* p, uint32_t n, double* out) {
    double l = 0.0;
    for (uint32_t i = 0; i < n; ++i)
        if (!isfinite(p[i].x) || !isfinite(p[i].y)) return false;
    for (uint32_t i = 0; i + 1 < n; ++i) l += seg_length(p, i);
    if (!isfinite(l)) return false;
    *out = l;
    return true;
}

__global__ void edge_integral_kernel(const PathRec* paths, uint32_t n_paths, const float2* original,
                                     const float2* current, double* out, uint32_t* status) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_paths) return;
    const PathRec r = paths[e];
    if (r.count == 0) {
        out[e] = 0.0;
        return;
    }
    const float2* a = original + r.point_offset;
    const float2* b = current + r.point_offset;
    double la, lb;
    if (!curve_length(a, r.count, &la) || !curve_length(b, r.count, &lb)) {
        atomicOr(status, 4u);
        out[e] = 0.0;
        return;
    }
    DevCursor ca, cb;
    ca.init(a, r.count, la);
    cb.init(b, r.count, lb);
    double value = 0.0, correction = 0.0, t = 0.0;
    while (!(t >= 1.0)) {
        ca.advance(t);
        cb.advance(t);
        const double next = fmin(ca.et, cb.et);
        if (!(next > t && next <= 1.0)) {
            atomicOr(status, 4u);
            out[e] = 0.0;
            return;
        }
        double px, py, qx, qy, rx, ry, sx, sy;
        ca.position(t, &px, &py);
        cb.position(t, &qx, &qy);
        ca.position(next, &rx, &ry);
        cb.position(next, &sx, &sy);
        const double ax = px - qx, ay = py - qy;
        const double bx = rx - sx, by = ry - sy;
        const double mx = ax + bx, my = ay + by;
        const double dx = bx - ax, dy = by - ay;
        const double mid = fma(mx, mx, my * my);
        const double chg = fma(dx, dx, dy * dy);
        const double term = (next - t) * (mid / 4.0 + chg / 12.0);
        const double adjusted = term - correction;
        const double nv = value + adjusted;
        correction = (nv - value) - adjusted;
        value = nv;
        t = next;
    }
    if (!(isfinite(value) && value >= 0.0)) atomicOr(status, 4u);
    out[e] = value;
}

}  // namespace

void launch_edge_integrals(const PathRec* paths, uint32_t n_paths, const float2* original, const float2* current,
                           double* out, uint32_t* status, cudaStream_t s) {
    if (n_paths == 0) return;
    edge_integral_kernel<<<div_up(n_paths, 128), 128, 0, s>>>(paths, n_paths, original, current, out, status);
}

}  // namespace bt
