// advect.cu — density-gradient advection, an iteration mode beyond the
// reference (kernel-density-estimation edge bundling): every sample that is
// not the first or last of its path climbs the gradient of the blurred,
// normalised density by a fixed step, then relaxes towards its advected path
// neighbours; the new positions are splatted for the next density pass. The
// oracle (or_advect) states the same operation order:
//  - map position (u, v) = ((x * 0.5 + 0.5) * (W - 1), (0.5 - y * 0.5) * (H - 1))
//    (the splat's texel space);
//  - bilinear density with clamp-to-edge; central differences one texel
//    apart, halved;
//  - `step` texels along the unit gradient (none when its length is not above
//    1e-12), back to clip units by 2 / (W - 1) and -2 / (H - 1);
//  - a + smooth * ((a_prev + a_next) * 0.5 - a).
// One thread per sample, sample order (paths are contiguous; edge ids change
// at path boundaries). Every quantity rounds once per operation.
#include "kernels.cuh"

namespace bt {
namespace {

__device__ __forceinline__ float density_at(const float* __restrict__ d, uint32_t w, uint32_t h, float u, float v) {
    const float uc = fminf(fmaxf(u, 0.0f), static_cast<float>(w - 1u));
    const float vc = fminf(fmaxf(v, 0.0f), static_cast<float>(h - 1u));
    const float fx0 = floorf(uc), fy0 = floorf(vc);
    const float fx = __fsub_rn(uc, fx0), fy = __fsub_rn(vc, fy0);
    const uint32_t x0 = static_cast<uint32_t>(fx0), y0 = static_cast<uint32_t>(fy0);
    const uint32_t x1 = min(x0 + 1u, w - 1u), y1 = min(y0 + 1u, h - 1u);
    const float* r0 = d + static_cast<size_t>(y0) * w;
    const float* r1 = d + static_cast<size_t>(y1) * w;
    const float top = __fadd_rn(__fmul_rn(__ldg(r0 + x0), __fsub_rn(1.0f, fx)), __fmul_rn(__ldg(r0 + x1), fx));
    const float bottom = __fadd_rn(__fmul_rn(__ldg(r1 + x0), __fsub_rn(1.0f, fx)), __fmul_rn(__ldg(r1 + x1), fx));
    return __fadd_rn(__fmul_rn(top, __fsub_rn(1.0f, fy)), __fmul_rn(bottom, fy));
}

// Bilinear set-up of density_at: the cell's corner and weights.
struct Bilinear {
    uint32_t x0, y0, x1, y1;
    float fx, fy;
};

__device__ __forceinline__ Bilinear bilinear_at(uint32_t w, uint32_t h, float u, float v) {
    const float uc = fminf(fmaxf(u, 0.0f), static_cast<float>(w - 1u));
    const float vc = fminf(fmaxf(v, 0.0f), static_cast<float>(h - 1u));
    const float fx0 = floorf(uc), fy0 = floorf(vc);
    Bilinear b;
    b.fx = __fsub_rn(uc, fx0);
    b.fy = __fsub_rn(vc, fy0);
    b.x0 = static_cast<uint32_t>(fx0);
    b.y0 = static_cast<uint32_t>(fy0);
    b.x1 = min(b.x0 + 1u, w - 1u);
    b.y1 = min(b.y0 + 1u, h - 1u);
    return b;
}

// density_at's combination of four texels.
__device__ __forceinline__ float blend(const Bilinear& b, float t00, float t10, float t01, float t11) {
    const float top = __fadd_rn(__fmul_rn(t00, __fsub_rn(1.0f, b.fx)), __fmul_rn(t10, b.fx));
    const float bottom = __fadd_rn(__fmul_rn(t01, __fsub_rn(1.0f, b.fx)), __fmul_rn(t11, b.fx));
    return __fadd_rn(__fmul_rn(top, __fsub_rn(1.0f, b.fy)), __fmul_rn(bottom, b.fy));
}

__device__ __forceinline__ float2 advected(const AdvectArgs& a, float2 p) {
    const float u = __fmul_rn(__fadd_rn(__fmul_rn(p.x, 0.5f), 0.5f), static_cast<float>(a.map.w - 1u));
    const float v = __fmul_rn(__fsub_rn(0.5f, __fmul_rn(p.y, 0.5f)), static_cast<float>(a.map.h - 1u));
    const uint32_t w = a.map.w, h = a.map.h;
    const Bilinear br = bilinear_at(w, h, __fadd_rn(u, 1.0f), v), bl = bilinear_at(w, h, __fsub_rn(u, 1.0f), v);
    const Bilinear bd = bilinear_at(w, h, u, __fadd_rn(v, 1.0f)), bu = bilinear_at(w, h, u, __fsub_rn(v, 1.0f));
    // The four samples' cells usually form a cross of 12 texels around
    // (X, Y) = the right sample's corner minus (1, 0): read each once.
    // Near the map's edges, or where u +- 1 rounds across a cell, the
    // corners differ and each sample reads its own four texels.
    const uint32_t X = bl.x1, Y = br.y0;
    const bool cross = br.x0 == X + 1u && br.x1 == X + 2u && br.y1 == Y + 1u && bl.x0 == X - 1u && bl.y0 == Y &&
                       bl.y1 == Y + 1u && bd.x0 == X && bd.x1 == X + 1u && bd.y0 == Y + 1u && bd.y1 == Y + 2u &&
                       bu.x0 == X && bu.x1 == X + 1u && bu.y0 == Y - 1u && bu.y1 == Y;
    const float* __restrict__ d = a.density;
    float gu, gv;
    if (cross) {
        const float* r0 = d + static_cast<size_t>(Y - 1u) * w;
        const float* r1 = r0 + w;
        const float* r2 = r1 + w;
        const float* r3 = r2 + w;
        const float a0 = __ldg(r0 + X), a1 = __ldg(r0 + X + 1u);
        const float b_ = __ldg(r1 + X - 1u), b0 = __ldg(r1 + X), b1 = __ldg(r1 + X + 1u), b2 = __ldg(r1 + X + 2u);
        const float c_ = __ldg(r2 + X - 1u), c0 = __ldg(r2 + X), c1 = __ldg(r2 + X + 1u), c2 = __ldg(r2 + X + 2u);
        const float e0 = __ldg(r3 + X), e1 = __ldg(r3 + X + 1u);
        gu = __fmul_rn(__fsub_rn(blend(br, b1, b2, c1, c2), blend(bl, b_, b0, c_, c0)), 0.5f);
        gv = __fmul_rn(__fsub_rn(blend(bd, c0, c1, e0, e1), blend(bu, a0, a1, b0, b1)), 0.5f);
    } else {
        gu = __fmul_rn(__fsub_rn(density_at(d, w, h, __fadd_rn(u, 1.0f), v), density_at(d, w, h, __fsub_rn(u, 1.0f), v)),
                       0.5f);
        gv = __fmul_rn(__fsub_rn(density_at(d, w, h, u, __fadd_rn(v, 1.0f)), density_at(d, w, h, u, __fsub_rn(v, 1.0f))),
                       0.5f);
    }
    const float len = __fsqrt_rn(__fadd_rn(__fmul_rn(gu, gu), __fmul_rn(gv, gv)));
    float du = 0.0f, dv = 0.0f;
    if (len > 1e-12f) {
        du = __fmul_rn(a.step, __fdiv_rn(gu, len));
        dv = __fmul_rn(a.step, __fdiv_rn(gv, len));
    }
    return make_float2(__fadd_rn(p.x, __fmul_rn(du, a.sx_inv)), __fsub_rn(p.y, __fmul_rn(dv, a.sy_inv)));
}

__device__ __forceinline__ bool movable(const uint32_t* __restrict__ ids, uint32_t n, uint32_t i) {
    return i > 0 && i + 1 < n && ids[i - 1] == ids[i] && ids[i + 1] == ids[i];
}

constexpr int kAdvectBlock = 256;

// Advected position of sample j when it moves, else its position.
__device__ __forceinline__ float2 moved_or_fixed(const AdvectArgs& a, uint32_t j) {
    const float2 q = a.xy[j];
    return movable(a.edge_ids, a.n, j) ? advected(a, q) : q;
}

// Each sample's advected position is evaluated once per CTA into shared
// memory, with one halo sample on either side, and read there by its path
// neighbours (a third of the gradient gathers and divisions of evaluating
// both neighbours per thread). Every lane of the grid's warps reaches the
// splat (idle lanes past n too): it is warp-aggregated.
// Eight CTAs of 256 per SM (32 registers, 20 bytes spilled): the density
// gathers are latency-bound, and 64 resident warps hide them better than 32
// at 61 registers (four CTAs: 0.252 ms per iteration of the large workload
// with the density passes; six at 40 registers: 0.219; eight: 0.210).
__global__ void __launch_bounds__(kAdvectBlock, 8) advect_kernel(AdvectArgs a) {
    __shared__ float2 adv[kAdvectBlock + 2];
    const uint32_t base = blockIdx.x * kAdvectBlock;
    const uint32_t i = base + threadIdx.x;
    if (i < a.n) adv[threadIdx.x + 1] = moved_or_fixed(a, i);
    // Halo: sample base - 1 (read only when sample base moves, so base > 0)
    // and sample base + kAdvectBlock (read only when the block's last sample
    // moves, so it exists).
    if (threadIdx.x == 0 && base > 0) adv[0] = moved_or_fixed(a, base - 1);
    if (threadIdx.x == 1 && base + kAdvectBlock < a.n) adv[kAdvectBlock + 1] = moved_or_fixed(a, base + kAdvectBlock);
    __syncthreads();
    uint32_t d = 0xFFFFFFFFu;                              // no texel
    if (i < a.n) {
        float2 out = a.xy[i];
        if (movable(a.edge_ids, a.n, i)) {
            const float2 s = adv[threadIdx.x + 1];
            const float2 p = adv[threadIdx.x];
            const float2 q = adv[threadIdx.x + 2];
            out.x = __fadd_rn(s.x, __fmul_rn(a.smooth, __fsub_rn(__fmul_rn(__fadd_rn(p.x, q.x), 0.5f), s.x)));
            out.y = __fadd_rn(s.y, __fmul_rn(a.smooth, __fsub_rn(__fmul_rn(__fadd_rn(p.y, q.y), 0.5f), s.y)));
        }
        a.out[i] = out;
        if (a.counts) splat_index(out.x, out.y, a.map, &d);
    }
    if (a.counts) {
        // One add per texel per warp: samples climbing to the same density
        // ridge share texels (integer counts: any order gives the same).
        const unsigned same = __match_any_sync(0xFFFFFFFFu, d);
        if (d != 0xFFFFFFFFu && (threadIdx.x & 31) == __ffs(same) - 1)
            atomicAdd(&a.counts[d], static_cast<uint32_t>(__popc(same)));
    }
}

}  // namespace

void launch_advect(const AdvectArgs& a, cudaStream_t s) {
    if (a.n) advect_kernel<<<div_up(a.n, static_cast<uint32_t>(kAdvectBlock)), kAdvectBlock, 0, s>>>(a);
}

}  // namespace bt
