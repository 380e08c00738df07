// Mixed-precision near field (P2P; the role of the near field of near.py:48-312 on
// the mixed path): FP32 pair arithmetic, FP64 only where accuracy needs it.
//   * Separations come from FP32 hi/lo position pairs, (hi - hi') + (lo - lo'), so
//     they carry a relative error of eps32 however close the points are (box-local
//     FP32 coordinates gave 3.7e-6 on clustered clouds).
//   * The phase k r is an FP32 product: r itself carries eps32, and forming k r in
//     FP64 with an FP64 reduction before sincosf measured the same error.
//   * Sums run in FP32 over one source leaf and are combined in FP64, as is the
//     final per-target sum.
// P2M, P2L, L2P and M2P stay FP64 on the mixed path: their outputs feed or read
// the damped decodes, and FP32 there reached 2.7e-2 on the sin component.
// Same outputs and layouts as particles_f64.cu.
#include "hfmm_internal.cuh"
#include "particles.cuh"

namespace hfmm {

namespace {

#ifndef HFMM_P2P_TPL
#define HFMM_P2P_TPL 1
#endif
constexpr int WARPS = 4;               // target leaves per CTA, one warp each
// targets per lane held at once (32 * TPL per pass); on the 1M-point p = 8 near
// field 1 was fastest (5.0 ms, against 6.6 for 2 and 8.0 for the former
// one-CTA-per-leaf kernel; same bits)
constexpr int TPL = HFMM_P2P_TPL;
constexpr int CHAIN = 128;             // sources per FP32 partial-sum chain

// sin and cos of a phase |x| <= SMALL_PHASE by their Taylor series about 0 (Horner
// form in x^2): the first omitted terms, x^13 / 13! and x^14 / 14!, stay below 3.2e-8
// and 3.3e-9 there, under the FP32 rounding of the pair arithmetic. Larger phases
// (big leaves at coarse levels, large k) take sincosf.
constexpr float SMALL_PHASE = 1.5f;
__device__ __forceinline__ void sincos_phase(float x, float* s, float* c) {
    if (fabsf(x) <= SMALL_PHASE) {
        const float x2 = x * x;
        float ps = -1.f / 39916800.f;
        ps = fmaf(ps, x2, 1.f / 362880.f);
        ps = fmaf(ps, x2, -1.f / 5040.f);
        ps = fmaf(ps, x2, 1.f / 120.f);
        ps = fmaf(ps, x2, -1.f / 6.f);
        ps = fmaf(ps, x2, 1.f);
        float pc = 1.f / 479001600.f;
        pc = fmaf(pc, x2, -1.f / 3628800.f);
        pc = fmaf(pc, x2, 1.f / 40320.f);
        pc = fmaf(pc, x2, -1.f / 720.f);
        pc = fmaf(pc, x2, 1.f / 24.f);
        pc = fmaf(pc, x2, -0.5f);
        *s = x * ps;
        *c = fmaf(pc, x2, 1.f);
    } else {
        sincosf(x, s, c);
    }
}

// One warp per target leaf: each lane keeps TPL targets in registers; the sources
// of each near leaf are staged 32 at a time in the warp's slice of shared memory
// (hi position + first charge column, lo position + second) and read back as
// broadcast loads, two per source; only __syncwarp orders the warp's own slice.
// The FP64 per-target sums live in shared memory, read and written once per chain of
// up to CHAIN sources, which keeps the kernel at 64 registers and 8 CTAs per SM (1M
// points, p = 8: the near field took 4.5 ms beside the upward pass at 96 registers,
// 4.2 at 72, 4.15 at 64).
template <int NF, int R, bool FIELD>
__global__ void __launch_bounds__(WARPS * 32, 8) k_p2p_mx(EvalView v, const int32_t* __restrict__ leaves,
                                                      int64_t nrows, const int32_t* __restrict__ off,
                                                      const int32_t* __restrict__ srcs, double* pot,
                                                      double* fld) {
    // Pair separations come from the FP32 hi/lo position pairs, (hi - hi') + (lo - lo'),
    // so each carries a relative error of about eps32 however close the points are
    // (clustered clouds); everything after that runs in FP32. The phase k r is an
    // FP32 product: r itself carries eps32, so a wider product would add nothing.
    constexpr int NA_ = NF * R * (FIELD ? 4 : 1);
    __shared__ float4 stage[WARPS][32][2];
    __shared__ double sacc[WARPS][NA_ * TPL][32];   // [sum][lane]: conflict-free per q
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row = (int64_t)blockIdx.x * WARPS + warp;
    if (row >= nrows) return;   // the whole warp leaves together
    const int t = leaves[row];
    const int s0t = v.leaf_start[t], cnt_t = v.counts[t];
    constexpr int NA = NF * R * (FIELD ? 4 : 1);
    const double C16 = 1.2621774483536189e-29;   // (16 * 2^-52)^2: the FP64 pair floor
    const double rt = v.rmax[t];
    const float kf = (float)v.k;
    const int64_t n = v.n;
    const int e0 = off[row], e1 = off[row + 1];
    float4(&sw)[32][2] = stage[warp];
    for (int i0 = 0; i0 < cnt_t; i0 += 32 * TPL) {
        float xh[TPL], yh[TPL], zh[TPL], xl[TPL], yl[TPL], zl[TPL];
        bool act[TPL];
        double(&acc)[NA_ * TPL][32] = sacc[warp];
#pragma unroll
        for (int u = 0; u < TPL; ++u) {
            const int i = i0 + 32 * u + lane;
            act[u] = i < cnt_t;
            const int64_t gi = s0t + (act[u] ? i : 0);
            xh[u] = v.pos_f[gi];
            yh[u] = v.pos_f[n + gi];
            zh[u] = v.pos_f[2 * n + gi];
            xl[u] = v.pos_f[3 * n + gi];
            yl[u] = v.pos_f[4 * n + gi];
            zl[u] = v.pos_f[5 * n + gi];
#pragma unroll
            for (int q = 0; q < NA; ++q) acc[u * NA + q][lane] = 0.0;
        }
        for (int e = e0; e < e1; ++e) {
            const int sb = srcs[e];
            const int s0 = v.leaf_start[sb], cnt = v.counts[sb];
            const double rs = rt + v.rmax[sb];
            const float thr = (float)(C16 * rs * rs);
            for (int c0 = 0; c0 < cnt; c0 += CHAIN) {
                const int cend = min(cnt, c0 + CHAIN);
                float a32[TPL][NA];
#pragma unroll
                for (int u = 0; u < TPL; ++u)
#pragma unroll
                    for (int q = 0; q < NA; ++q) a32[u][q] = 0.f;
                for (int b0 = c0; b0 < cend; b0 += 32) {
                    const int nbat = min(32, cend - b0);
                    __syncwarp();   // the previous batch has been read
                    if (lane < nbat) {
                        const int64_t gs = s0 + b0 + lane;
                        const float q0 = (float)v.q_s[gs];
                        const float q1 = R > 1 ? (float)v.q_s[n + gs] : 0.f;
                        sw[lane][0] = make_float4(v.pos_f[gs], v.pos_f[n + gs], v.pos_f[2 * n + gs], q0);
                        sw[lane][1] = make_float4(v.pos_f[3 * n + gs], v.pos_f[4 * n + gs],
                                                  v.pos_f[5 * n + gs], q1);
                    }
                    __syncwarp();
                    for (int j = 0; j < nbat; ++j) {
                        const float4 ph = sw[j][0], pl = sw[j][1];
                        const float sq[2] = {ph.w, pl.w};
#pragma unroll
                        for (int u = 0; u < TPL; ++u) {
                            const float dx = (xh[u] - ph.x) + (xl[u] - pl.x);
                            const float dy = (yh[u] - ph.y) + (yl[u] - pl.y);
                            const float dz = (zh[u] - ph.z) + (zl[u] - pl.z);
                            const float d2 = dx * dx + dy * dy + dz * dz;
                            // pairs under the floor (the target itself) contribute nothing
                            const float ir = d2 > thr ? rsqrtf(d2) : 0.f;
                            const float rr = d2 * ir;
                            const float kr = kf * rr;
                            float sn, cs_;
                            if (v.yukawa)   // the kernel seam (particles.cuh): one family
                                sn = cs_ = __expf(-kr) * 0.0795774715f;
                            else
                                sincos_phase(kr, &sn, &cs_);
                            const float w[2] = {cs_ * ir, sn * ir};
                            float wf[2] = {0.f, 0.f};
                            if (FIELD) {
                                const float ir3 = ir * ir * ir;
                                wf[0] = (cs_ + kr * sn) * ir3;
                                wf[1] = (sn - kr * cs_) * ir3;
                            }
#pragma unroll
                            for (int f = 0; f < NF; ++f)
#pragma unroll
                                for (int r = 0; r < R; ++r) {
                                    const float qv = sq[r];
                                    a32[u][f * R + r] += qv * w[f];
                                    if (FIELD) {
                                        const float qw = qv * wf[f];
                                        a32[u][NF * R + (f * R + r) * 3 + 0] += qw * dx;
                                        a32[u][NF * R + (f * R + r) * 3 + 1] += qw * dy;
                                        a32[u][NF * R + (f * R + r) * 3 + 2] += qw * dz;
                                    }
                                }
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < TPL; ++u)
#pragma unroll
                    for (int q = 0; q < NA; ++q) acc[u * NA + q][lane] += (double)a32[u][q];
            }
        }
#pragma unroll
        for (int u = 0; u < TPL; ++u) {
            if (!act[u]) continue;
            const int64_t gi = s0t + i0 + 32 * u + lane;
#pragma unroll
            for (int q = 0; q < NF * R; ++q) pot[q * n + gi] = acc[u * NA + q][lane];
            if (FIELD)
#pragma unroll
                for (int q = 0; q < NF * R * 3; ++q) fld[q * n + gi] = acc[u * NA + NF * R + q][lane];
        }
    }
}

template <int NF, int R, bool FIELD>
void impl(const ParticlePass& p, cudaStream_t s) {
    if (p.op != ParticleOp::P2P)
        throw Error{HFMM_ERR_STATE, "particles_mixed: only the near field runs in FP32"};
    HFMM_LAUNCH((k_p2p_mx<NF, R, FIELD>), (unsigned)ceil_div(p.nrows, WARPS), WARPS * 32, 0, s, p.v,
                p.rows, p.nrows, p.off, p.srcs, p.pot, p.fld);
}

}  // namespace

void particles_mixed(const ParticlePass& p, cudaStream_t s) {
    if (p.nrows == 0) return;
    const int key = (p.nf - 1) * 4 + (p.R - 1) * 2 + (p.field ? 1 : 0);
    switch (key) {
        case 0: impl<1, 1, false>(p, s); break;
        case 1: impl<1, 1, true>(p, s); break;
        case 2: impl<1, 2, false>(p, s); break;
        case 3: impl<1, 2, true>(p, s); break;
        case 4: impl<2, 1, false>(p, s); break;
        case 5: impl<2, 1, true>(p, s); break;
        case 6: impl<2, 2, false>(p, s); break;
        case 7: impl<2, 2, true>(p, s); break;
        default: throw Error{HFMM_ERR_ARG, "particles_mixed: bad configuration"};
    }
}

}  // namespace hfmm
