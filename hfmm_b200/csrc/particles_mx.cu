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

constexpr int STAGE = 128;

template <int NF, int R, bool FIELD>
__global__ void __launch_bounds__(128) k_p2p_mx(EvalView v, const int32_t* __restrict__ leaves,
                                               const int32_t* __restrict__ off,
                                               const int32_t* __restrict__ srcs, double* pot,
                                               double* fld) {
    // Pair separations come from the FP32 hi/lo position pairs, (hi - hi') + (lo - lo'),
    // so each carries a relative error of about eps32 however close the points are
    // (clustered clouds); everything after that runs in FP32. The phase k r is an
    // FP32 product: r itself carries eps32, so a wider product would add nothing.
    __shared__ float sxh[STAGE], syh[STAGE], szh[STAGE], sxl[STAGE], syl[STAGE], szl[STAGE];
    __shared__ float sq[R][STAGE];
    const int row = blockIdx.x;
    const int t = leaves[row];
    const int s0t = v.leaf_start[t], cnt_t = v.counts[t];
    constexpr int NA = NF * R * (FIELD ? 4 : 1);
    const double C16 = 1.2621774483536189e-29;   // (16 * 2^-52)^2: the FP64 pair floor
    const double rt = v.rmax[t];
    const float kf = (float)v.k;
    const int64_t n = v.n;
    for (int i0 = 0; i0 < cnt_t; i0 += blockDim.x) {
        const int i = i0 + threadIdx.x;
        const bool act = i < cnt_t;
        float xh = 0, yh = 0, zh = 0, xl = 0, yl = 0, zl = 0;
        if (act) {
            const int64_t gi = s0t + i;
            xh = v.pos_f[gi];
            yh = v.pos_f[n + gi];
            zh = v.pos_f[2 * n + gi];
            xl = v.pos_f[3 * n + gi];
            yl = v.pos_f[4 * n + gi];
            zl = v.pos_f[5 * n + gi];
        }
        double acc[NA];
#pragma unroll
        for (int q = 0; q < NA; ++q) acc[q] = 0.0;
        for (int e = off[row]; e < off[row + 1]; ++e) {
            const int sb = srcs[e];
            const int s0 = v.leaf_start[sb], cnt = v.counts[sb];
            const double rs = rt + v.rmax[sb];
            const float thr = (float)(C16 * rs * rs);
            for (int p0 = 0; p0 < cnt; p0 += STAGE) {
                __syncthreads();
                for (int k = threadIdx.x; k < STAGE && p0 + k < cnt; k += blockDim.x) {
                    const int64_t gi = s0 + p0 + k;
                    sxh[k] = v.pos_f[gi];
                    syh[k] = v.pos_f[n + gi];
                    szh[k] = v.pos_f[2 * n + gi];
                    sxl[k] = v.pos_f[3 * n + gi];
                    syl[k] = v.pos_f[4 * n + gi];
                    szl[k] = v.pos_f[5 * n + gi];
#pragma unroll
                    for (int r = 0; r < R; ++r) sq[r][k] = (float)v.q_s[r * n + gi];
                }
                __syncthreads();
                if (!act) continue;
                const int np = min(STAGE, cnt - p0);
                float a32[NA];
#pragma unroll
                for (int q = 0; q < NA; ++q) a32[q] = 0.f;
                for (int k = 0; k < np; ++k) {
                    const float dx = (xh - sxh[k]) + (xl - sxl[k]);
                    const float dy = (yh - syh[k]) + (yl - syl[k]);
                    const float dz = (zh - szh[k]) + (zl - szl[k]);
                    const float d2 = dx * dx + dy * dy + dz * dz;
                    if (!(d2 > thr)) continue;
                    const float ir = rsqrtf(d2);
                    const float rr = d2 * ir;
                    const float kr = kf * rr;
                    float sn, cs_;
                    sincosf(kr, &sn, &cs_);
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
                            const float qv = sq[r][k];
                            a32[f * R + r] += qv * w[f];
                            if (FIELD) {
                                const float qw = qv * wf[f];
                                a32[NF * R + (f * R + r) * 3 + 0] += qw * dx;
                                a32[NF * R + (f * R + r) * 3 + 1] += qw * dy;
                                a32[NF * R + (f * R + r) * 3 + 2] += qw * dz;
                            }
                        }
                }
#pragma unroll
                for (int q = 0; q < NA; ++q) acc[q] += (double)a32[q];
            }
        }
        if (act) {
            const int64_t gi = s0t + i;
#pragma unroll
            for (int q = 0; q < NF * R; ++q) pot[q * n + gi] = acc[q];
            if (FIELD)
#pragma unroll
                for (int q = 0; q < NF * R * 3; ++q) fld[q * n + gi] = acc[NF * R + q];
        }
    }
}

template <int NF, int R, bool FIELD>
void impl(const ParticlePass& p, cudaStream_t s) {
    if (p.op != ParticleOp::P2P)
        throw Error{HFMM_ERR_STATE, "particles_mixed: only the near field runs in FP32"};
    HFMM_LAUNCH((k_p2p_mx<NF, R, FIELD>), p.nrows, 128, 0, s, p.v, p.rows, p.off, p.srcs,
                p.pot, p.fld);
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
