// Mixed-precision particle kernels: P2P, P2M/P2L and L2P/M2P with FP32 pair
// arithmetic (the role of the mixed near field of near.py:140-160 and 222-232),
// and FP64 only where stability needs it:
//   * the phase k r is reduced modulo pi/2 in FP64 (Cody-Waite with a two-part
//     pi/2) and only the reduced argument in [-pi/4, pi/4] goes to FP32 sincosf;
//   * sums run in FP32 over short chains (one source leaf, or one lane's share of
//     the surface points) and are combined in FP64, as is the final per-target sum.
// Same outputs and layouts as particles_f64.cu.
#include "hfmm_internal.cuh"
#include "particles.cuh"

namespace hfmm {

namespace {

constexpr int STAGE = 128;
constexpr double TWO_OVER_PI = 0.63661977236758134308;
constexpr double PIO2_HI = 1.5707963267948966192;      // nearest double to pi/2
constexpr double PIO2_LO = 6.1232339957367660359e-17;  // pi/2 - PIO2_HI

// sin and cos of k*r: FP64 reduction of the phase, FP32 evaluation.
__device__ __forceinline__ void sincos_kr(double k, float r, float& s, float& c, float& krf) {
    const double kr = k * (double)r;
    const double n = rint(kr * TWO_OVER_PI);
    const double red = fma(-n, PIO2_HI, kr) - n * PIO2_LO;
    float sr, cr;
    sincosf((float)red, &sr, &cr);
    const int q = ((int)(long long)n) & 3;
    s = q == 0 ? sr : q == 1 ? cr : q == 2 ? -sr : -cr;
    c = q == 0 ? cr : q == 1 ? -sr : q == 2 ? -cr : sr;
    krf = (float)kr;
}

template <int NF, int R, bool FIELD>
__global__ void __launch_bounds__(128) k_p2p_mx(EvalView v, const int32_t* __restrict__ leaves,
                                               const int32_t* __restrict__ off,
                                               const int32_t* __restrict__ srcs, double* pot,
                                               double* fld) {
    // Pair separations are formed in FP64 and rounded once to FP32, so each pair's
    // distance carries a relative error of eps32 however close the points are
    // (clustered clouds); everything after that runs in FP32.
    __shared__ double sx[STAGE], sy[STAGE], sz[STAGE];
    __shared__ float sq[R][STAGE];
    const int row = blockIdx.x;
    const int t = leaves[row];
    const int s0t = v.leaf_start[t], cnt_t = v.counts[t];
    constexpr int NA = NF * R * (FIELD ? 4 : 1);
    const double C16 = 1.2621774483536189e-29;   // (16 * 2^-52)^2: the FP64 pair floor
    const double rt = v.rmax[t];
    for (int i0 = 0; i0 < cnt_t; i0 += blockDim.x) {
        const int i = i0 + threadIdx.x;
        const bool act = i < cnt_t;
        double x = 0, y = 0, z = 0;
        if (act) {
            x = v.pos_s[s0t + i];
            y = v.pos_s[v.n + s0t + i];
            z = v.pos_s[2 * v.n + s0t + i];
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
                    int64_t gi = s0 + p0 + k;
                    sx[k] = v.pos_s[gi];
                    sy[k] = v.pos_s[v.n + gi];
                    sz[k] = v.pos_s[2 * v.n + gi];
#pragma unroll
                    for (int r = 0; r < R; ++r) sq[r][k] = (float)v.q_s[r * v.n + gi];
                }
                __syncthreads();
                if (!act) continue;
                const int np = min(STAGE, cnt - p0);
                float a32[NA];
#pragma unroll
                for (int q = 0; q < NA; ++q) a32[q] = 0.f;
                for (int k = 0; k < np; ++k) {
                    const float dx = (float)(x - sx[k]), dy = (float)(y - sy[k]), dz = (float)(z - sz[k]);
                    const float d2 = dx * dx + dy * dy + dz * dz;
                    if (!(d2 > thr)) continue;
                    const float ir = rsqrtf(d2);
                    const float rr = d2 * ir;
                    float sn, cs_, kr;
                    sincos_kr(v.k, rr, sn, cs_, kr);
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
            for (int q = 0; q < NF * R; ++q) pot[q * v.n + gi] = acc[q];
            if (FIELD)
#pragma unroll
                for (int q = 0; q < NF * R * 3; ++q) fld[q * v.n + gi] = acc[NF * R + q];
        }
    }
}

// P2M (check surface of the leaf) / P2L (downward check surface of an X-list target).
template <int NF, int R>
__global__ void __launch_bounds__(256) k_surface_from_particles_mx(
    EvalView v, const int32_t* __restrict__ tgt_boxes, const int32_t* __restrict__ off,
    const int32_t* __restrict__ srcs, const double* __restrict__ surf, int only_level,
    double* check, int64_t fam_stride, int accumulate) {
    __shared__ float sx[STAGE], sy[STAGE], sz[STAGE], sq[R][STAGE];
    const int row = blockIdx.x;
    const int b = tgt_boxes[row];
    const int lvl = v.lvls[b];
    if (lvl < 2 || (only_level >= 0 && lvl != only_level)) return;
    const double h = v.hbox[b];
    const double cb[3] = {v.centre[b], v.centre[v.nb + b], v.centre[2 * v.nb + b]};
    const int e0 = off ? off[row] : 0, e1 = off ? off[row + 1] : 1;
    for (int j0 = 0; j0 < v.n_s; j0 += blockDim.x) {
        const int j = j0 + threadIdx.x;
        const bool jok = j < v.n_s;
        float px = 0, py = 0, pz = 0;   // surface point relative to the box centre
        if (jok) {
            px = (float)(surf[j] * h);
            py = (float)(surf[v.n_s + j] * h);
            pz = (float)(surf[2 * v.n_s + j] * h);
        }
        double acc[NF][R];
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
            for (int r = 0; r < R; ++r) acc[f][r] = 0.0;
        for (int e = e0; e < e1; ++e) {
            const int sb = srcs ? srcs[e] : b;
            const int s0 = v.leaf_start[sb], cnt = v.counts[sb];
            const double cs[3] = {v.centre[sb], v.centre[v.nb + sb], v.centre[2 * v.nb + sb]};
            const float ox = px + (float)(cb[0] - cs[0]);
            const float oy = py + (float)(cb[1] - cs[1]);
            const float oz = pz + (float)(cb[2] - cs[2]);
            for (int p0 = 0; p0 < cnt; p0 += STAGE) {
                __syncthreads();
                for (int i = threadIdx.x; i < STAGE && p0 + i < cnt; i += blockDim.x) {
                    int64_t gi = s0 + p0 + i;
                    sx[i] = (float)(v.pos_s[gi] - cs[0]);
                    sy[i] = (float)(v.pos_s[v.n + gi] - cs[1]);
                    sz[i] = (float)(v.pos_s[2 * v.n + gi] - cs[2]);
#pragma unroll
                    for (int r = 0; r < R; ++r) sq[r][i] = (float)v.q_s[r * v.n + gi];
                }
                __syncthreads();
                if (!jok) continue;
                const int np = min(STAGE, cnt - p0);
                float a32[NF][R];
#pragma unroll
                for (int f = 0; f < NF; ++f)
#pragma unroll
                    for (int r = 0; r < R; ++r) a32[f][r] = 0.f;
                for (int i = 0; i < np; ++i) {
                    const float dx = ox - sx[i], dy = oy - sy[i], dz = oz - sz[i];
                    const float d2 = dx * dx + dy * dy + dz * dz;
                    const float ir = rsqrtf(d2);
                    float sn, cs_, kr;
                    sincos_kr(v.k, d2 * ir, sn, cs_, kr);
                    const float wc = cs_ * ir, ws = sn * ir;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        a32[0][r] += sq[r][i] * wc;
                        if (NF == 2) a32[NF - 1][r] += sq[r][i] * ws;
                    }
                }
#pragma unroll
                for (int f = 0; f < NF; ++f)
#pragma unroll
                    for (int r = 0; r < R; ++r) acc[f][r] += (double)a32[f][r];
            }
        }
        if (jok) {
#pragma unroll
            for (int f = 0; f < NF; ++f)
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    double* o = check + f * fam_stride + ((int64_t)b * R + r) * v.ld + j;
                    *o = accumulate ? *o + acc[f][r] : acc[f][r];
                }
        }
    }
}

// L2P (downward equivalent surface of the leaf) / M2P (upward equivalent surfaces of
// W-list sources): warp per particle, lanes over surface points, FP32 per lane,
// FP64 warp reduction.
template <int NF, int R, bool FIELD>
__global__ void __launch_bounds__(256) k_particles_from_surface_mx(
    EvalView v, const int32_t* __restrict__ tgt_leaves, const int32_t* __restrict__ off,
    const int32_t* __restrict__ srcs, const double* __restrict__ surf,
    const double* __restrict__ dens, int64_t fam_stride, double* pot, double* fld) {
    extern __shared__ float shf[];
    float* dn = shf;                          // [NF][R][n_s]
    float* ex = shf + NF * R * v.n_s;         // [3][n_s], relative to the target leaf centre
    const int row = blockIdx.x;
    const int t = tgt_leaves[row];
    if (v.lvls[t] < 2 && !off) return;
    const int s0 = v.leaf_start[t], cnt = v.counts[t];
    const double ct[3] = {v.centre[t], v.centre[v.nb + t], v.centre[2 * v.nb + t]};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int e0 = off ? off[row] : 0, e1 = off ? off[row + 1] : 1;
    constexpr int NA = NF * R * (FIELD ? 4 : 1);
    for (int e = e0; e < e1; ++e) {
        const int sb = srcs ? srcs[e] : t;
        const double h = v.hbox[sb];
        const double dc[3] = {v.centre[sb] - ct[0], v.centre[v.nb + sb] - ct[1],
                              v.centre[2 * v.nb + sb] - ct[2]};
        __syncthreads();
        for (int j = threadIdx.x; j < v.n_s; j += blockDim.x) {
#pragma unroll
            for (int a = 0; a < 3; ++a) ex[a * v.n_s + j] = (float)(surf[a * v.n_s + j] * h + dc[a]);
#pragma unroll
            for (int f = 0; f < NF; ++f)
#pragma unroll
                for (int r = 0; r < R; ++r)
                    dn[(f * R + r) * v.n_s + j] =
                        (float)dens[f * fam_stride + ((int64_t)sb * R + r) * v.ld + j];
        }
        __syncthreads();
        for (int i = warp; i < cnt; i += nw) {
            const int64_t gi = s0 + i;
            const float x = (float)(v.pos_s[gi] - ct[0]);
            const float y = (float)(v.pos_s[v.n + gi] - ct[1]);
            const float z = (float)(v.pos_s[2 * v.n + gi] - ct[2]);
            float a32[NA];
#pragma unroll
            for (int q = 0; q < NA; ++q) a32[q] = 0.f;
            for (int j = lane; j < v.n_s; j += 32) {
                const float dx = x - ex[j], dy = y - ex[v.n_s + j], dz = z - ex[2 * v.n_s + j];
                const float d2 = dx * dx + dy * dy + dz * dz;
                const float ir = rsqrtf(d2);
                float sn, cs_, kr;
                sincos_kr(v.k, d2 * ir, sn, cs_, kr);
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
                        const float d = dn[(f * R + r) * v.n_s + j];
                        a32[f * R + r] += d * w[f];
                        if (FIELD) {
                            const float dw = d * wf[f];
                            a32[NF * R + (f * R + r) * 3 + 0] += dw * dx;
                            a32[NF * R + (f * R + r) * 3 + 1] += dw * dy;
                            a32[NF * R + (f * R + r) * 3 + 2] += dw * dz;
                        }
                    }
            }
            double acc[NA];
#pragma unroll
            for (int q = 0; q < NA; ++q) {
                acc[q] = (double)a32[q];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
            }
            if (lane == 0) {
#pragma unroll
                for (int q = 0; q < NF * R; ++q) pot[q * v.n + gi] += acc[q];
                if (FIELD)
#pragma unroll
                    for (int q = 0; q < NF * R * 3; ++q) fld[q * v.n + gi] += acc[NF * R + q];
            }
        }
    }
}

template <int NF, int R, bool FIELD>
void impl(const ParticlePass& p, cudaStream_t s) {
    const EvalView& v = p.v;
    switch (p.op) {
        case ParticleOp::P2M:
            HFMM_LAUNCH((k_surface_from_particles_mx<NF, R>), p.nrows, 256, 0, s, v, p.rows, p.off,
                        p.srcs, p.surf, -1, p.out, p.fam_stride, 0);
            break;
        case ParticleOp::P2L:
            HFMM_LAUNCH((k_surface_from_particles_mx<NF, R>), p.nrows, 256, 0, s, v, p.rows, p.off,
                        p.srcs, p.surf, p.level, p.out, p.fam_stride, 1);
            break;
        case ParticleOp::L2P:
        case ParticleOp::M2P: {
            size_t smem = (size_t)(NF * R + 3) * v.n_s * sizeof(float);
            auto kern = k_particles_from_surface_mx<NF, R, FIELD>;
            HFMM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            HFMM_LAUNCH(kern, p.nrows, 256, smem, s, v, p.rows, p.off, p.srcs, p.surf, p.dens,
                        p.fam_stride, p.pot, p.fld);
            break;
        }
        case ParticleOp::P2P:
            HFMM_LAUNCH((k_p2p_mx<NF, R, FIELD>), p.nrows, 128, 0, s, v, p.rows, p.off, p.srcs,
                        p.pot, p.fld);
            break;
        case ParticleOp::COMBINE:
            throw Error{HFMM_ERR_STATE, "particles_mixed: combine runs in particles_f64"};
    }
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
