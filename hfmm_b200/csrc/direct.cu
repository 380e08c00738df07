// Direct-sum referee: phi_t = sum_{s: r > 0} q_s e^{ikr} / r at sampled targets
// (test.py:11-18), and the field -grad phi = sum q_s e^{ikr} (1 - ikr) / r^3 (x_t - x_s).
// With the screened-Coulomb kernel (yukawa != 0, k = kappa): phi_t = sum q_s G(r),
// G = exp(-kappa r) / (4 pi r), field sum q_s (1 + kappa r) exp(-kappa r) / (4 pi r^3) d.
//
// Sources are split into n_split contiguous chunks; each (target block, chunk)
// CTA writes its partial sums to scratch, and a second kernel adds the chunks
// in a fixed order, so the result does not depend on scheduling.
#include "hfmm_internal.cuh"

#include <algorithm>

namespace hfmm {

namespace {

// sin and cos of a phase: Cody-Waite reduction against pi/2 with a two-part constant
// (1.5707963267948966 + 6.123233995736766e-17, the first being pi/2 rounded to FP64,
// both from pi itself) done with FMAs, so r = x - n pi/2 is exact to about 1e-28 for
// |x| <= 1e5; then the Taylor series of sin and cos on |r| <= pi/4 (through r^15 and
// r^16: the first omitted terms stay under 4.7e-17 and 2.1e-18) and the quadrant
// n mod 4. Larger phases take sincos.
__device__ __forceinline__ void sincos_reduced(double x, double* s, double* c) {
    if (!(fabs(x) <= 1.0e5)) {
        sincos(x, s, c);
        return;
    }
    const double n = rint(x * 0.6366197723675814);   // x / (pi / 2), rounded
    double r = fma(-n, 1.5707963267948966, x);
    r = fma(-n, 6.123233995736766e-17, r);
    const double r2 = r * r;
    double ps = 1.0 / 1307674368000.0;               // 1/15!
    ps = fma(ps, r2, -1.0 / 6227020800.0);           // -1/13!
    ps = fma(ps, r2, 1.0 / 39916800.0);              // 1/11!
    ps = fma(ps, r2, -1.0 / 362880.0);               // -1/9!
    ps = fma(ps, r2, 1.0 / 5040.0);                  // 1/7!
    ps = fma(ps, r2, -1.0 / 120.0);                  // -1/5!
    ps = fma(ps, r2, 1.0 / 6.0);                     // 1/3!
    double pc = -1.0 / 20922789888000.0;             // -1/16!
    pc = fma(pc, r2, 1.0 / 87178291200.0);           // 1/14!
    pc = fma(pc, r2, -1.0 / 479001600.0);            // -1/12!
    pc = fma(pc, r2, 1.0 / 3628800.0);               // 1/10!
    pc = fma(pc, r2, -1.0 / 40320.0);                // -1/8!
    pc = fma(pc, r2, 1.0 / 720.0);                   // 1/6!
    pc = fma(pc, r2, -1.0 / 24.0);                   // -1/4!
    pc = fma(pc, r2, 0.5);                           // 1/2!
    const double sr = fma(-r * r2, ps, r);           // sin r = r - r^3 (1/3! - ...)
    const double cr = fma(-r2, pc, 1.0);             // cos r = 1 - r^2 (1/2! - ...)
    switch ((int)((long long)n & 3)) {
        case 0: *s = sr; *c = cr; break;
        case 1: *s = cr; *c = -sr; break;
        case 2: *s = -sr; *c = -cr; break;
        default: *s = -cr; *c = sr; break;
    }
}

constexpr int DT = 128;        // targets per CTA
constexpr int DSTAGE = 256;    // sources staged per pass
constexpr int NV = 8;          // phi re/im + field 3 x re/im

__global__ void __launch_bounds__(DT) k_direct_partial(const double* __restrict__ pos,
                                                       const double* __restrict__ q_re,
                                                       const double* __restrict__ q_im, int64_t n,
                                                       const int32_t* __restrict__ tg, int64_t n_t,
                                                       double k, int field, int n_split,
                                                       double* scratch, int* err, int yukawa) {
    __shared__ double sx[DSTAGE], sy[DSTAGE], sz[DSTAGE], sqr[DSTAGE], sqi[DSTAGE];
    const int64_t ti = blockIdx.x * (int64_t)DT + threadIdx.x;
    const int split = blockIdx.y;
    const int64_t chunk = (n + n_split - 1) / n_split;
    const int64_t lo = split * chunk, hi = (lo + chunk < n) ? lo + chunk : n;
    bool act = ti < n_t;
    double x = 0, y = 0, z = 0;
    if (act) {
        int64_t t = tg[ti];
        if (t < 0 || t >= n) {
            atomicOr(err, ERRF_BOUNDS);
            act = false;
        } else {
            x = pos[3 * t];
            y = pos[3 * t + 1];
            z = pos[3 * t + 2];
        }
    }
    double acc[NV] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t p0 = lo; p0 < hi; p0 += DSTAGE) {
        __syncthreads();
        for (int i = threadIdx.x; i < DSTAGE; i += DT) {
            int64_t s = p0 + i;
            if (s < hi) {
                sx[i] = pos[3 * s];
                sy[i] = pos[3 * s + 1];
                sz[i] = pos[3 * s + 2];
                sqr[i] = q_re[s];
                sqi[i] = q_im ? q_im[s] : 0.0;
            }
        }
        __syncthreads();
        if (!act) continue;
        const int np = (int)((hi - p0 < DSTAGE) ? hi - p0 : DSTAGE);
        for (int i = 0; i < np; ++i) {
            double dx = x - sx[i], dy = y - sy[i], dz = z - sz[i];
            double r2 = dx * dx + dy * dy + dz * dz;
            if (!(r2 > 0.0)) continue;
            double ir = rsqrt(r2), r = r2 * ir;
            double kr = k * r, sn, cs;
            if (yukawa) {   // real kernel: w = G, field weight (1 + kr) G / r^2
                cs = exp(-kr) * 0.07957747154594767;
                sn = 0.0;
            } else {
                sincos_reduced(kr, &sn, &cs);
            }
            // w = e^{ikr}/r; q w
            double wr = cs * ir, wi = sn * ir;
            acc[0] += sqr[i] * wr - sqi[i] * wi;
            acc[1] += sqr[i] * wi + sqi[i] * wr;
            if (field) {
                // e^{ikr}(1 - ikr)/r^3 = ((cs + kr sn) + i (sn - kr cs)) / r^3
                double ir3 = ir * ir * ir;
                double fr = (cs + kr * sn) * ir3, fi = (sn - kr * cs) * ir3;
                if (yukawa) {
                    fr = cs * (1.0 + kr) * ir3;
                    fi = 0.0;
                }
                double gr = sqr[i] * fr - sqi[i] * fi, gi = sqr[i] * fi + sqi[i] * fr;
                acc[2] += gr * dx;
                acc[3] += gi * dx;
                acc[4] += gr * dy;
                acc[5] += gi * dy;
                acc[6] += gr * dz;
                acc[7] += gi * dz;
            }
        }
    }
    if (act)
        for (int v = 0; v < NV; ++v) scratch[((int64_t)split * n_t + ti) * NV + v] = acc[v];
}

// The chunks' partial sums of one (target, value) pair added by one warp: lane j takes
// chunks j, j + 32, ... in order, then a fixed shuffle tree adds the lanes, so the
// result does not depend on scheduling. (One thread per target had walked all chunks
// serially: 0.26 ms for the 256-target check at 1e6 sources.)
__global__ void k_direct_reduce(const double* __restrict__ scratch, int64_t n_t, int n_split,
                                int field, double* phi, double* fld) {
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n_t * NV) return;
    const int64_t ti = w / NV;
    const int v = (int)(w % NV);
    if (!field && v >= 2) return;
    double acc = 0.0;
    for (int s = lane; s < n_split; s += 32) acc += scratch[((int64_t)s * n_t + ti) * NV + v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane != 0) return;
    if (v < 2) phi[2 * ti + v] = acc;
    else if (fld) fld[(ti * 3 + (v - 2) / 2) * 2 + (v - 2) % 2] = acc;
}

}  // namespace

int direct_splits(int64_t n, int64_t n_t) {
    int64_t tblocks = ceil_div(std::max<int64_t>(n_t, 1), DT);
    int64_t want = ceil_div(4 * 148, tblocks);                 // about 4 CTAs per SM
    int64_t by_work = ceil_div(std::max<int64_t>(n, 1), 2048);  // at least 2048 sources a split
    return (int)std::max<int64_t>(1, std::min<int64_t>(want, by_work));
}

void direct_sum(const double* pos, const double* q_re, const double* q_im, int64_t n,
                const int32_t* targets, int64_t n_t, double k, double* phi, double* fld,
                double* scratch, int n_split, cudaStream_t s, int* err, int yukawa) {
    if (n_t == 0) return;
    dim3 grid((unsigned)ceil_div(n_t, DT), (unsigned)n_split);
    HFMM_LAUNCH(k_direct_partial, grid, DT, 0, s, pos, q_re, q_im, n, targets, n_t, k,
                fld ? 1 : 0, n_split, scratch, err, yukawa);
    HFMM_LAUNCH(k_direct_reduce, (unsigned)ceil_div(n_t * NV * 32, 256), 256, 0, s, scratch, n_t, n_split,
                fld ? 1 : 0, phi, fld);
}

}  // namespace hfmm
