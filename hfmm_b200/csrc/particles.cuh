// Shared view of a plan for the particle kernels (plain and mixed precision).
#pragma once
#include "hfmm_internal.cuh"

namespace hfmm {

struct EvalView {
    int64_t n, nb;
    int n_s, ld;
    double k;                  // Helmholtz wavenumber, or the screening constant kappa
    int yukawa;                // 0: Helmholtz (two families); 1: exp(-kappa r) / (4 pi r)
    const double* pos_s;       // 3 x n, leaf-major sorted
    const float* pos_f;        // 6 x n: FP32 hi parts x|y|z, then lo parts (pos = hi + lo)
    const double* q_s;         // R x n, leaf-major sorted
    const int32_t* leaf_start;
    const int32_t* counts;
    const int32_t* lvls;
    const double* centre;      // 3 x nb
    const double* hbox;
    const double* rmax;
};

enum class ParticleOp { P2M, P2L, L2P, M2P, P2P, COMBINE };

struct ParticlePass {
    ParticleOp op;
    EvalView v;
    int nf = 1, R = 1;
    bool field = false;
    const int32_t* rows = nullptr;   // target boxes (P2M/P2L/L2P/M2P/P2P) or sort_idx (COMBINE)
    int64_t nrows = 0;
    const int32_t* off = nullptr;    // CSR offsets into srcs (P2L/M2P/P2P)
    const int32_t* srcs = nullptr;
    const double* surf = nullptr;    // unit surface (3 x n_s)
    const double* dens = nullptr;    // equivalent densities [fam][box][R][ld]
    double* out = nullptr;           // check potentials [fam][box][R][ld]
    int64_t fam_stride = 0;
    int level = -1;
    double* pot = nullptr;           // [fam*R][n]
    double* fld = nullptr;           // [fam*R*3][n]
    double* phi = nullptr;           // COMBINE outputs (complex interleaved)
    double* E = nullptr;
};

// sin and cos of a phase |x| <= 1.5 by their Taylor series about 0 (Horner form in
// x^2, through x^21 and x^22): the first omitted terms, x^23 / 23! and x^24 / 24!, stay
// below 4.4e-19 and 2.8e-20 there, under FP64 rounding. Larger phases take sincos.
__device__ __forceinline__ void sincos_phase64(double x, double* s, double* c) {
    if (fabs(x) <= 1.5) {
        const double x2 = x * x;
        // sin x / x = sum (-1)^i x^(2i) / (2i+1)!,  cos x = sum (-1)^i x^(2i) / (2i)!
        double ps = -1.0 / 51090942171709440000.0;   // -1/21!
        ps = fma(ps, x2, 1.0 / 121645100408832000.0);   // 1/19!
        ps = fma(ps, x2, -1.0 / 355687428096000.0);     // -1/17!
        ps = fma(ps, x2, 1.0 / 1307674368000.0);        // 1/15!
        ps = fma(ps, x2, -1.0 / 6227020800.0);          // -1/13!
        ps = fma(ps, x2, 1.0 / 39916800.0);             // 1/11!
        ps = fma(ps, x2, -1.0 / 362880.0);              // -1/9!
        ps = fma(ps, x2, 1.0 / 5040.0);                 // 1/7! (sign applied below)
        ps = fma(ps, x2, -1.0 / 120.0);
        ps = fma(ps, x2, 1.0 / 6.0);
        double pc = 1.0 / 1124000727777607680000.0;     // 1/22!
        pc = fma(pc, x2, -1.0 / 2432902008176640000.0); // -1/20!
        pc = fma(pc, x2, 1.0 / 6402373705728000.0);     // 1/18!
        pc = fma(pc, x2, -1.0 / 20922789888000.0);      // -1/16!
        pc = fma(pc, x2, 1.0 / 87178291200.0);          // 1/14!
        pc = fma(pc, x2, -1.0 / 479001600.0);           // -1/12!
        pc = fma(pc, x2, 1.0 / 3628800.0);              // 1/10!
        pc = fma(pc, x2, -1.0 / 40320.0);               // -1/8!
        pc = fma(pc, x2, 1.0 / 720.0);                  // 1/6!
        pc = fma(pc, x2, -1.0 / 24.0);                  // -1/4!
        pc = fma(pc, x2, 0.5);                          // 1/2!
        *s = fma(-x * x2, ps, x);                       // x - x^3 (1/3! - x^2/5! + ...)
        *c = fma(-x2, pc, 1.0);                         // 1 - x^2 (1/2! - x^2/4! + ...)
    } else {
        sincos(x, s, c);
    }
}

// The kernel seam of the particle kernels. Helmholtz: (sn, cs) = sin, cos of the phase
// kr, so family 0 is cs / r, family 1 sn / r and their field weights (cs + kr sn) / r^3
// and (sn - kr cs) / r^3 (HFMM.py:25-40). The screened-Coulomb kernel (one family,
// jaxfmm/kernels/yukawa/kernel.py:36-75; kappa = 0 is Laplace,
// kernels/laplace/kernel.py:40-104) puts exp(-kr) / (4 pi) in both slots, so family 0's
// value cs / r and field weight (cs + kr sn) / r^3 = (1 + kr) exp(-kr) / (4 pi r^3) come
// out of the same expressions.
constexpr double INV_4PI = 0.07957747154594767;
__device__ __forceinline__ void kernel_pair64(int yukawa, double kr, double* sn, double* cs) {
    if (yukawa) {
        const double e = exp(-kr) * INV_4PI;
        *sn = e;
        *cs = e;
    } else {
        sincos_phase64(kr, sn, cs);
    }
}

void particles_f64(const ParticlePass& p, cudaStream_t s);
void particles_mixed(const ParticlePass& p, cudaStream_t s);
void gather_charges(int64_t n, const int32_t* sidx, const double* q_re, const double* q_im,
                    double* q_s, cudaStream_t s);

}  // namespace hfmm
