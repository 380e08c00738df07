// Shared view of a plan for the particle kernels (plain and mixed precision).
#pragma once
#include "hfmm_internal.cuh"

namespace hfmm {

struct EvalView {
    int64_t n, nb;
    int n_s, ld;
    double k;
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

void particles_f64(const ParticlePass& p, cudaStream_t s);
void particles_mixed(const ParticlePass& p, cudaStream_t s);
void gather_charges(int64_t n, const int32_t* sidx, const double* q_re, const double* q_im,
                    double* q_s, cudaStream_t s);

}  // namespace hfmm
