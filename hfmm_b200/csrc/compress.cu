// Compressed M2L of the mixed path: the 316 M2L matrices of a level share their
// dominant subspace U (n_s x r), so K_d ~ U C_d U^T with C_d = U^T K_d U (r x r).
// The M2L of a level then runs as: compress the densities (x' = U^T x, FP64
// GEMM), apply the C_d per V pair on the tensor cores (3xTF32, the kernel of
// m2l_tf32x3.cu with ld = the padded rank), expand (y = U y', FP64 GEMM) into
// the check potential. No counterpart in the reference, which applies every
// K_d densely (jaxfmm/kifmm/phases.py:176-237); U and C_d come from the host
// library (hfmm_b200/compress.py: leading eigenvectors of sum_d K_d K_d^T).
// This file packs them into the layouts the GEMMs read and prepares the buffers.
#include "hfmm_internal.cuh"
#include "mixed.cuh"

#include <cstring>

namespace hfmm {

namespace {

constexpr int N_M2L = 316;

// compress table, A^T of U^T: out[k][m] = U[k][m] (k < n_s rows of U, m < r), ld x cw
__global__ void k_pack_cmp(const double* __restrict__ U, int n_s, int r, int ld, int cw,
                           double* out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (m >= cw || k >= ld) return;
    out[(int64_t)k * cw + m] = (k < n_s && m < r) ? U[(int64_t)k * r + m] : 0.0;
}

// expand table, A^T of U: out[k][m] = U[m][k] (k < r, m < n_s), ch x ld
__global__ void k_pack_exp(const double* __restrict__ U, int n_s, int r, int ld, int ch,
                           double* out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (m >= ld || k >= ch) return;
    out[(int64_t)k * ld + m] = (k < r && m < n_s) ? U[(int64_t)m * r + k] : 0.0;
}

__device__ __forceinline__ float tf32_round(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// C_d as TF32 hi/lo halves in the A layout [d][m][k] of the tcgen05 kernel (cmld x ckld)
__global__ void k_pack_c(const double* __restrict__ C, int r, int ckld, int cmld, float* hi,
                         float* lo) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    const int d = blockIdx.z;
    if (k >= ckld || m >= cmld) return;
    const double v = (m < r && k < r) ? C[((int64_t)d * r + m) * r + k] : 0.0;
    const float h = tf32_round((float)v);
    const int64_t o = ((int64_t)d * cmld + m) * ckld + k;
    hi[o] = h;
    lo[o] = tf32_round((float)(v - (double)h));
}

// C = A B for row-major FP64 matrices, batched over blockIdx.z with element strides
// (0: the operand is shared). Setup only: it builds the folded tables.
__global__ void k_matmul(const double* __restrict__ A, int lda, int64_t sa,
                         const double* __restrict__ B, int ldb, int64_t sb, double* C, int ldc,
                         int64_t scs, int M, int N, int K) {
    __shared__ double As[16][17], Bs[16][17];
    const int z = blockIdx.z;
    A += z * sa;
    B += z * sb;
    C += z * scs;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int row = blockIdx.y * 16 + ty, col = blockIdx.x * 16 + tx;
    double acc = 0.0;
    for (int k0 = 0; k0 < K; k0 += 16) {
        As[ty][tx] = (row < M && k0 + tx < K) ? A[(int64_t)row * lda + k0 + tx] : 0.0;
        Bs[ty][tx] = (k0 + ty < K && col < N) ? B[(int64_t)(k0 + ty) * ldb + col] : 0.0;
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) acc = fma(As[ty][kk], Bs[kk][tx], acc);
        __syncthreads();
    }
    if (row < M && col < N) C[(int64_t)row * ldc + col] = acc;
}

void matmul(const double* A, int lda, int64_t sa, const double* B, int ldb, int64_t sb, double* C,
            int ldc, int64_t scs, int M, int N, int K, int batch) {
    const dim3 grid((unsigned)ceil_div(N, 16), (unsigned)ceil_div(M, 16), (unsigned)batch);
    HFMM_LAUNCH(k_matmul, grid, dim3(16, 16), 0, 0, A, lda, sa, B, ldb, sb, C, ldc, scs, M, N, K);
}

// The folded tables of one level and family. Every operator is kept as the row-major
// right multiplier of a box's row vector (the A^T layout the GEMMs read), so
//   y(parent) = d_up .* sum_o y(child_o) [Vt_up(l+1) M2M_o^T U_up(l)]
//   x'        = y Vt_up(l) U_c
//   y_dn      = d_dn .* (y' U_c^T U_dn(l) + y_dn(parent) [Vt_dn(l-1) L2L_o^T U_dn(l)])
// and only leaves leave the coordinates: U_up after P2M, Vt_dn before L2P. The scale d
// is never multiplied into a table: the decodes' rounding then stays along the
// directions their small singular values damp, as in the two-step decode.
void fold_level(hfmm_plan* P, int f, int l, DevBuf<double>& tmp) {
    LevelTables& T = P->tables[f][l];
    const int ld = P->ld;
    const int64_t mat = (int64_t)ld * ld;
    if (l < P->md) {
        const LevelTables& C = P->tables[f][l + 1];
        T.m2m_f.alloc(8 * (size_t)mat);
        matmul(C.up_Vt.p, ld, 0, T.m2m.p, ld, mat, tmp.p, ld, mat, ld, ld, ld, 8);
        matmul(tmp.p, ld, mat, T.up_U.p, ld, 0, T.m2m_f.p, ld, mat, ld, ld, ld, 8);
    } else {
        T.m2m_f.release();
    }
    if (l >= 3) {
        const LevelTables& Pa = P->tables[f][l - 1];
        T.l2l_f.alloc(8 * (size_t)mat);
        matmul(Pa.dn_Vt.p, ld, 0, T.l2l.p, ld, mat, tmp.p, ld, mat, ld, ld, ld, 8);
        matmul(tmp.p, ld, mat, T.dn_U.p, ld, 0, T.l2l_f.p, ld, mat, ld, ld, ld, 8);
    } else {
        T.l2l_f.release();
    }
    T.cmp_f.alloc((size_t)ld * T.ckld);
    matmul(T.up_Vt.p, ld, 0, T.c_cmp.p, T.ckld, 0, T.cmp_f.p, T.ckld, 0, ld, T.ckld, ld, 1);
    T.exp_f.alloc((size_t)T.cmld * ld);
    matmul(T.c_exp.p, ld, 0, T.dn_U.p, ld, 0, T.exp_f.p, ld, 0, T.cmld, ld, ld, 1);
}

}  // namespace

void compressed_prepare(hfmm_plan* P) {
    P->compressed = false;
    if (P->ld < 128) return;
    for (int f = 0; f < P->n_fam; ++f)
        for (int l = 2; l <= P->md; ++l)
            if (!P->tables[f][l].cr) return;
    if (!P->cx_maps) P->cx_maps = new MixedMaps[2 * MAX_LEVELS];
    MixedMaps* maps = static_cast<MixedMaps*>(P->cx_maps);
    std::memset(maps, 0, sizeof(MixedMaps) * 2 * MAX_LEVELS);
    for (int f = 0; f < P->n_fam; ++f)
        for (int l = 2; l <= P->md; ++l) {
            LevelTables& T = P->tables[f][l];
            const size_t rows = (size_t)(P->level_hi[l] - P->level_lo[l]) * 2;   // R <= 2
            T.xc.alloc(rows * T.ckld);
            T.yc.alloc(rows * T.cmld);
            T.xc_hi.alloc(rows * T.ckld);
            T.xc_lo.alloc(rows * T.ckld);
            T.xc.zero();
            T.yc.zero();
            T.xc_hi.zero();
            T.xc_lo.zero();
            make_table_map(&maps[f * MAX_LEVELS + l].a_hi[0], T.c_hi.p, T.ckld, N_M2L, T.cmld);
            make_table_map(&maps[f * MAX_LEVELS + l].a_lo[0], T.c_lo.p, T.ckld, N_M2L, T.cmld);
            // complete level: the complex-charge M2L reads its densities from a dense grid
            T.grid = 0;
            T.xg_hi.release();
            T.xg_lo.release();
            if (P->gx_tiles[l].ntiles > 0) {
                const int G = 1 << l;
                const size_t cells = (size_t)G * G * G * 2 * T.ckld;
                T.xg_hi.alloc(cells);
                T.xg_lo.alloc(cells);
                T.xg_hi.zero();
                T.xg_lo.zero();
                make_grid_map(&maps[f * MAX_LEVELS + l].b_hi[0], T.xg_hi.p, T.ckld, G);
                make_grid_map(&maps[f * MAX_LEVELS + l].b_lo[0], T.xg_lo.p, T.ckld, G);
                T.grid = G;
            }
        }
    {
        DevBuf<double> tmp;
        tmp.alloc(8 * (size_t)P->ld * P->ld);
        for (int f = 0; f < P->n_fam; ++f)
            for (int l = 2; l <= P->md; ++l) fold_level(P, f, l, tmp);
        HFMM_CUDA(cudaDeviceSynchronize());   // tmp is freed on return
    }
    if (!P->cx_fork) {   // side streams and fork/join events of the concurrent M2L
        HFMM_CUDA(cudaEventCreateWithFlags(&P->cx_fork, cudaEventDisableTiming));
        for (int k = 0; k < hfmm_plan::CX_STREAMS; ++k) {
            HFMM_CUDA(cudaStreamCreateWithFlags(&P->cx_side[k], cudaStreamNonBlocking));
            HFMM_CUDA(cudaEventCreateWithFlags(&P->cx_join[k], cudaEventDisableTiming));
        }
        for (int l = 0; l < MAX_LEVELS; ++l)
            for (int f = 0; f < 2; ++f)
                HFMM_CUDA(cudaEventCreateWithFlags(&P->cx_level[l][f], cudaEventDisableTiming));
    }
    P->compressed = true;
}

void compressed_release(hfmm_plan* P) {
    if (P->cx_fork) cudaEventDestroy(P->cx_fork);
    for (int k = 0; k < hfmm_plan::CX_STREAMS; ++k) {
        if (P->cx_side[k]) cudaStreamDestroy(P->cx_side[k]);
        if (P->cx_join[k]) cudaEventDestroy(P->cx_join[k]);
        P->cx_side[k] = nullptr;
        P->cx_join[k] = nullptr;
    }
    P->cx_fork = nullptr;
    for (int l = 0; l < MAX_LEVELS; ++l)
        for (int f = 0; f < 2; ++f) {
            if (P->cx_level[l][f]) cudaEventDestroy(P->cx_level[l][f]);
            P->cx_level[l][f] = nullptr;
        }
}

}  // namespace hfmm

using namespace hfmm;

extern "C" {

int hfmm_plan_set_m2l_compressed(hfmm_plan* P, int32_t family, int32_t level, int32_t rank,
                                 const double* U_dev, const double* C_dev) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    if (P->n_s == 0) return fail(HFMM_ERR_STATE, "set the kernel first");
    if (family < 0 || family >= P->n_fam) return fail(HFMM_ERR_ARG, "family out of range");
    if (level < 2 || level > P->md) return fail(HFMM_ERR_ARG, "level must be in [2, max_depth]");
    if (rank < 1 || rank > P->n_s) return fail(HFMM_ERR_ARG, "rank must be in [1, n_s]");
    if (!U_dev || !C_dev) return fail(HFMM_ERR_ARG, "U and C are required");
    try {
        require_device_ptr(U_dev, "U");
        require_device_ptr(C_dev, "C");
        LevelTables& T = P->tables[family][level];
        const int ckld = std::max(32, (int)round_up(rank, 32));    // K: one 32-wide chunk at least
        const int cmld = std::max(128, (int)round_up(rank, 32));   // M: one 128-row MMA tile at least
        T.cr = rank;
        T.ckld = ckld;
        T.cmld = cmld;
        T.c_cmp.alloc((size_t)P->ld * ckld);
        T.c_exp.alloc((size_t)cmld * P->ld);
        T.c_hi.alloc((size_t)N_M2L * cmld * ckld);
        T.c_lo.alloc((size_t)N_M2L * cmld * ckld);
        HFMM_LAUNCH(k_pack_cmp, dim3((unsigned)ceil_div(ckld, 128), (unsigned)P->ld), 128, 0, 0,
                    U_dev, P->n_s, rank, P->ld, ckld, T.c_cmp.p);
        HFMM_LAUNCH(k_pack_exp, dim3((unsigned)ceil_div(P->ld, 128), (unsigned)cmld), 128, 0, 0,
                    U_dev, P->n_s, rank, P->ld, cmld, T.c_exp.p);
        HFMM_LAUNCH(k_pack_c, dim3((unsigned)ceil_div(ckld, 128), (unsigned)cmld, N_M2L), 128, 0, 0,
                    C_dev, rank, ckld, cmld, T.c_hi.p, T.c_lo.p);
        HFMM_CUDA(cudaDeviceSynchronize());
        P->finalized = false;
        return HFMM_OK;
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    }
}

}  // extern "C"
