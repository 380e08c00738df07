// Rotation-based M2L of the FP64 evaluate: rotate, shift along z, rotate back.
//
// The alternative to the dense M2L tables (the reference's Helmholtz path uses KIFMM
// operators, kifmm/phases.py:176-237; its rotation M2L is Laplace's,
// kernels/laplace/transf.py:143-250). Per level and kernel family:
//   1. k_rot_multipole: multipole coefficients of every box of the level from its
//      equivalent density, M[b][r] = Q x[b][r] (Q: (P+1)^2 x n_s complex);
//   2. k_rot_m2l: one CTA per target box walks its V list; per source it rotates the
//      source's coefficients into the frame whose z axis is the displacement (T_n per
//      degree n, (2n+1)^2 complex), shifts them coaxially by |d| (one real
//      (P+1-|m|)^2 matrix per order m), rotates the result back (T_n^H) and adds it to
//      the target's local coefficients in shared memory; at the end the target's
//      check potential is Re(pref E L) (E: n_s x (P+1)^2 complex), which the L2L GEMM
//      and the decode then use as in the dense path.
// The operators are built on the host in FP64 (hfmm_b200/rotation.py) and uploaded by
// hfmm_plan_set_m2l_rotation / hfmm_plan_set_rotation_level. Every stage is O(P^3)
// per pair. Accumulation order is fixed (V entries in slot order), so results are
// deterministic.
#include "hfmm_internal.cuh"

#include <algorithm>
#include <vector>

namespace hfmm {

namespace {

struct RotCall {
    const double2* T;          // [343][TS] rotation blocks per displacement slot
    const int32_t* dist;       // [343] coaxial matrix index (-1: adjacent slot)
    const double2* Q;          // [NC][n_s]
    const double2* E;          // [n_s][NC]
    const double* C;           // [n_dist][2P+1][P+1][P+1]
    const int32_t* src_tab;    // [nb][351]
    const double* equiv;       // family base of the equivalent densities [nb][R][ld]
    double* check;             // family base of the check potentials [nb][R][ld]
    double2* M;                // work: [hi - lo][R][NC]
    double pref;
    int P, NC, TS, n_s, ld, R;
    int64_t lo, hi, nb;
    int* err;
};

__device__ __forceinline__ int tri_off(int n) { return n * (4 * n * n - 1) / 3; }   // sum (2k+1)^2, k < n

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {   // conj(a) b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

__global__ void __launch_bounds__(256) k_rot_multipole(RotCall c) {
    extern __shared__ double xs[];   // [R][n_s]
    const int64_t b = c.lo + blockIdx.x;
    for (int i = threadIdx.x; i < c.R * c.n_s; i += blockDim.x) {
        const int r = i / c.n_s, s = i % c.n_s;
        xs[i] = c.equiv[(b * c.R + r) * c.ld + s];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < c.R * c.NC; i += blockDim.x) {
        const int r = i / c.NC, q = i % c.NC;
        const double2* qr = c.Q + (int64_t)q * c.n_s;
        const double* x = xs + r * c.n_s;
        double2 acc = make_double2(0.0, 0.0);
        for (int s = 0; s < c.n_s; ++s) {
            const double2 w = qr[s];
            acc.x += w.x * x[s];
            acc.y += w.y * x[s];
        }
        c.M[((int64_t)blockIdx.x * c.R + r) * c.NC + q] = acc;
    }
}

__global__ void __launch_bounds__(256) k_rot_m2l(RotCall c) {
    extern __shared__ double2 sm[];
    double2* A = sm;                    // [R][NC] source coefficients, then the shifted ones
    double2* B = sm + c.R * c.NC;       // [R][NC] rotated
    double2* L = sm + 2 * c.R * c.NC;   // [R][NC] the target's local coefficients
    const int64_t t = c.lo + blockIdx.x;
    const int RN = c.R * c.NC, P = c.P;
    for (int i = threadIdx.x; i < RN; i += blockDim.x) L[i] = make_double2(0.0, 0.0);
    for (int e = 0; e < N_DISP; ++e) {
        const int di = c.dist[e];
        if (di < 0) continue;
        const int s_ = c.src_tab[t * M2L_ENTRIES + e];
        if (s_ < 0) continue;
        if (s_ < c.lo || s_ >= c.hi) {   // sources share the target's level
            if (threadIdx.x == 0) atomicOr(c.err, ERRF_BOUNDS);
            continue;
        }
        __syncthreads();   // the previous entry's last stage has read A
        const double2* Ms = c.M + (int64_t)(s_ - c.lo) * RN;
        for (int i = threadIdx.x; i < RN; i += blockDim.x) A[i] = Ms[i];
        __syncthreads();
        const double2* T = c.T + (int64_t)e * c.TS;
        // rotate: B[(n, m)] = sum_m'' T_n[m][m''] A[(n, m'')]
        for (int i = threadIdx.x; i < RN; i += blockDim.x) {
            const int r = i / c.NC, q = i % c.NC;
            const int n = (int)sqrtf((float)q + 0.5f), m = q - n * n - n;
            const double2* Tn = T + tri_off(n) + (m + n) * (2 * n + 1);
            const double2* a = A + r * c.NC + n * n;
            double2 acc = make_double2(0.0, 0.0);
            for (int j = 0; j <= 2 * n; ++j) {
                const double2 p = cmul(Tn[j], a[j]);
                acc.x += p.x;
                acc.y += p.y;
            }
            B[i] = acc;
        }
        __syncthreads();
        // shift along z: A[(n', m)] = sum_{n >= |m|} C[m][n'][n] B[(n, m)]
        const double* Cd = c.C + (int64_t)di * (2 * P + 1) * (P + 1) * (P + 1);
        for (int i = threadIdx.x; i < RN; i += blockDim.x) {
            const int r = i / c.NC, q = i % c.NC;
            const int n2 = (int)sqrtf((float)q + 0.5f), m = q - n2 * n2 - n2;
            const int am = m < 0 ? -m : m;
            const double* Cm = Cd + ((int64_t)(m + P) * (P + 1) + n2) * (P + 1);
            const double2* b = B + r * c.NC;
            double2 acc = make_double2(0.0, 0.0);
            for (int n = am; n <= P; ++n) {
                const double w = Cm[n];
                const double2 v = b[n * n + n + m];
                acc.x += w * v.x;
                acc.y += w * v.y;
            }
            A[i] = acc;
        }
        __syncthreads();
        // rotate back and accumulate: L[(n, m'')] += sum_m conj(T_n[m][m'']) A[(n, m)]
        for (int i = threadIdx.x; i < RN; i += blockDim.x) {
            const int r = i / c.NC, q = i % c.NC;
            const int n = (int)sqrtf((float)q + 0.5f), mm = q - n * n - n;
            const double2* Tn = T + tri_off(n) + (mm + n);
            const double2* a = A + r * c.NC + n * n;
            double2 acc = L[i];
            for (int j = 0; j <= 2 * n; ++j) {
                const double2 p = cmulc(Tn[j * (2 * n + 1)], a[j]);
                acc.x += p.x;
                acc.y += p.y;
            }
            L[i] = acc;
        }
    }
    __syncthreads();
    // the check potential at the target's check points: Re(pref E L), padding zeroed
    for (int i = threadIdx.x; i < c.R * c.ld; i += blockDim.x) {
        const int r = i / c.ld, j = i % c.ld;
        double v = 0.0;
        if (j < c.n_s) {
            const double2* Ej = c.E + (int64_t)j * c.NC;
            const double2* l = L + r * c.NC;
            for (int q = 0; q < c.NC; ++q) v += Ej[q].x * l[q].x - Ej[q].y * l[q].y;
            v *= c.pref;
        }
        c.check[(t * c.R + r) * c.ld + j] = v;
    }
}

}  // namespace

size_t rot_workspace_doubles(const hfmm_plan* P) {
    int64_t widest = 0;
    for (int l = 2; l <= P->md; ++l) widest = std::max<int64_t>(widest, P->level_hi[l] - P->level_lo[l]);
    return (size_t)widest * 2 * (P->rot_P + 1) * (P->rot_P + 1) * 2;
}

void rot_m2l(hfmm_plan* P, int l, int R, int64_t fam_stride, cudaStream_t s) {
    const int Pn = P->rot_P, NC = (Pn + 1) * (Pn + 1);
    if (P->rot_M.n < rot_workspace_doubles(P))   // a rebuilt tree with a wider level
        throw Error{HFMM_ERR_STATE, "rotation M2L: set the rotation again after the plan was rebuilt"};
    for (int f = 0; f < P->n_fam; ++f) {
        LevelTables& T = P->tables[f][l];
        if (!T.rot_Q.p) throw Error{HFMM_ERR_STATE, "rotation M2L: level operators missing"};
        RotCall c{};
        c.T = reinterpret_cast<const double2*>(P->rot_T.p);
        c.dist = P->rot_dist.p;
        c.Q = reinterpret_cast<const double2*>(T.rot_Q.p);
        c.E = reinterpret_cast<const double2*>(T.rot_E.p);
        c.C = T.rot_C.p;
        c.src_tab = P->m2l_src.p;
        c.equiv = P->equiv.p + f * fam_stride;
        c.check = P->check.p + f * fam_stride;
        c.M = reinterpret_cast<double2*>(P->rot_M.p);
        c.pref = T.rot_pref;
        c.P = Pn;
        c.NC = NC;
        c.TS = Pn >= 0 ? (Pn + 1) * (4 * (Pn + 1) * (Pn + 1) - 1) / 3 : 0;
        c.n_s = P->n_s;
        c.ld = P->ld;
        c.R = R;
        c.lo = P->level_lo[l];
        c.hi = P->level_hi[l];
        c.nb = P->nb;
        c.err = P->d_err.p;
        const unsigned nbl = (unsigned)(c.hi - c.lo);
        if (nbl == 0) continue;
        HFMM_LAUNCH(k_rot_multipole, nbl, 256, (size_t)R * P->n_s * sizeof(double), s, c);
        const size_t smem = (size_t)3 * R * NC * sizeof(double2);
        HFMM_CUDA(cudaFuncSetAttribute(k_rot_m2l, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        HFMM_LAUNCH(k_rot_m2l, nbl, 256, smem, s, c);
    }
}

}  // namespace hfmm

using namespace hfmm;

extern "C" {

int hfmm_plan_set_m2l_rotation(hfmm_plan* P, int32_t order, const double* T_host,
                               const int32_t* dist_host, int32_t n_dist) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    if (order == 0) {   // back to the dense M2L tables
        P->rot_P = 0;
        return HFMM_OK;
    }
    if (order < 1 || order > 40) return fail(HFMM_ERR_ARG, "rotation order must be in [1, 40]");
    if (!T_host || !dist_host || n_dist < 1) return fail(HFMM_ERR_ARG, "rotations and distances are required");
    try {
        const size_t TS = (size_t)(order + 1) * (4 * (order + 1) * (order + 1) - 1) / 3;
        std::vector<int32_t> d(dist_host, dist_host + N_DISP);
        for (int e = 0; e < N_DISP; ++e)
            if (d[e] >= n_dist) return fail(HFMM_ERR_ARG, "distance index out of range");
        P->rot_T.alloc(N_DISP * TS * 2);
        HFMM_CUDA(cudaMemcpy(P->rot_T.p, T_host, N_DISP * TS * 2 * sizeof(double), cudaMemcpyHostToDevice));
        P->rot_dist.alloc(N_DISP);
        HFMM_CUDA(cudaMemcpy(P->rot_dist.p, d.data(), N_DISP * sizeof(int32_t), cudaMemcpyHostToDevice));
        P->rot_P = order;
        P->rot_n_dist = n_dist;
        for (int f = 0; f < 2; ++f)
            for (int l = 0; l < MAX_LEVELS; ++l) {
                P->tables[f][l].rot_Q.release();
                P->tables[f][l].rot_E.release();
                P->tables[f][l].rot_C.release();
            }
        P->rot_M.alloc(rot_workspace_doubles(P));
        return HFMM_OK;
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    }
}

int hfmm_plan_set_rotation_level(hfmm_plan* P, int32_t family, int32_t level, const double* Q_host,
                                 const double* E_host, const double* C_host, double pref) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    if (P->rot_P < 1) return fail(HFMM_ERR_STATE, "set the rotation order first");
    if (family < 0 || family >= P->n_fam) return fail(HFMM_ERR_ARG, "family out of range");
    if (level < 2 || level > P->md) return fail(HFMM_ERR_ARG, "level must be in [2, max_depth]");
    if (!Q_host || !E_host || !C_host) return fail(HFMM_ERR_ARG, "Q, E and C are required");
    try {
        const size_t NC = (size_t)(P->rot_P + 1) * (P->rot_P + 1);
        const size_t nc = (size_t)P->rot_n_dist * (2 * P->rot_P + 1) * (P->rot_P + 1) * (P->rot_P + 1);
        LevelTables& T = P->tables[family][level];
        T.rot_Q.alloc(NC * P->n_s * 2);
        T.rot_E.alloc(NC * P->n_s * 2);
        T.rot_C.alloc(nc);
        HFMM_CUDA(cudaMemcpy(T.rot_Q.p, Q_host, NC * P->n_s * 2 * sizeof(double), cudaMemcpyHostToDevice));
        HFMM_CUDA(cudaMemcpy(T.rot_E.p, E_host, NC * P->n_s * 2 * sizeof(double), cudaMemcpyHostToDevice));
        HFMM_CUDA(cudaMemcpy(T.rot_C.p, C_host, nc * sizeof(double), cudaMemcpyHostToDevice));
        T.rot_pref = pref;
        return HFMM_OK;
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    }
}

}  // extern "C"
