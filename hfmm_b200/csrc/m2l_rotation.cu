// Rotation-based M2L of the FP64 evaluate: rotate, shift along z, rotate back.
//
// The alternative to the dense M2L tables (the reference's Helmholtz path uses KIFMM
// operators, kifmm/phases.py:176-237; its rotation M2L is Laplace's,
// kernels/laplace/transf.py:143-250). Per level and kernel family:
//   1. k_rot_multipole: multipole coefficients of every box of the level from its
//      equivalent density, M[b][r] = Q x[b][r] (Q: (P+1)^2 x n_s complex), a tile of
//      boxes per CTA so that each row of Q is read once per tile;
//   2. k_rot_m2l: a CTA owns a tile of target boxes (TT targets x R charge columns,
//      at most 16 columns) and walks the 343 displacement slots in order. Per slot it
//      gathers the tile's sources' coefficients (zero where a target has no source
//      there), rotates them into the frame whose z axis is the displacement (T_n per
//      degree n, (2n+1)^2 complex), shifts them coaxially by |d| (one real
//      (P+1-|m|)^2 matrix per order m) and rotates the result back (T_n^H) into the
//      targets' local coefficients, which stay in registers. A thread owns whole
//      coefficient rows across the tile's columns, so each table value it loads feeds
//      every column; the slot's tables are read once per tile instead of once per pair. At the end the targets' check
//      potentials are Re(pref E L) (E: n_s x (P+1)^2 complex), which the L2L GEMM and
//      the decode then use as in the dense path.
// The operators are built on the host in FP64 (hfmm_b200/rotation.py) and uploaded by
// hfmm_plan_set_m2l_rotation / hfmm_plan_set_rotation_level (the y-rotation blocks
// also transposed, Q, E and the coaxial matrices transposed on upload, for reads
// coalesced over the thread index). A slot's rotation R_y(-theta) R_z(-phi) factors
// as T_n = D_n(theta) diag(e^{i m phi}) with D_n real: the gather applies the phases,
// the two rotation stages multiply by real blocks shared by the slots of one polar
// angle, and the rotation back applies the conjugate phases per row. Every stage is O(P^3) per
// pair. Each target sums its slots in slot order, so results are deterministic.
#include "hfmm_internal.cuh"

#include <algorithm>
#include <vector>

namespace hfmm {

namespace {

constexpr int ROT_THREADS = 256;  // two CTAs per SM: one's barrier waits overlap the other's work
constexpr int ROT_MAXI = 14;     // local coefficients a thread holds: rows x columns
constexpr int ROT_MAXROWS = 7;   // (P+1)^2 <= 7 x 256 covers P <= 40
constexpr int ROT_MAXCOL = 16;   // charge columns (targets x R) per CTA
constexpr int ROT_MP_THREADS = 256;

struct RotCall {
    const double* D;           // [n_theta][TS] real y-rotation blocks D_n[m][m''] per polar angle
    const double* Dt;          // [n_theta][TS] the same blocks transposed, D_n^T
    const int32_t* theta;      // [343] polar angle index of each slot (-1: adjacent slot)
    const double2* phase;      // [343][2P+1] e^{i m phi} of each slot: T_n = D_n diag(phase)
    const int32_t* dist;       // [343] coaxial matrix index (-1: adjacent slot)
    const double2* QT;         // [n_s][NC]
    const double2* ET;         // [NC][n_s]
    const double* C;           // [n_dist][2P+1][P+1][P+1], C[d][m][n][n'] (source n, local n')
    const int32_t* src_tab;    // [nb][351]
    const double* equiv;       // family base of the equivalent densities [nb][R][ld]
    double* check;             // family base of the check potentials [nb][R][ld]
    double2* M;                // work: [hi - lo][R][NC]
    double pref;
    int P, NC, TS, n_s, ld, R, TT;
    int64_t lo, hi;
    int* err;
};

__device__ __forceinline__ int tri_off(int n) { return n * (4 * n * n - 1) / 3; }   // sum (2k+1)^2, k < n
__device__ __forceinline__ int deg_of(int q) { return (int)sqrtf((float)q + 0.5f); }  // q = n^2 + n + m

__device__ __forceinline__ void cmac(double2& acc, double2 a, double2 b) {   // acc += a b
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}
__device__ __forceinline__ void cmacc(double2& acc, double2 a, double2 b) {  // acc += conj(a) b
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
}

// M[b][r][q] = sum_s Q[q][s] x[b][r][s] for a tile of TT boxes (TT R <= ROT_MAXCOL).
__global__ void __launch_bounds__(ROT_MP_THREADS) k_rot_multipole(RotCall c) {
    extern __shared__ double xs[];   // [TT R][n_s]
    const int64_t b0 = c.lo + (int64_t)blockIdx.x * c.TT;
    const int nt = (int)min((int64_t)c.TT, c.hi - b0);
    const int ncol = nt * c.R;
    for (int i = threadIdx.x; i < ncol * c.n_s; i += blockDim.x) {
        const int cc = i / c.n_s, s = i - cc * c.n_s;
        xs[i] = c.equiv[(b0 * c.R + cc) * c.ld + s];   // column cc = tt R + r of box b0 + tt
    }
    __syncthreads();
    for (int q = threadIdx.x; q < c.NC; q += blockDim.x) {
        double2 acc[ROT_MAXCOL];
#pragma unroll
        for (int cc = 0; cc < ROT_MAXCOL; ++cc) acc[cc] = make_double2(0.0, 0.0);
        for (int s = 0; s < c.n_s; ++s) {
            const double2 w = __ldg(c.QT + (int64_t)s * c.NC + q);
#pragma unroll
            for (int cc = 0; cc < ROT_MAXCOL; ++cc)
                if (cc < ncol) {
                    const double x = xs[cc * c.n_s + s];
                    acc[cc].x = fma(w.x, x, acc[cc].x);
                    acc[cc].y = fma(w.y, x, acc[cc].y);
                }
        }
#pragma unroll
        for (int cc = 0; cc < ROT_MAXCOL; ++cc)
            if (cc < ncol) c.M[((b0 - c.lo) * c.R + cc) * c.NC + q] = acc[cc];
    }
}

// One thread per coefficient row (n, m) and every charge column of the tile: each
// table value a thread loads feeds all of the tile's columns. ROWS = rows per thread
// ((P+1)^2 <= ROWS x ROT_THREADS), NCM = the columns the registers hold for them.
template <int ROWS>
__global__ void __launch_bounds__(ROT_THREADS, 2) k_rot_m2l(RotCall c) {
    constexpr int NCM = (ROT_MAXI / ROWS) < 12 ? ROT_MAXI / ROWS : 12;
    extern __shared__ double2 sm[];
    __shared__ int32_t src[ROT_MAXCOL];
    const int NC = c.NC, NCOL = c.TT * c.R, NI = NC * NCOL, P = c.P;
    double2* X = sm;        // [NC][NCOL] gathered source coefficients, then the shifted ones
    double2* Y = sm + NI;   // [NC][NCOL] rotated
    int16_t* mq = reinterpret_cast<int16_t*>(sm + 2 * NI);   // [NC] rows in m-major order
    for (int i = threadIdx.x; i < NC; i += ROT_THREADS) {    // i -> (m, n), m = -P..P, n = |m|..P
        int m = -P, base = 0;
        while (base + P + 1 - (m < 0 ? -m : m) <= i) {
            base += P + 1 - (m < 0 ? -m : m);
            ++m;
        }
        const int n = (m < 0 ? -m : m) + (i - base);
        mq[i] = (int16_t)(n * n + n + m);
    }
    const int64_t t0 = c.lo + (int64_t)blockIdx.x * c.TT;
    const int nt = (int)min((int64_t)c.TT, c.hi - t0);
    double2 L[ROWS][NCM];   // local coefficients of rows threadIdx.x + k ROT_THREADS
#pragma unroll
    for (int k = 0; k < ROWS; ++k)
#pragma unroll
        for (int cc = 0; cc < NCM; ++cc) L[k][cc] = make_double2(0.0, 0.0);
    for (int e = 0; e < N_DISP; ++e) {
        const int di = c.dist[e];
        if (di < 0) continue;   // adjacent slot: no V pair
        __syncthreads();        // the previous slot's last stage has read X and src (and mq is built)
        if (threadIdx.x < c.TT) {
            int sb = -1;
            if (threadIdx.x < nt) {
                sb = c.src_tab[(t0 + threadIdx.x) * M2L_ENTRIES + e];
                if (sb >= 0 && (sb < c.lo || sb >= c.hi)) {   // sources share the target's level
                    atomicOr(c.err, ERRF_BOUNDS);
                    sb = -1;
                }
            }
            src[threadIdx.x] = sb < 0 ? -1 : (int)(sb - c.lo);
        }
        __syncthreads();
        bool any = false;
        for (int tt = 0; tt < nt; ++tt) any |= src[tt] >= 0;
        if (!any) continue;     // the same answer for every thread of the CTA
        const double2* __restrict__ ph = c.phase + (int64_t)e * (2 * P + 1) + P;   // ph[m]
        for (int i = threadIdx.x; i < NI; i += ROT_THREADS) {   // coalesced over q
            const int cc = i / NC, q = i - cc * NC;
            const int tt = cc / c.R, r = cc - tt * c.R;
            const int sb = src[tt];
            double2 v = make_double2(0.0, 0.0);
            if (sb >= 0) {   // the z-rotation: coefficient (n, m) times e^{i m phi}
                const int n = deg_of(q);
                cmac(v, c.M[((int64_t)sb * c.R + r) * NC + q], __ldg(ph + (q - n * n - n)));
            }
            X[q * NCOL + cc] = v;
        }
        __syncthreads();
        const int64_t toff = (int64_t)c.theta[e] * c.TS;
        // rotate about y: Y[(n, m)] = sum_j D_n[m][j] X[(n, j - n)], D_n^T read along m
#pragma unroll
        for (int k = 0; k < ROWS; ++k) {
            const int q = threadIdx.x + k * ROT_THREADS;
            if (q < NC) {
                const int n = deg_of(q), m = q - n * n - n, w = 2 * n + 1;
                const double* __restrict__ Dt = c.Dt + toff + tri_off(n) + (m + n);
                const double2* x = X + n * n * NCOL;
                double2 acc[NCM];
#pragma unroll
                for (int cc = 0; cc < NCM; ++cc) acc[cc] = make_double2(0.0, 0.0);
                for (int j = 0; j < w; ++j) {
                    const double t = __ldg(Dt + j * w);
                    const double2* xj = x + j * NCOL;
#pragma unroll
                    for (int cc = 0; cc < NCM; ++cc)
                        if (cc < NCOL) {
                            acc[cc].x = fma(t, xj[cc].x, acc[cc].x);
                            acc[cc].y = fma(t, xj[cc].y, acc[cc].y);
                        }
                }
#pragma unroll
                for (int cc = 0; cc < NCM; ++cc)
                    if (cc < NCOL) Y[q * NCOL + cc] = acc[cc];
            }
        }
        __syncthreads();
        // shift along z: X[(n', m)] = sum_{n >= |m|} C[m][n'][n] Y[(n, m)], rows in m-major
        // order so that a warp reads the same Y rows; C stored as [m][n][n'] (coalesced)
        const double* __restrict__ Cd = c.C + (int64_t)di * (2 * P + 1) * (P + 1) * (P + 1);
#pragma unroll
        for (int k = 0; k < ROWS; ++k) {
            const int i = threadIdx.x + k * ROT_THREADS;
            if (i < NC) {
                const int q = mq[i];
                const int n2 = deg_of(q), m = q - n2 * n2 - n2;
                const int am = m < 0 ? -m : m;
                const double* Cm = Cd + (int64_t)(m + P) * (P + 1) * (P + 1) + n2;
                double2 acc[NCM];
#pragma unroll
                for (int cc = 0; cc < NCM; ++cc) acc[cc] = make_double2(0.0, 0.0);
                for (int n = am; n <= P; ++n) {
                    const double w = __ldg(Cm + n * (P + 1));
                    const double2* y = Y + (n * n + n + m) * NCOL;
#pragma unroll
                    for (int cc = 0; cc < NCM; ++cc)
                        if (cc < NCOL) {
                            const double2 v = y[cc];
                            acc[cc].x = fma(w, v.x, acc[cc].x);
                            acc[cc].y = fma(w, v.y, acc[cc].y);
                        }
                }
#pragma unroll
                for (int cc = 0; cc < NCM; ++cc)
                    if (cc < NCOL) X[q * NCOL + cc] = acc[cc];
            }
        }
        __syncthreads();
        // rotate back and accumulate: L[(n, m)] += conj(ph[m]) sum_j D_n[j][m] X[(n, j - n)]
#pragma unroll
        for (int k = 0; k < ROWS; ++k) {
            const int q = threadIdx.x + k * ROT_THREADS;
            if (q < NC) {
                const int n = deg_of(q), m = q - n * n - n, w = 2 * n + 1;
                const double* __restrict__ Dn = c.D + toff + tri_off(n) + (m + n);
                const double2* x = X + n * n * NCOL;
                double2 acc[NCM];
#pragma unroll
                for (int cc = 0; cc < NCM; ++cc) acc[cc] = make_double2(0.0, 0.0);
                for (int j = 0; j < w; ++j) {
                    const double t = __ldg(Dn + j * w);
                    const double2* xj = x + j * NCOL;
#pragma unroll
                    for (int cc = 0; cc < NCM; ++cc)
                        if (cc < NCOL) {
                            acc[cc].x = fma(t, xj[cc].x, acc[cc].x);
                            acc[cc].y = fma(t, xj[cc].y, acc[cc].y);
                        }
                }
                const double2 z = __ldg(ph + m);
#pragma unroll
                for (int cc = 0; cc < NCM; ++cc)
                    if (cc < NCOL) cmacc(L[k][cc], z, acc[cc]);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < ROWS; ++k) {
        const int q = threadIdx.x + k * ROT_THREADS;
        if (q < NC)
#pragma unroll
            for (int cc = 0; cc < NCM; ++cc)
                if (cc < NCOL) X[q * NCOL + cc] = L[k][cc];
    }
    __syncthreads();
    // the check potentials at the targets' check points: Re(pref E L), padding zeroed
    const int ncol = nt * c.R;
    for (int j = threadIdx.x; j < c.ld; j += ROT_THREADS) {
        double acc[ROT_MAXCOL];
#pragma unroll
        for (int cc = 0; cc < ROT_MAXCOL; ++cc) acc[cc] = 0.0;
        if (j < c.n_s)
            for (int q = 0; q < NC; ++q) {
                const double2 w = __ldg(c.ET + (int64_t)q * c.n_s + j);
                const double2* l = X + q * NCOL;
#pragma unroll
                for (int cc = 0; cc < ROT_MAXCOL; ++cc)
                    if (cc < ncol) {
                        acc[cc] = fma(w.x, l[cc].x, acc[cc]);
                        acc[cc] = fma(-w.y, l[cc].y, acc[cc]);
                    }
            }
#pragma unroll
        for (int cc = 0; cc < ROT_MAXCOL; ++cc)
            if (cc < ncol) c.check[(t0 * c.R + cc) * c.ld + j] = c.pref * acc[cc];
    }
}

}  // namespace

size_t rot_workspace_doubles(const hfmm_plan* P) {
    int64_t widest = 0;
    for (int l = 2; l <= P->md; ++l) widest = std::max<int64_t>(widest, P->level_hi[l] - P->level_lo[l]);
    return (size_t)widest * 2 * (P->rot_P + 1) * (P->rot_P + 1) * 2;
}

void rot_check(const hfmm_plan* P) {
    if (P->rot_M.n < rot_workspace_doubles(P))   // a rebuilt tree with a wider level
        throw Error{HFMM_ERR_STATE, "rotation M2L: set the rotation again after the plan was rebuilt"};
    for (int f = 0; f < P->n_fam; ++f)
        for (int l = 2; l <= P->md; ++l)
            if (!P->tables[f][l].rot_Q.p) throw Error{HFMM_ERR_STATE, "rotation M2L: level operators missing"};
}

void rot_m2l(hfmm_plan* P, int l, int R, int64_t fam_stride, cudaStream_t s) {
    const int Pn = P->rot_P, NC = (Pn + 1) * (Pn + 1);
    rot_check(P);
    // rows per thread, then targets per CTA: the columns a thread's registers hold
    const int rows = (int)ceil_div(NC, ROT_THREADS);
    const int TT = rows <= ROT_MAXROWS ? std::min(std::min(ROT_MAXCOL, 12), ROT_MAXI / rows) / R : 0;
    if (TT < 1) throw Error{HFMM_ERR_ARG, "rotation M2L: order too high for one CTA"};
    for (int f = 0; f < P->n_fam; ++f) {
        LevelTables& T = P->tables[f][l];
        if (!T.rot_Q.p) throw Error{HFMM_ERR_STATE, "rotation M2L: level operators missing"};
        RotCall c{};
        c.D = P->rot_D.p;
        c.Dt = c.D + (int64_t)P->rot_n_theta * ((Pn + 1) * (4 * (Pn + 1) * (Pn + 1) - 1) / 3);
        c.theta = P->rot_theta.p;
        c.phase = reinterpret_cast<const double2*>(P->rot_phase.p);
        c.dist = P->rot_dist.p;
        c.QT = reinterpret_cast<const double2*>(T.rot_Q.p);
        c.ET = reinterpret_cast<const double2*>(T.rot_E.p);
        c.C = T.rot_C.p;
        c.src_tab = P->m2l_src.p;
        c.equiv = P->equiv.p + f * fam_stride;
        c.check = P->check.p + f * fam_stride;
        c.M = reinterpret_cast<double2*>(P->rot_M.p);
        c.pref = T.rot_pref;
        c.P = Pn;
        c.NC = NC;
        c.TS = (Pn + 1) * (4 * (Pn + 1) * (Pn + 1) - 1) / 3;
        c.n_s = P->n_s;
        c.ld = P->ld;
        c.R = R;
        c.lo = P->level_lo[l];
        c.hi = P->level_hi[l];
        c.err = P->d_err.p;
        const int64_t nbl = c.hi - c.lo;
        if (nbl == 0) continue;
        c.TT = ROT_MAXCOL / R;
        const size_t smem_mp = (size_t)c.TT * R * P->n_s * sizeof(double);
        HFMM_CUDA(cudaFuncSetAttribute(k_rot_multipole, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem_mp));
        HFMM_LAUNCH(k_rot_multipole, (unsigned)ceil_div(nbl, (int64_t)c.TT), ROT_MP_THREADS, smem_mp, s, c);
        c.TT = TT;
        // X and Y, then the m-major row table (int16) rounded up to 16 bytes
        const size_t smem = (size_t)2 * NC * TT * R * sizeof(double2) + (size_t)ceil_div(NC * 2, 16) * 16;
        const unsigned grid = (unsigned)ceil_div(nbl, (int64_t)TT);
        auto launch = [&](auto kern) {
            HFMM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            HFMM_LAUNCH(kern, grid, ROT_THREADS, smem, s, c);
        };
        switch (rows) {
            case 1: launch(k_rot_m2l<1>); break;
            case 2: launch(k_rot_m2l<2>); break;
            case 3: launch(k_rot_m2l<3>); break;
            case 4: launch(k_rot_m2l<4>); break;
            case 5: launch(k_rot_m2l<5>); break;
            case 6: launch(k_rot_m2l<6>); break;
            default: launch(k_rot_m2l<7>); break;
        }
    }
}

}  // namespace hfmm

using namespace hfmm;

extern "C" {

int hfmm_plan_set_m2l_rotation(hfmm_plan* P, int32_t order, const double* D_host, int32_t n_theta,
                               const int32_t* theta_host, const double* phase_host,
                               const int32_t* dist_host, int32_t n_dist) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    if (order == 0) {   // back to the dense M2L tables
        P->rot_P = 0;
        return HFMM_OK;
    }
    if (order < 1 || order > 40) return fail(HFMM_ERR_ARG, "rotation order must be in [1, 40]");
    if (!D_host || n_theta < 1 || !theta_host || !phase_host || !dist_host || n_dist < 1)
        return fail(HFMM_ERR_ARG, "rotations, phases and distances are required");
    try {
        const size_t TS = (size_t)(order + 1) * (4 * (order + 1) * (order + 1) - 1) / 3;
        const size_t NZ = 2 * (size_t)order + 1;
        std::vector<int32_t> d(dist_host, dist_host + N_DISP), th(theta_host, theta_host + N_DISP);
        for (int e = 0; e < N_DISP; ++e) {
            if (d[e] >= n_dist) return fail(HFMM_ERR_ARG, "distance index out of range");
            if (d[e] >= 0 && (th[e] < 0 || th[e] >= n_theta))   // every V slot needs its rotation
                return fail(HFMM_ERR_ARG, "polar angle index out of range");
        }
        // the blocks as given, then each block transposed (D_n^T)
        std::vector<double> dt((size_t)n_theta * TS);
        for (size_t a = 0; a < (size_t)n_theta; ++a)
            for (int n = 0, off = 0; n <= order; off += (2 * n + 1) * (2 * n + 1), ++n) {
                const size_t w = 2 * n + 1, b = a * TS + off;
                for (size_t i = 0; i < w; ++i)
                    for (size_t j = 0; j < w; ++j) dt[b + j * w + i] = D_host[b + i * w + j];
            }
        P->rot_D.alloc(2 * (size_t)n_theta * TS);
        HFMM_CUDA(cudaMemcpy(P->rot_D.p, D_host, (size_t)n_theta * TS * sizeof(double), cudaMemcpyHostToDevice));
        HFMM_CUDA(cudaMemcpy(P->rot_D.p + (size_t)n_theta * TS, dt.data(), (size_t)n_theta * TS * sizeof(double),
                             cudaMemcpyHostToDevice));
        P->rot_theta.alloc(N_DISP);
        HFMM_CUDA(cudaMemcpy(P->rot_theta.p, th.data(), N_DISP * sizeof(int32_t), cudaMemcpyHostToDevice));
        P->rot_phase.alloc(N_DISP * NZ * 2);
        HFMM_CUDA(cudaMemcpy(P->rot_phase.p, phase_host, N_DISP * NZ * 2 * sizeof(double), cudaMemcpyHostToDevice));
        P->rot_n_theta = n_theta;
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
        const size_t ns = (size_t)P->n_s;
        // stored transposed: Q^T [n_s][NC] and E^T [NC][n_s] (complex as re, im pairs)
        std::vector<double> qt(NC * ns * 2), et(NC * ns * 2);
        for (size_t q = 0; q < NC; ++q)
            for (size_t j = 0; j < ns; ++j)
                for (int z = 0; z < 2; ++z) {
                    qt[(j * NC + q) * 2 + z] = Q_host[(q * ns + j) * 2 + z];
                    et[(q * ns + j) * 2 + z] = E_host[(j * NC + q) * 2 + z];
                }
        T.rot_Q.alloc(NC * ns * 2);
        T.rot_E.alloc(NC * ns * 2);
        // C[d][m][n'][n] stored as [d][m][n][n'] (the shift reads it along n')
        const size_t p1 = (size_t)P->rot_P + 1;
        std::vector<double> ct(nc);
        for (size_t dm = 0; dm < nc / (p1 * p1); ++dm)
            for (size_t a = 0; a < p1; ++a)
                for (size_t b = 0; b < p1; ++b) ct[(dm * p1 + b) * p1 + a] = C_host[(dm * p1 + a) * p1 + b];
        T.rot_C.alloc(nc);
        HFMM_CUDA(cudaMemcpy(T.rot_Q.p, qt.data(), NC * ns * 2 * sizeof(double), cudaMemcpyHostToDevice));
        HFMM_CUDA(cudaMemcpy(T.rot_E.p, et.data(), NC * ns * 2 * sizeof(double), cudaMemcpyHostToDevice));
        HFMM_CUDA(cudaMemcpy(T.rot_C.p, ct.data(), nc * sizeof(double), cudaMemcpyHostToDevice));
        T.rot_pref = pref;
        return HFMM_OK;
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    }
}

}  // extern "C"
