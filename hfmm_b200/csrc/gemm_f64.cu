// FP64 output-stationary gather-GEMM for the plain (float64) path.
//
// For a tile of target boxes t_1..t_T (same level; for M2L also the same octant)
// and one M-tile of the n_s surface rows it computes
//     out[t_j][r][m] (+)= scale[m] * sum_e sum_k A_e[m][k] * B_e[src(t_j, e)][r][k]
// with the accumulator kept on chip across every entry e, so no partial sum
// ever goes back to memory and the result is deterministic. One kernel serves
// the four dense contractions of the KIFMM evaluate:
//   M2M  (phases.py:163-171): e = child octant, A_e = M2M_K_lv[parent][e]
//   M2L  (phases.py:211-236): e = displacement (343 slots), A_e = M2L_K_lv[level][e];
//        plus L2L (phases.py:273-278): e = 343 + octant, A_e = L2L_K_lv[level-1][octant],
//        src = parent -- the L2L check potential is summed with the M2L one and
//        decoded once (the decode is linear)
//   decode (phases.py:21-34): A = U^T with scale d, then A = Vt^T.
// A is stored transposed (k-major, leading dimension ld, zero padded) so both
// operand tiles stream into shared memory with 16-byte cp.async copies.
//
// Tensor path: mma.sync.m16n8k4 f64 (DMMA). tcgen05 has no f64 kind, so this
// is the FP64 tensor path on sm_100a. CTA tile 64 (m) x 64 (n = targets x R),
// k-chunk 16, 4 warps of 32 x 32, two-stage cp.async pipeline.
// Small grids (coarse levels: a few dozen output tiles, each walking all its entries)
// are latency-bound, so there the entries are split into contiguous ranges, one CTA
// per range and output tile; each writes its partial tile to a scratch array and
// k_gemm_reduce adds the partials in range order before the usual epilogue, so the
// result does not depend on scheduling.
#include "hfmm_internal.cuh"

#include <algorithm>

namespace hfmm {

namespace {

constexpr int TM = 64, TN = 64, KC = 16;
constexpr int AP = TM + 8;   // As[k][AP]: conflict-free a-fragment loads (AP = 8 mod 16)
constexpr int BP = KC + 4;   // Bs[n][BP]: conflict-free b-fragment loads (BP = 4 mod 16)
constexpr int MAX_ENTRIES = 352;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int sz = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
        "{%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

struct __align__(16) Smem {
    union {
        struct {
            double A[2][KC][AP];
            double B[2][TN][BP];
        } ld;
        double C[TN][TM + 2];   // epilogue staging, column-major by target column
    } u;
    int tgt[TN];
    short act[MAX_ENTRIES];
    unsigned char used[MAX_ENTRIES];   // entry has a source for some target of the tile
    int n_act;
};

template <int R>
__global__ void __launch_bounds__(128, 5) k_gemm_f64(GemmCall c, int* err) {
    constexpr int TT = TN / R;
    __shared__ Smem sm;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int S = c.n_split > 1 ? c.n_split : 1;
    const int tile = blockIdx.x, m0 = blockIdx.y * TM, fam = blockIdx.z / S, split = blockIdx.z % S;
    const int e_lo = (int)((int64_t)split * c.n_entries / S);
    const int e_hi = (int)((int64_t)(split + 1) * c.n_entries / S);
    const double* const* A = c.A + (int64_t)fam * c.a_fam_stride;
    const double* B0 = c.B0 + (int64_t)fam * c.fam_stride;
    const double* B1 = c.B1 ? c.B1 + (int64_t)fam * c.fam_stride : nullptr;
    double* out = c.out + (int64_t)fam * c.fam_stride;

    if (tid < TT) {
        int t = c.tile_tgt[(int64_t)tile * TT + tid];
        if (t >= c.nb) {
            atomicOr(err, ERRF_BOUNDS);
            t = -1;
        }
        sm.tgt[tid] = t;
    }
    if (tid == 0) sm.n_act = 0;
    for (int e = tid; e < c.n_entries; e += 128) sm.used[e] = c.src_tab ? 0 : 1;
    __syncthreads();
    // active entries: A present and at least one target of the tile has a source. Every
    // thread tests (target, entry) pairs, the loads of a batch independent of each other
    if (c.src_tab) {
        constexpr int BATCH = 8;
        const int pairs = TT * c.n_entries;
        for (int i0 = tid; i0 < pairs; i0 += 128 * BATCH) {
            int src[BATCH];
#pragma unroll
            for (int u = 0; u < BATCH; ++u) {
                const int i = i0 + u * 128;
                src[u] = -1;
                if (i < pairs) {
                    const int t = sm.tgt[i / c.n_entries];
                    if (t >= 0) src[u] = __ldg(c.src_tab + (int64_t)t * c.src_ld + i % c.n_entries);
                }
            }
#pragma unroll
            for (int u = 0; u < BATCH; ++u)
                if (src[u] >= 0) sm.used[(i0 + u * 128) % c.n_entries] = 1;
        }
        __syncthreads();
    }
    if (warp == 0) {
        int base = 0;
        for (int e0 = 0; e0 < c.n_entries; e0 += 32) {
            int e = e0 + lane;
            const bool act = e >= e_lo && e < e_hi && A[e] != nullptr && sm.used[e];
            unsigned bal = __ballot_sync(0xffffffffu, act);
            if (act) sm.act[base + __popc(bal & ((1u << lane) - 1))] = (short)e;
            base += __popc(bal);
        }
        if (lane == 0) sm.n_act = base;
    }
    __syncthreads();
    const int n_act = sm.n_act;
    const int kch = c.k_valid > 0 ? (c.k_valid + KC - 1) / KC : c.ldk / KC;
    const int nq = n_act * kch;

    auto load = [&](int q, int buf) {
        const int e = sm.act[q / kch];
        const int k0 = (q % kch) * KC;
        const double* Ae = A[e];
        const double* Bsel = (e >= c.b_split && B1) ? B1 : B0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {   // A: 16 rows x 64 doubles = 512 x 16 B
            int ch = tid + 128 * i;
            int row = ch >> 5, col = (ch & 31) * 2;
            bool ok = (m0 + col) < c.ldm;
            const double* g = ok ? Ae + (int64_t)(k0 + row) * c.ldm + m0 + col : Ae;
            cp_async16(&sm.u.ld.A[buf][row][col], g, ok);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {   // B: 64 columns x 16 doubles = 512 x 16 B
            int ch = tid + 128 * i;
            int col = ch >> 3, part = (ch & 7) * 2;
            int j = col / R, r = col % R;
            int t = sm.tgt[j];
            int s = -1;
            if (t >= 0) s = c.src_tab ? c.src_tab[(int64_t)t * c.src_ld + e] : t;
            bool ok = s >= 0 && s < c.nb;
            if (s >= c.nb) atomicOr(err, ERRF_BOUNDS);
            const double* g = ok ? Bsel + ((int64_t)s * R + r) * c.ldk + k0 + part : B0;
            cp_async16(&sm.u.ld.B[buf][col][part], g, ok);
        }
    };

    double acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int d = 0; d < 4; ++d) acc[a][b][d] = 0.0;

    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
    const int g = lane >> 2, t4 = lane & 3;
    if (nq > 0) {
        load(0, 0);
        cp_async_commit();
    }
    for (int q = 0; q < nq; ++q) {
        const int buf = q & 1;
        if (q + 1 < nq) {
            load(q + 1, buf ^ 1);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KC; kk += 4) {
            double a[2][2], b[4];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi) {
                a[mi][0] = sm.u.ld.A[buf][kk + t4][wm + mi * 16 + g];
                a[mi][1] = sm.u.ld.A[buf][kk + t4][wm + mi * 16 + g + 8];
            }
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) b[ni] = sm.u.ld.B[buf][wn + ni * 8 + g][kk + t4];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) dmma(acc[mi][ni], a[mi][0], a[mi][1], b[ni]);
        }
        __syncthreads();
    }
    // epilogue: stage through shared memory, write columns coalesced along m
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
            int m = wm + mi * 16 + g, n = wn + ni * 8 + 2 * t4;
            sm.u.C[n][m] = acc[mi][ni][0];
            sm.u.C[n + 1][m] = acc[mi][ni][1];
            sm.u.C[n][m + 8] = acc[mi][ni][2];
            sm.u.C[n + 1][m + 8] = acc[mi][ni][3];
        }
    __syncthreads();
    if (S > 1) {   // a split: the partial tile goes to the scratch, k_gemm_reduce finishes it
        double* dst = c.part + ((int64_t)(blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) * TN * TM;
        for (int idx = tid; idx < TN * TM; idx += 128) dst[idx] = sm.u.C[idx / TM][idx % TM];
        return;
    }
    const double* sc = (fam == 1 && c.scale_f1) ? c.scale_f1 : c.scale;
    for (int idx = tid; idx < TN * (TM / 2); idx += 128) {
        int col = idx / (TM / 2), mm = (idx % (TM / 2)) * 2;
        int j = col / R, r = col % R;
        int t = sm.tgt[j];
        int m = m0 + mm;
        if (t < 0 || m >= c.ldm) continue;
        double v0 = sm.u.C[col][mm], v1 = sm.u.C[col][mm + 1];
        if (sc) {
            v0 *= sc[m];
            v1 *= sc[m + 1];
        }
        double2* o = reinterpret_cast<double2*>(out + ((int64_t)t * R + r) * c.ldm + m);
        if (c.accumulate) {
            double2 old = *o;
            v0 += old.x;
            v1 += old.y;
        }
        *o = make_double2(v0, v1);
    }
}

// The split GEMM's epilogue: per output tile, the n_split partial tiles added in
// entry-range order, then the scale, accumulation and store of k_gemm_f64.
template <int R>
__global__ void __launch_bounds__(128) k_gemm_reduce(GemmCall c, int* err) {
    constexpr int TT = TN / R;
    __shared__ int tgt[TT];
    const int tid = threadIdx.x;
    const int tile = blockIdx.x, m0 = blockIdx.y * TM, fam = blockIdx.z, S = c.n_split;
    double* out = c.out + (int64_t)fam * c.fam_stride;
    if (tid < TT) {
        int t = c.tile_tgt[(int64_t)tile * TT + tid];
        if (t >= c.nb) {
            atomicOr(err, ERRF_BOUNDS);
            t = -1;
        }
        tgt[tid] = t;
    }
    __syncthreads();
    const double* sc = (fam == 1 && c.scale_f1) ? c.scale_f1 : c.scale;
    for (int idx = tid; idx < TN * (TM / 2); idx += 128) {
        int col = idx / (TM / 2), mm = (idx % (TM / 2)) * 2;
        int j = col / R, r = col % R;
        int t = tgt[j];
        int m = m0 + mm;
        if (t < 0 || m >= c.ldm) continue;
        double v0 = 0.0, v1 = 0.0;
        for (int sp = 0; sp < S; ++sp) {
            const double* src = c.part +
                ((int64_t)((fam * S + sp) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) * TN * TM;
            v0 += src[col * TM + mm];
            v1 += src[col * TM + mm + 1];
        }
        if (sc) {
            v0 *= sc[m];
            v1 *= sc[m + 1];
        }
        double2* o = reinterpret_cast<double2*>(out + ((int64_t)t * R + r) * c.ldm + m);
        if (c.accumulate) {
            double2 old = *o;
            v0 += old.x;
            v1 += old.y;
        }
        *o = make_double2(v0, v1);
    }
}

}  // namespace

int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0, v = 0;
        HFMM_CUDA(cudaGetDevice(&dev));
        HFMM_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
        n = v > 0 ? v : 148;
    }
    return n;
}

void gemm_f64(const GemmCall& call, int* d_err, cudaStream_t s) {
    if (call.ntiles == 0) return;
    GemmCall c = call;
    if (!c.ldk) c.ldk = c.ld;
    if (!c.ldm) c.ldm = c.ld;
    if (c.ldk % KC != 0 || c.ldm % KC != 0)
        throw Error{HFMM_ERR_STATE, "gemm_f64: ld must be a multiple of 16"};
    if (c.k_valid > c.ldk) throw Error{HFMM_ERR_STATE, "gemm_f64: k_valid beyond ldk"};
    if (c.n_entries > MAX_ENTRIES) throw Error{HFMM_ERR_STATE, "gemm_f64: too many entries"};
    if (c.R != 1 && c.R != 2) throw Error{HFMM_ERR_ARG, "gemm_f64: R must be 1 or 2"};
    dim3 grid(c.ntiles, (c.ldm + TM - 1) / TM, c.n_fam);
    // entry splits when the grid gives the SMs fewer than four CTAs each (a CTA of 128
    // threads hides little latency on its own): up to about four per SM
    const int64_t ctas = (int64_t)grid.x * grid.y * grid.z;
    const int sms = sm_count();
    int S = 1;
    if (c.part && c.n_entries > 1 && ctas < 4 * sms) {
        S = (int)std::min<int64_t>({(int64_t)c.n_entries, 16, (4 * sms + ctas - 1) / ctas});
        while (S > 1 && ctas * S * TN * TM > c.part_cap) --S;
    }
    c.n_split = S;
    grid.z *= S;
    if (c.R == 1) HFMM_LAUNCH(k_gemm_f64<1>, grid, 128, 0, s, c, d_err);
    else HFMM_LAUNCH(k_gemm_f64<2>, grid, 128, 0, s, c, d_err);
    if (S > 1) {
        grid.z /= S;
        if (c.R == 1) HFMM_LAUNCH(k_gemm_reduce<1>, grid, 128, 0, s, c, d_err);
        else HFMM_LAUNCH(k_gemm_reduce<2>, grid, 128, 0, s, c, d_err);
    }
}

}  // namespace hfmm
