// Device generation of the per-level kernel matrices: M2L (316 non-adjacent
// displacements), M2M (8 octants, parent level, child scale) and L2L (8 octants,
// child level) -- the kernel-evaluation part of build_operators /
// build_operators_leveled (kifmm/operators.py:363-403, 616-640), which the host
// otherwise assembles in NumPy. Only the two damped-SVD decodes per level stay on
// the host (they need an SVD).
//
// Entry (m, k) of each matrix is G(x_m s, y_k s) = trig(k r) / r, r = |x_m s - y_k s|,
// with the same point sets as the reference:
//   M2L: x = equiv + 2 d,  y = equiv        (scale of the level)
//   M2M: x = 2 check,      y = equiv + o_c  (scale of the CHILD level)
//   L2L: x = equiv + o_c,  y = 2 check      (scale of the level)
// The ULP-relative zero of HFMM.py:20-23 never triggers for these point sets
// (their minimum separation is >= 1.9 s), so it is not evaluated. The result is
// written straight into the GEMM layout (A^T, k-major, ld x ld, zero padded).
#include "hfmm_internal.cuh"

namespace hfmm {

namespace {

// The 316 non-adjacent displacements (dx, dy, dz) in [-3, 3]^3, max |d| >= 2, in
// (dx+3)*49 + (dy+3)*7 + (dz+3) order: the M2L table order.
struct DispTable {
    signed char d[316][3];
    constexpr DispTable() : d{} {
        int c = 0;
        for (int i = 0; i < N_DISP; ++i) {
            const int ix = i / 49 - 3, iy = (i / 7) % 7 - 3, iz = i % 7 - 3;
            const int ax = ix < 0 ? -ix : ix, ay = iy < 0 ? -iy : iy, az = iz < 0 ? -iz : iz;
            const int mx = ax > ay ? (ax > az ? ax : az) : (ay > az ? ay : az);
            if (mx > 1) {
                d[c][0] = (signed char)ix;
                d[c][1] = (signed char)iy;
                d[c][2] = (signed char)iz;
                ++c;
            }
        }
    }
};
__constant__ DispTable c_disp = DispTable();

__device__ __forceinline__ void disp_of(int c, double& dx, double& dy, double& dz) {
    dx = 2.0 * c_disp.d[c][0];
    dy = 2.0 * c_disp.d[c][1];
    dz = 2.0 * c_disp.d[c][2];
}

// fam: 0 cos(kw r) / r, 1 sin(kw r) / r (the Helmholtz components), 2 exp(-kw r) / (4 pi r)
// (the screened-Coulomb kernel; kw = 0: Laplace)
__global__ void k_gen(int kind, const double* __restrict__ eq, const double* __restrict__ ck,
                      int n_s, int ld, double s, double kw, int fam, double* out) {
    const int c = blockIdx.z;
    const int m = blockIdx.y * blockDim.y + threadIdx.y;   // row: target point
    const int kk = blockIdx.x * blockDim.x + threadIdx.x;  // column: source point
    if (m >= ld || kk >= ld) return;
    double* o = out + (int64_t)c * ld * ld + (int64_t)kk * ld + m;   // A^T[k][m]
    if (m >= n_s || kk >= n_s) {
        *o = 0.0;
        return;
    }
    double ox = 0, oy = 0, oz = 0;
    if (kind == 0) disp_of(c, ox, oy, oz);
    else {
        ox = (c & 1) ? 1.0 : -1.0;
        oy = (c & 2) ? 1.0 : -1.0;
        oz = (c & 4) ? 1.0 : -1.0;
    }
    double x[3], y[3];
    for (int a = 0; a < 3; ++a) {
        const double e_m = eq[a * n_s + m], c_m = ck[a * n_s + m];
        const double e_k = eq[a * n_s + kk], c_k = ck[a * n_s + kk];
        const double off = a == 0 ? ox : a == 1 ? oy : oz;
        double xm, yk;
        if (kind == 0) {          // M2L
            xm = __dadd_rn(e_m, off);
            yk = e_k;
        } else if (kind == 1) {   // M2M
            xm = __dmul_rn(c_m, 2.0);
            yk = __dadd_rn(e_k, off);
        } else {                  // L2L
            xm = __dadd_rn(e_m, off);
            yk = __dmul_rn(c_k, 2.0);
        }
        x[a] = __dmul_rn(xm, s);
        y[a] = __dmul_rn(yk, s);
    }
    const double dx = __dsub_rn(x[0], y[0]), dy = __dsub_rn(x[1], y[1]), dz = __dsub_rn(x[2], y[2]);
    const double r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    if (fam == 2) {
        *o = exp(-kw * r) / (4.0 * M_PI * r);
        return;
    }
    double sn, cs;
    sincos(kw * r, &sn, &cs);
    *o = (fam == 1 ? sn : cs) / r;
}

__device__ __forceinline__ float tf32_round(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// Streamed M2L tables of one level, both kernel families from one sincos per
// entry. layout 0: FP64 A^T [fam][c][k][m] (the FP64 GEMM); layout 1: TF32 hi/lo
// halves as A [fam][c][m][k] (the tcgen05 path), hi at ws, lo after the hi block.
// The fastest thread index runs along the contiguous axis of the layout.
__global__ void k_gen_m2l_stream(const double* __restrict__ eq, int n_s, int ld, double s, double kw,
                                 int n_fam, int yukawa, int layout, void* ws) {
    const int c = blockIdx.z;
    const int a = blockIdx.x * blockDim.x + threadIdx.x;   // contiguous axis
    const int b = blockIdx.y * blockDim.y + threadIdx.y;
    if (a >= ld || b >= ld) return;
    const int m = layout == 0 ? a : b;
    const int kk = layout == 0 ? b : a;
    const size_t mat = (size_t)ld * ld;
    const size_t idx = (size_t)c * mat + (size_t)b * ld + a;
    const size_t fam_stride = (size_t)316 * mat;
    double v[2] = {0.0, 0.0};
    if (m < n_s && kk < n_s) {
        double ox, oy, oz;
        disp_of(c, ox, oy, oz);
        const double dx = __dsub_rn(__dmul_rn(__dadd_rn(eq[m], ox), s), __dmul_rn(eq[kk], s));
        const double dy = __dsub_rn(__dmul_rn(__dadd_rn(eq[n_s + m], oy), s), __dmul_rn(eq[n_s + kk], s));
        const double dz = __dsub_rn(__dmul_rn(__dadd_rn(eq[2 * n_s + m], oz), s),
                                    __dmul_rn(eq[2 * n_s + kk], s));
        const double r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
        if (yukawa) {
            v[0] = exp(-kw * r) / (4.0 * M_PI * r);
        } else {
            double sn, cs;
            sincos(kw * r, &sn, &cs);
            v[0] = cs / r;
            v[1] = sn / r;
        }
    }
    if (layout == 0) {
        double* o = static_cast<double*>(ws);
        for (int f = 0; f < n_fam; ++f) o[f * fam_stride + idx] = v[f];
    } else {
        float* hi = static_cast<float*>(ws);
        float* lo = hi + n_fam * fam_stride;
        for (int f = 0; f < n_fam; ++f) {
            const float h = tf32_round((float)v[f]);
            hi[f * fam_stride + idx] = h;
            lo[f * fam_stride + idx] = tf32_round((float)(v[f] - (double)h));
        }
    }
}

}  // namespace

size_t stream_ws_bytes(const hfmm_plan* P) {
    return (size_t)P->n_fam * 316 * (size_t)P->ld * P->ld * sizeof(double);
}

void generate_m2l_stream(hfmm_plan* P, int level, bool mixed, void* ws, cudaStream_t st) {
    const double s = P->extent * std::ldexp(1.0, -(level + 1));
    dim3 blk(32, 8);
    dim3 grid((unsigned)ceil_div(P->ld, 32), (unsigned)ceil_div(P->ld, 8), 316u);
    HFMM_LAUNCH(k_gen_m2l_stream, grid, blk, 0, st, P->equiv_pts.p, P->n_s, P->ld, s, P->k,
                P->n_fam, P->yukawa ? 1 : 0, mixed ? 1 : 0, ws);
}

void generate_tables(hfmm_plan* P, int fam, int level) {
    LevelTables& T = P->tables[fam][level];
    const int n_s = P->n_s, ld = P->ld;
    const double extent = P->extent;
    const double s = extent * std::ldexp(1.0, -(level + 1));
    const double s_child = extent * std::ldexp(1.0, -(level + 2));
    const int imag = P->yukawa ? 2 : (fam == 1 ? 1 : 0);   // the k_gen family code
    const size_t mat = (size_t)ld * ld;
    dim3 blk(32, 8);
    auto grid = [&](int count) {
        return dim3((unsigned)ceil_div(ld, 32), (unsigned)ceil_div(ld, 8), (unsigned)count);
    };
    if (P->streamed) {
        T.m2l.release();   // regenerated per evaluate (generate_m2l_stream)
    } else {
        T.m2l.alloc(316 * mat);
        HFMM_LAUNCH(k_gen, grid(316), blk, 0, 0, 0, P->equiv_pts.p, P->check_pts.p, n_s, ld, s, P->k,
                    imag, T.m2l.p);
    }
    if (level < P->md) {
        T.m2m.alloc(8 * mat);
        HFMM_LAUNCH(k_gen, grid(8), blk, 0, 0, 1, P->equiv_pts.p, P->check_pts.p, n_s, ld, s_child,
                    P->k, imag, T.m2m.p);
    } else {
        T.m2m.release();
    }
    if (level >= 3) {
        T.l2l.alloc(8 * mat);
        HFMM_LAUNCH(k_gen, grid(8), blk, 0, 0, 2, P->equiv_pts.p, P->check_pts.p, n_s, ld, s, P->k,
                    imag, T.l2l.p);
    } else {
        T.l2l.release();
    }
    HFMM_CUDA(cudaDeviceSynchronize());
}

}  // namespace hfmm
