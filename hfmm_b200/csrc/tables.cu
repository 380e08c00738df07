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

__device__ __forceinline__ void disp_of(int c, double& dx, double& dy, double& dz) {
    // the c-th non-adjacent displacement in (dx+3)*49 + (dy+3)*7 + (dz+3) order
    int seen = -1;
    for (int d = 0; d < N_DISP; ++d) {
        int ix = d / 49 - 3, iy = (d / 7) % 7 - 3, iz = d % 7 - 3;
        int mx = max(abs(ix), max(abs(iy), abs(iz)));
        if (mx > 1 && ++seen == c) {
            dx = 2.0 * ix;
            dy = 2.0 * iy;
            dz = 2.0 * iz;
            return;
        }
    }
    dx = dy = dz = 0.0;
}

__global__ void k_gen(int kind, const double* __restrict__ eq, const double* __restrict__ ck,
                      int n_s, int ld, double s, double kw, int imag, double* out) {
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
    double sn, cs;
    sincos(kw * r, &sn, &cs);
    *o = (imag ? sn : cs) / r;
}

}  // namespace

void generate_tables(hfmm_plan* P, int fam, int level) {
    LevelTables& T = P->tables[fam][level];
    const int n_s = P->n_s, ld = P->ld;
    const double extent = P->extent;
    const double s = extent * std::ldexp(1.0, -(level + 1));
    const double s_child = extent * std::ldexp(1.0, -(level + 2));
    const int imag = fam == 1 ? 1 : 0;
    const size_t mat = (size_t)ld * ld;
    dim3 blk(32, 8);
    auto grid = [&](int count) {
        return dim3((unsigned)ceil_div(ld, 32), (unsigned)ceil_div(ld, 8), (unsigned)count);
    };
    T.m2l.alloc(316 * mat);
    HFMM_LAUNCH(k_gen, grid(316), blk, 0, 0, 0, P->equiv_pts.p, P->check_pts.p, n_s, ld, s, P->k,
                imag, T.m2l.p);
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
