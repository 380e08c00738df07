// FP64 particle kernels of the plain path: P2M, P2L, L2P, M2P, P2P, the charge
// gather into leaf-major order and the final complex combine.
//
// Every kernel evaluates both Helmholtz components from one sincos per pair
// (family 0: cos(kr)/r, family 1: sin(kr)/r, HFMM.py:25-27) for R charge
// columns at once, and optionally the field -grad phi with the weights
// (cos + kr sin)/r^3 and (sin - kr cos)/r^3 (HFMM.py:29-40).
// Particles are in Morton-sorted order, so each leaf is a contiguous slice of
// the SoA position arrays (the role of _build_padded, near.py:589-598, without
// the padded copy).
#include "hfmm_internal.cuh"
#include "particles.cuh"

namespace hfmm {

namespace {

constexpr int STAGE = 128;   // particles staged in shared memory per pass

// Check potentials of one leaf at its upward check surface (phases.py:118-124).
// Also P2L (phases.py:1755-1769) when `surf` is the equivalent surface of a
// target box and the sources are the particles of its X-list leaves.
template <int NF, int R>
__global__ void __launch_bounds__(512) k_surface_from_particles(
    EvalView v, const int32_t* __restrict__ tgt_boxes, const int32_t* __restrict__ off,
    const int32_t* __restrict__ srcs, const double* __restrict__ surf, int only_level,
    double* check, int64_t fam_stride, int accumulate) {
    __shared__ double sx[STAGE], sy[STAGE], sz[STAGE], sq[R][STAGE];
    const int row = blockIdx.x;
    const int b = tgt_boxes[row];
    const int lvl = v.lvls[b];
    if (lvl < 2 || (only_level >= 0 && lvl != only_level)) return;
    const double h = v.hbox[b];
    const double cx = v.centre[b], cy = v.centre[v.nb + b], cz = v.centre[2 * v.nb + b];
    const int e0 = off ? off[row] : 0, e1 = off ? off[row + 1] : 1;
    for (int j0 = 0; j0 < v.n_s; j0 += blockDim.x) {
        const int j = j0 + threadIdx.x;
        const bool jok = j < v.n_s;
        double px = 0, py = 0, pz = 0;
        if (jok) {
            px = surf[j] * h + cx;
            py = surf[v.n_s + j] * h + cy;
            pz = surf[2 * v.n_s + j] * h + cz;
        }
        double acc[NF][R];
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
            for (int r = 0; r < R; ++r) acc[f][r] = 0.0;
        for (int e = e0; e < e1; ++e) {
            const int sb = srcs ? srcs[e] : b;
            const int s0 = v.leaf_start[sb], cnt = v.counts[sb];
            for (int p0 = 0; p0 < cnt; p0 += STAGE) {
                __syncthreads();
                for (int i = threadIdx.x; i < STAGE && p0 + i < cnt; i += blockDim.x) {
                    int64_t gi = s0 + p0 + i;
                    sx[i] = v.pos_s[gi];
                    sy[i] = v.pos_s[v.n + gi];
                    sz[i] = v.pos_s[2 * v.n + gi];
#pragma unroll
                    for (int r = 0; r < R; ++r) sq[r][i] = v.q_s[r * v.n + gi];
                }
                __syncthreads();
                if (jok) {
                    const int np = min(STAGE, cnt - p0);
                    for (int i = 0; i < np; ++i) {
                        double dx = px - sx[i], dy = py - sy[i], dz = pz - sz[i];
                        double r2 = dx * dx + dy * dy + dz * dz;
                        double ir = rsqrt(r2);
                        double rr = r2 * ir;
                        double sn, cs;
                        kernel_pair64(v.yukawa, v.k * rr, &sn, &cs);
                        double wc = cs * ir, ws = sn * ir;
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            acc[0][r] += sq[r][i] * wc;
                            if (NF == 2) acc[NF - 1][r] += sq[r][i] * ws;
                        }
                    }
                }
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

// Particle potentials (and field) from surface densities: L2P (phases.py:1571-1582,
// downward equivalent surface R_CHECK of the leaf itself) and M2P (phases.py:1101-1140,
// upward equivalent surface R_EQUIV of each W-list source box). One CTA per target
// leaf; a group of GL lanes shares a particle, each lane taking every GL-th surface
// point, so a warp works on 32 / GL particles at once and reduces over GL lanes only.
constexpr int GL = 8;
template <int NF, int R, bool FIELD>
__global__ void __launch_bounds__(256) k_particles_from_surface(
    EvalView v, const int32_t* __restrict__ tgt_leaves, const int32_t* __restrict__ off,
    const int32_t* __restrict__ srcs, const double* __restrict__ surf,
    const double* __restrict__ dens, int64_t fam_stride, double* pot, double* fld) {
    extern __shared__ double sh[];
    double* dn = sh;                          // [NF][R][n_s]
    double* ex = sh + NF * R * v.n_s;         // [3][n_s]
    const int row = blockIdx.x;
    const int t = tgt_leaves[row];
    if (v.lvls[t] < 2 && !off) return;        // L2P: no local expansion above level 2
    const int s0 = v.leaf_start[t], cnt = v.counts[t];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int grp = lane / GL, gl = lane % GL;   // particle slot of the warp, lane within it
    constexpr int PW = 32 / GL;                  // particles per warp at once
    const int e0 = off ? off[row] : 0, e1 = off ? off[row + 1] : 1;
    constexpr int NA = NF * R * (FIELD ? 4 : 1);
    for (int e = e0; e < e1; ++e) {
        const int sb = srcs ? srcs[e] : t;
        const double h = v.hbox[sb];
        const double c[3] = {v.centre[sb], v.centre[v.nb + sb], v.centre[2 * v.nb + sb]};
        __syncthreads();
        for (int j = threadIdx.x; j < v.n_s; j += blockDim.x) {
#pragma unroll
            for (int a = 0; a < 3; ++a) ex[a * v.n_s + j] = surf[a * v.n_s + j] * h + c[a];
#pragma unroll
            for (int f = 0; f < NF; ++f)
#pragma unroll
                for (int r = 0; r < R; ++r)
                    dn[(f * R + r) * v.n_s + j] = dens[f * fam_stride + ((int64_t)sb * R + r) * v.ld + j];
        }
        __syncthreads();
        for (int i0 = warp * PW; i0 < cnt; i0 += nw * PW) {
            const int i = i0 + grp;
            const bool act = i < cnt;
            const int64_t gi = s0 + (act ? i : 0);
            const double x = v.pos_s[gi], y = v.pos_s[v.n + gi], z = v.pos_s[2 * v.n + gi];
            double acc[NA];
#pragma unroll
            for (int q = 0; q < NA; ++q) acc[q] = 0.0;
            for (int j = gl; j < v.n_s; j += GL) {
                double dx = x - ex[j], dy = y - ex[v.n_s + j], dz = z - ex[2 * v.n_s + j];
                double r2 = dx * dx + dy * dy + dz * dz;
                double ir = rsqrt(r2);
                double rr = r2 * ir;
                double sn, cs;
                double kr = v.k * rr;
                kernel_pair64(v.yukawa, kr, &sn, &cs);
                double w[2] = {cs * ir, sn * ir};
                double wf[2] = {0.0, 0.0};
                if (FIELD) {
                    double ir3 = ir * ir * ir;
                    wf[0] = (cs + kr * sn) * ir3;
                    wf[1] = (sn - kr * cs) * ir3;
                }
#pragma unroll
                for (int f = 0; f < NF; ++f)
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        double d = dn[(f * R + r) * v.n_s + j];
                        acc[f * R + r] += d * w[f];
                        if (FIELD) {
                            double dw = d * wf[f];
                            acc[NF * R + (f * R + r) * 3 + 0] += dw * dx;
                            acc[NF * R + (f * R + r) * 3 + 1] += dw * dy;
                            acc[NF * R + (f * R + r) * 3 + 2] += dw * dz;
                        }
                    }
            }
#pragma unroll
            for (int q = 0; q < NA; ++q)
#pragma unroll
                for (int o = GL / 2; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
            if (gl == 0 && act) {
#pragma unroll
                for (int q = 0; q < NF * R; ++q) pot[q * v.n + gi] += acc[q];
                if (FIELD)
#pragma unroll
                    for (int q = 0; q < NF * R * 3; ++q) fld[q * v.n + gi] += acc[NF * R + q];
            }
        }
    }
}

// Near field over the U list + self pair of each target leaf (near.py:193-312),
// with the "pair" coincidence floor (near.py:252-261):
// d2 <= (16 eps)^2 (rmax_t + rmax_s)^2 counts as coincident and contributes 0.
template <int NF, int R, bool FIELD>
__global__ void __launch_bounds__(128) k_p2p(EvalView v, const int32_t* __restrict__ leaves,
                                            const int32_t* __restrict__ off,
                                            const int32_t* __restrict__ srcs, double* pot,
                                            double* fld) {
    __shared__ double sx[STAGE], sy[STAGE], sz[STAGE], sq[R][STAGE];
    const int row = blockIdx.x;
    const int t = leaves[row];
    const int s0t = v.leaf_start[t], cnt_t = v.counts[t];
    const double rt = v.rmax[t];
    constexpr int NA = NF * R * (FIELD ? 4 : 1);
    const double C16 = 1.2621774483536189e-29;   // (16 * 2^-52)^2
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
            const double rs = __dadd_rn(rt, v.rmax[sb]);
            const double thr = __dmul_rn(C16, __dmul_rn(rs, rs));
            for (int p0 = 0; p0 < cnt; p0 += STAGE) {
                __syncthreads();
                for (int k = threadIdx.x; k < STAGE && p0 + k < cnt; k += blockDim.x) {
                    int64_t gi = s0 + p0 + k;
                    sx[k] = v.pos_s[gi];
                    sy[k] = v.pos_s[v.n + gi];
                    sz[k] = v.pos_s[2 * v.n + gi];
#pragma unroll
                    for (int r = 0; r < R; ++r) sq[r][k] = v.q_s[r * v.n + gi];
                }
                __syncthreads();
                if (!act) continue;
                const int np = min(STAGE, cnt - p0);
                for (int k = 0; k < np; ++k) {
                    double dx = x - sx[k], dy = y - sy[k], dz = z - sz[k];
                    double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                    if (!(d2 > thr)) continue;
                    double rr = sqrt(d2);
                    double kr = v.k * rr;
                    double sn, cs;
                    if (v.yukawa) {
                        sn = cs = exp(-kr) * INV_4PI;
                    } else {
                        sincos(kr, &sn, &cs);
                    }
                    double ir = 1.0 / rr;
                    double w[2] = {cs * ir, sn * ir};
                    double wf[2] = {0.0, 0.0};
                    if (FIELD) {
                        double ir3 = ir * ir * ir;
                        wf[0] = (cs + kr * sn) * ir3;
                        wf[1] = (sn - kr * cs) * ir3;
                    }
#pragma unroll
                    for (int f = 0; f < NF; ++f)
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            double q = sq[r][k];
                            acc[f * R + r] += q * w[f];
                            if (FIELD) {
                                double qw = q * wf[f];
                                acc[NF * R + (f * R + r) * 3 + 0] += qw * dx;
                                acc[NF * R + (f * R + r) * 3 + 1] += qw * dy;
                                acc[NF * R + (f * R + r) * 3 + 2] += qw * dz;
                            }
                        }
                }
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

__global__ void k_gather_q(int64_t n, const int32_t* __restrict__ sidx, const double* __restrict__ q_re,
                           const double* __restrict__ q_im, double* q_s) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t o = sidx[i];
    q_s[i] = q_re[o];
    if (q_im) q_s[n + i] = q_im[o];
}

// phi = E_cos(q_re) - E_sin(q_im) + i (E_sin(q_re) + E_cos(q_im)), back to input order
template <int NF, int R, bool FIELD>
__global__ void k_combine(int64_t n, const int32_t* __restrict__ sidx, const double* __restrict__ pot,
                          const double* __restrict__ fld, double* phi, double* E) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t o = sidx[i];
    double c0 = pot[(0 * R + 0) * n + i];
    double c1 = R == 2 ? pot[(0 * R + 1) * n + i] : 0.0;
    double s0 = NF == 2 ? pot[(1 * R + 0) * n + i] : 0.0;
    double s1 = (NF == 2 && R == 2) ? pot[(1 * R + 1) * n + i] : 0.0;
    double re = c0 - s1, im = s0 + c1;
    phi[2 * o] = re;
    phi[2 * o + 1] = im;
    if (FIELD) {
        for (int a = 0; a < 3; ++a) {
            double c0 = fld[((0 * R + 0) * 3 + a) * n + i];
            double c1 = R == 2 ? fld[((0 * R + 1) * 3 + a) * n + i] : 0.0;
            double s0 = NF == 2 ? fld[((1 * R + 0) * 3 + a) * n + i] : 0.0;
            double s1 = (NF == 2 && R == 2) ? fld[((1 * R + 1) * 3 + a) * n + i] : 0.0;
            E[(o * 3 + a) * 2] = c0 - s1;
            E[(o * 3 + a) * 2 + 1] = s0 + c1;
        }
    }
}

inline int nblk(int64_t n, int t) { return (int)std::max<int64_t>(1, ceil_div(n, t)); }

// threads of a surface kernel: one per surface point in as few passes as possible
// (n_s = 296 at p = 8 takes 320 threads in one pass, not 256 + 40 in two)
inline int surface_threads(int n_s) {
    const int passes = (int)ceil_div(n_s, 512);
    return (int)std::min<int64_t>(512, round_up(ceil_div(n_s, passes), 32));
}

template <int NF, int R, bool FIELD>
void particles_impl(const ParticlePass& p, cudaStream_t s) {
    const EvalView& v = p.v;
    switch (p.op) {
        case ParticleOp::P2M:
            HFMM_LAUNCH((k_surface_from_particles<NF, R>), p.nrows, surface_threads(v.n_s), 0, s, v,
                        p.rows, p.off, p.srcs, p.surf, -1, p.out, p.fam_stride, 0);
            break;
        case ParticleOp::P2L:
            HFMM_LAUNCH((k_surface_from_particles<NF, R>), p.nrows, surface_threads(v.n_s), 0, s, v,
                        p.rows, p.off, p.srcs, p.surf, p.level, p.out, p.fam_stride, 1);
            break;
        case ParticleOp::L2P:
        case ParticleOp::M2P: {
            size_t smem = (size_t)(NF * R + 3) * v.n_s * sizeof(double);
            auto kern = k_particles_from_surface<NF, R, FIELD>;
            HFMM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            HFMM_LAUNCH(kern, p.nrows, 256, smem, s, v, p.rows, p.off, p.srcs, p.surf, p.dens,
                        p.fam_stride, p.pot, p.fld);
            break;
        }
        case ParticleOp::P2P:
            HFMM_LAUNCH((k_p2p<NF, R, FIELD>), p.nrows, 128, 0, s, v, p.rows, p.off, p.srcs, p.pot,
                        p.fld);
            break;
        case ParticleOp::COMBINE:
            HFMM_LAUNCH((k_combine<NF, R, FIELD>), nblk(v.n, 256), 256, 0, s, v.n, p.rows, p.pot,
                        p.fld, p.phi, p.E);
            break;
    }
}

}  // namespace

void gather_charges(int64_t n, const int32_t* sidx, const double* q_re, const double* q_im,
                    double* q_s, cudaStream_t s) {
    HFMM_LAUNCH(k_gather_q, nblk(n, 256), 256, 0, s, n, sidx, q_re, q_im, q_s);
}

void particles_f64(const ParticlePass& p, cudaStream_t s) {
    if (p.nrows == 0 && p.op != ParticleOp::COMBINE) return;
    const int key = (p.nf - 1) * 4 + (p.R - 1) * 2 + (p.field ? 1 : 0);
    switch (key) {
        case 0: particles_impl<1, 1, false>(p, s); break;
        case 1: particles_impl<1, 1, true>(p, s); break;
        case 2: particles_impl<1, 2, false>(p, s); break;
        case 3: particles_impl<1, 2, true>(p, s); break;
        case 4: particles_impl<2, 1, false>(p, s); break;
        case 5: particles_impl<2, 1, true>(p, s); break;
        case 6: particles_impl<2, 2, false>(p, s); break;
        case 7: particles_impl<2, 2, true>(p, s); break;
        default: throw Error{HFMM_ERR_ARG, "particles_f64: bad configuration"};
    }
}

}  // namespace hfmm
