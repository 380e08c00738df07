// Device octree build: the B200 form of build_fmm_tree / build_fmm_tree_auto /
// assign_particles (jaxfmm/trees/cubic.py:316-695).
//
// Integer work, reproduced index for index (box numbering, parent pointers,
// leaf slots). The reference runs every step over its whole fixed buffer; here
// each coarsening step touches only the level being merged and its new parents:
//
//   particles:  Morton code at max_depth (cubic.py:385-392) -> stable radix sort
//               (cubic.py:397) -> run-length boxes (cubic.py:404-411)
//   per level:  parents by run of Morton/8 (cubic.py:429-441), counts, the 2:1
//               balance test (cubic.py:454-475), deletion of merged children and
//               fine-to-coarse compaction with parent remap (cubic.py:477-502)
//   leaves:     start of each leaf in the sorted particle order (the scaled-Morton
//               ordering of assign_particles, cubic.py:655-693)
//
// The reference's child table is a scatter with repeated indices; rows that the
// balance test reads are reproduced with last-write-wins (largest writer index),
// the same convention as the oracle.
#include "hfmm_internal.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>

namespace hfmm {

namespace {

constexpr int TPB = 256;

__global__ void k_minmax_partial(const double* __restrict__ pos, int64_t n, double* part,
                                 int* bad) {
    __shared__ double smin[3][TPB], smax[3][TPB];
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        for (int a = 0; a < 3; ++a) {
            double v = pos[i * 3 + a];
            if (!isfinite(v)) atomicOr(bad, 1);
            mn[a] = fmin(mn[a], v);
            mx[a] = fmax(mx[a], v);
        }
    }
    for (int a = 0; a < 3; ++a) {
        smin[a][threadIdx.x] = mn[a];
        smax[a][threadIdx.x] = mx[a];
    }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int a = 0; a < 3; ++a) {
                smin[a][threadIdx.x] = fmin(smin[a][threadIdx.x], smin[a][threadIdx.x + s]);
                smax[a][threadIdx.x] = fmax(smax[a][threadIdx.x], smax[a][threadIdx.x + s]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int a = 0; a < 3; ++a) {
            part[blockIdx.x * 6 + a] = smin[a][0];
            part[blockIdx.x * 6 + 3 + a] = smax[a][0];
        }
}

__global__ void k_minmax_final(const double* part, int nblk, double* out) {
    int a = threadIdx.x;   // 6 threads: 3 min, 3 max
    if (a >= 6) return;
    double v = a < 3 ? INFINITY : -INFINITY;
    for (int b = 0; b < nblk; ++b) v = a < 3 ? fmin(v, part[b * 6 + a]) : fmax(v, part[b * 6 + a]);
    out[a] = v;
}

// Morton code at depth md: uint64(((x - pmin) / extent) * 2^md), clipped (cubic.py:390-392).
__global__ void k_morton(const double* __restrict__ pos, int64_t n, double p0, double p1,
                         double p2, double extent, int md, uint64_t* keys, int32_t* vals) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double grid = (double)(1ull << md);
    uint64_t gmax = (1ull << md) - 1;
    uint64_t g[3];
    double pm[3] = {p0, p1, p2};
    for (int a = 0; a < 3; ++a) {
        double s = __dmul_rn(__ddiv_rn(__dsub_rn(pos[i * 3 + a], pm[a]), extent), grid);
        uint64_t c = (extent > 0.0 && s > 0.0) ? __double2ull_rz(s) : 0ull;
        g[a] = c > gmax ? gmax : c;
    }
    keys[i] = morton3(g[0], g[1], g[2]);
    vals[i] = (int32_t)i;
}

__global__ void k_heads(const uint64_t* __restrict__ k, int64_t n, int32_t* head) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    head[i] = (i == 0 || k[i] != k[i - 1]) ? 1 : 0;
}

// Finest boxes from the runs of equal codes: counts and codes (cubic.py:404-411).
__global__ void k_runs(const uint64_t* __restrict__ k, const int32_t* __restrict__ incl,
                       int64_t n, int32_t* run_start) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i == 0 || k[i] != k[i - 1]) run_start[incl[i] - 1] = (int32_t)i;
}

__global__ void k_finest(const uint64_t* __restrict__ k, const int32_t* __restrict__ run_start,
                         int64_t nu, int64_t n, int md, uint64_t* m_id, int32_t* p_id,
                         int32_t* lvls, int32_t* counts, uint8_t* is_leaf) {
    int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= nu) return;
    int64_t s = run_start[b];
    int64_t e = (b + 1 < nu) ? run_start[b + 1] : n;
    m_id[b] = k[s];
    counts[b] = (int32_t)(e - s);
    lvls[b] = md;
    p_id[b] = 0;
    is_leaf[b] = 1;
}

// flag[j] = 1 where box a+j starts a new parent run (cubic.py:436-441)
__global__ void k_parent_heads(const uint64_t* __restrict__ m, int64_t a, int64_t nL,
                               int32_t* flag) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nL) return;
    flag[j] = (j > 0 && (m[a + j] >> 3) != (m[a + j - 1] >> 3)) ? 1 : 0;
}

__global__ void k_make_parents(uint64_t* m, int32_t* p_id, int32_t* lvls, int32_t* counts,
                               uint8_t* is_leaf, const int32_t* __restrict__ pidx, int64_t a,
                               int64_t nL, int64_t ofs, int L) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nL) return;
    int64_t P = ofs + pidx[j];
    p_id[a + j] = (int32_t)P;
    atomicAdd(&counts[P], counts[a + j]);
    if (j == 0 || pidx[j] != pidx[j - 1]) {
        m[P] = m[a + j] >> 3;
        lvls[P] = L - 1;
        p_id[P] = 0;          // unset until the next step (the reference's initial 0)
        is_leaf[P] = 0;
    }
}

// child table rows written by every box (last write = largest index wins)
__global__ void k_child_table(const uint64_t* __restrict__ m, const int32_t* __restrict__ p_id,
                              int64_t nbox, int32_t* child_tab, int* err) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nbox) return;
    int64_t r = p_id[j];
    if (r < 0 || r >= nbox) {
        atomicOr(err, ERRF_BOUNDS);
        return;
    }
    atomicMax(&child_tab[r * 8 + (int)(m[j] & 7ull)], (int32_t)j);
}

__device__ __forceinline__ bool adj_child(int d, int c) {
    int dx, dy, dz;
    neigh_offset(d, dx, dy, dz);
    int o[3] = {dx, dy, dz};
    for (int ax = 0; ax < 3; ++ax) {
        int cb = (c >> ax) & 1;
        bool ok = (o[ax] == -1 && cb == 1) || (o[ax] == 1 && cb == 0) || o[ax] == 0;
        if (!ok) return false;
    }
    return true;
}

// 2:1 balance (cubic.py:454-475) and the merge decision for each new parent.
__global__ void k_balance(const uint64_t* __restrict__ m, const int32_t* __restrict__ counts,
                          const uint8_t* __restrict__ is_leaf,
                          const int32_t* __restrict__ child_tab, int64_t ofs, int64_t np, int L,
                          int n_max, int check_balance, uint8_t* merge) {
    int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= np) return;
    int64_t P = ofs + q;
    bool ok = counts[P] <= n_max;
    if (ok && check_balance) {
        int64_t x, y, z;
        demorton3(m[P], x, y, z);
        int64_t grid = 1ll << (L - 1);
        for (int d = 0; d < 26 && ok; ++d) {
            int dx, dy, dz;
            neigh_offset(d, dx, dy, dz);
            int64_t nx = x + dx, ny = y + dy, nz = z + dz;
            if (nx < 0 || ny < 0 || nz < 0 || nx >= grid || ny >= grid || nz >= grid) continue;
            uint64_t nm = morton3(nx, ny, nz);
            // searchsorted(side='right') - 1 over [0]*ofs ++ parent codes ++ [MAX]*
            int64_t lo = 0, hi = np;   // first parent code > nm
            while (lo < hi) {
                int64_t mid = (lo + hi) >> 1;
                if (m[ofs + mid] <= nm) lo = mid + 1;
                else hi = mid;
            }
            int64_t row;
            if (lo > 0 && m[ofs + lo - 1] == nm) row = ofs + lo - 1;
            else if (lo == 0 && nm == 0ull) row = ofs - 1;   // matches the zero-filled prefix
            else continue;
            for (int c = 0; c < 8; ++c)
                if (adj_child(d, c) && !is_leaf[child_tab[row * 8 + c]]) {
                    ok = false;
                    break;
                }
        }
    }
    merge[q] = ok ? 1 : 0;
}

// keep flags over [a, a+nL+np): level-L boxes are dropped when their parent merges
__global__ void k_keep(const int32_t* __restrict__ p_id, const uint8_t* __restrict__ merge,
                       int64_t a, int64_t nL, int64_t np, int64_t ofs, int32_t* keep) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nL + np) return;
    if (j < nL) keep[j] = merge[p_id[a + j] - ofs] ? 0 : 1;
    else keep[j] = 1;
}

__device__ __forceinline__ int64_t remap(int64_t x, int64_t a, const int32_t* incl) {
    return x < a ? x : a + incl[x - a] - 1;
}

__global__ void k_compact(const uint64_t* m, const int32_t* p_id, const int32_t* lvls,
                          const int32_t* counts, const uint8_t* is_leaf,
                          const uint8_t* __restrict__ merge, const int32_t* __restrict__ keep,
                          const int32_t* __restrict__ incl, int64_t a, int64_t nL, int64_t np,
                          int64_t nbox, uint64_t* m2, int32_t* p2, int32_t* l2, int32_t* c2,
                          uint8_t* f2, int64_t nbox_old_total) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nbox) return;
    int64_t dst;
    if (j < a) dst = j;
    else {
        if (!keep[j - a]) return;
        dst = a + incl[j - a] - 1;
    }
    int64_t pp = p_id[j];
    if (pp < 0) pp += nbox_old_total;   // negative indices wrap (JAX index normalisation)
    m2[dst] = m[j];
    l2[dst] = lvls[j];
    c2[dst] = counts[j];
    uint8_t leaf = is_leaf[j];
    if (j >= a + nL) leaf = leaf | merge[j - a - nL];
    f2[dst] = leaf;
    p2[dst] = (pp >= 0 && pp < nbox) ? (int32_t)remap(pp, a, incl) : 0;
}

__global__ void k_level1_self(const int32_t* __restrict__ lvls, int64_t nb, int32_t* p_id) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < nb && lvls[j] == 1) p_id[j] = (int32_t)j;
}

// Leaf start in the Morton-sorted particle order = lower_bound of its scaled code.
__global__ void k_leaf_start(const uint64_t* __restrict__ m, const int32_t* __restrict__ lvls,
                             const uint8_t* __restrict__ is_leaf,
                             const uint64_t* __restrict__ skeys, int64_t n, int64_t nb, int md,
                             int32_t* leaf_start) {
    int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= nb) return;
    if (!is_leaf[b] || lvls[b] <= 0) {
        leaf_start[b] = -1;
        return;
    }
    uint64_t code = m[b] << (3 * (md - lvls[b]));
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (skeys[mid] < code) lo = mid + 1;
        else hi = mid;
    }
    leaf_start[b] = (int32_t)lo;
}

__global__ void k_sorted_layout(const double* __restrict__ pos, const int32_t* __restrict__ sidx,
                                int64_t n, double* pos_s, int32_t* rank) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t o = sidx[i];
    for (int a = 0; a < 3; ++a) pos_s[a * n + i] = pos[o * 3 + a];
    rank[o] = (int32_t)i;
}

// Box centres and half-sides (cubic.py:116-160).
__global__ void k_geometry(const uint64_t* __restrict__ m, const int32_t* __restrict__ lvls,
                           int64_t nb, double extent, double p0, double p1, double p2,
                           double* centre, double* h) {
    int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= nb) return;
    int64_t g[3];
    demorton3(m[b], g[0], g[1], g[2]);
    int l = lvls[b];
    double pm[3] = {p0, p1, p2};
    double div = (double)(1ll << l);
    double half = extent * ldexp(1.0, -(l + 1));
    for (int a = 0; a < 3; ++a)
        centre[a * nb + b] = __dadd_rn(__dadd_rn(__ddiv_rn(__dmul_rn((double)g[a], extent), div), half), pm[a]);
    h[b] = half;
}

// sqrt(max |x|^2) over a leaf's padded slots; padding slots hold particle 0
// (near.py:589-598), so they count when the leaf is not full.
__global__ void k_rmax(const double* __restrict__ pos, const double* __restrict__ pos_s,
                       const int32_t* __restrict__ leaf_start, const int32_t* __restrict__ counts,
                       int64_t n, int64_t nb, int maxleaf, double* rmax) {
    int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= nb) return;
    int64_t s = leaf_start[b];
    if (s < 0) {
        rmax[b] = 0.0;
        return;
    }
    double mx = 0.0;
    int c = counts[b];
    for (int i = 0; i < c; ++i) {
        double x = pos_s[s + i], y = pos_s[n + s + i], z = pos_s[2 * n + s + i];
        mx = fmax(mx, __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
    }
    if (c < maxleaf) {
        double x = pos[0], y = pos[1], z = pos[2];
        mx = fmax(mx, __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
    }
    rmax[b] = sqrt(mx);
}

inline int nblocks(int64_t n) { return (int)std::max<int64_t>(1, ceil_div(n, TPB)); }

template <typename T>
void to_host(std::vector<T>& v, const T* d, size_t n) {
    v.resize(n);
    if (n) HFMM_CUDA(cudaMemcpy(v.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost));
}

template <typename T>
T scalar_to_host(const T* d) {
    T v;
    HFMM_CUDA(cudaMemcpy(&v, d, sizeof(T), cudaMemcpyDeviceToHost));
    return v;
}

void inclusive_scan(const int32_t* in, int32_t* out, int64_t n, DevBuf<uint8_t>& tmp) {
    size_t bytes = 0;
    HFMM_CUDA(cub::DeviceScan::InclusiveSum(nullptr, bytes, in, out, (int)n));
    if (bytes > tmp.n) tmp.alloc(bytes);
    HFMM_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, bytes, in, out, (int)n));
}

struct BoxArrays {
    DevBuf<uint64_t> m;
    DevBuf<int32_t> p, l, c;
    DevBuf<uint8_t> f;
    void alloc(int64_t cap) {
        m.alloc(cap);
        p.alloc(cap);
        l.alloc(cap);
        c.alloc(cap);
        f.alloc(cap);
    }
};

struct BuildResult {
    int64_t nb;
    int64_t max_box_count;
    int levels_counts[MAX_LEVELS];
};

// One fixed-depth build (cubic.py:316-527). Leaves the boxes in `A`.
BuildResult build_depth(int64_t n, int md, int n_max, const DevBuf<uint64_t>& skeys,
                        BoxArrays& A, BoxArrays& B, DevBuf<int32_t>& w1, DevBuf<int32_t>& w2,
                        DevBuf<uint8_t>& mergebuf, DevBuf<int32_t>& child_tab,
                        DevBuf<uint8_t>& tmp, int* d_err) {
    BuildResult res{};
    // run-length boxes
    DevBuf<int32_t> head, incl;
    head.alloc(n);
    incl.alloc(n);
    HFMM_LAUNCH(k_heads, nblocks(n), TPB, 0, 0, skeys.p, n, head.p);
    inclusive_scan(head.p, incl.p, n, tmp);
    int64_t nu = scalar_to_host(incl.p + (n - 1));
    // capacity: boxes per level <= min(nu, 8^l)
    int64_t cap = 0;
    for (int l = 1; l <= md; ++l) cap += std::min<int64_t>(nu, l < 21 ? (1ll << (3 * l)) : nu);
    cap = std::max<int64_t>(cap, nu) + 8;
    A.alloc(cap);
    B.alloc(cap);
    w1.alloc(cap);
    w2.alloc(cap);
    mergebuf.alloc(cap);
    child_tab.alloc(cap * 8);
    {
        DevBuf<int32_t> run_start;
        run_start.alloc(nu);
        HFMM_LAUNCH(k_runs, nblocks(n), TPB, 0, 0, skeys.p, incl.p, n, run_start.p);
        HFMM_LAUNCH(k_finest, nblocks(nu), TPB, 0, 0, skeys.p, run_start.p, nu, n, md, A.m.p,
                    A.p.p, A.l.p, A.c.p, A.f.p);
    }
    res.max_box_count = nu - 1;
    int64_t nact = nu;   // boxes [0, nact) active, all at levels >= L
    int64_t nL = nu;     // the last run (level L) = [nact - nL, nact)
    for (int i = 0; i <= md - 2; ++i) {
        int L = md - i;
        int64_t a = nact - nL, ofs = nact;
        HFMM_LAUNCH(k_parent_heads, nblocks(nL), TPB, 0, 0, A.m.p, a, nL, w1.p);
        inclusive_scan(w1.p, w2.p, nL, tmp);
        int64_t np = (int64_t)scalar_to_host(w2.p + (nL - 1)) + 1;
        res.max_box_count = std::max<int64_t>(res.max_box_count, ofs + np);
        if (ofs + np > (int64_t)A.m.n) throw Error{HFMM_ERR_CAPACITY, "tree: box capacity exceeded"};
        HFMM_CUDA(cudaMemset(A.c.p + ofs, 0, np * sizeof(int32_t)));
        HFMM_LAUNCH(k_make_parents, nblocks(nL), TPB, 0, 0, A.m.p, A.p.p, A.l.p, A.c.p, A.f.p,
                    w2.p, a, nL, ofs, L);
        int check_balance = i >= 1 ? 1 : 0;
        if (check_balance) {
            HFMM_CUDA(cudaMemset(child_tab.p, 0, (ofs + np) * 8 * sizeof(int32_t)));
            HFMM_LAUNCH(k_child_table, nblocks(ofs + np), TPB, 0, 0, A.m.p, A.p.p, ofs + np,
                        child_tab.p, d_err);
        }
        HFMM_LAUNCH(k_balance, nblocks(np), TPB, 0, 0, A.m.p, A.c.p, A.f.p, child_tab.p, ofs,
                    np, L, n_max, check_balance, mergebuf.p);
        HFMM_LAUNCH(k_keep, nblocks(nL + np), TPB, 0, 0, A.p.p, mergebuf.p, a, nL, np, ofs, w1.p);
        inclusive_scan(w1.p, w2.p, nL + np, tmp);
        int64_t kept = scalar_to_host(w2.p + (nL + np - 1));
        int64_t nbox = ofs + np;
        HFMM_LAUNCH(k_compact, nblocks(nbox), TPB, 0, 0, A.m.p, A.p.p, A.l.p, A.c.p, A.f.p,
                    mergebuf.p, w1.p, w2.p, a, nL, np, nbox, B.m.p, B.p.p, B.l.p, B.c.p, B.f.p,
                    nbox);
        std::swap(A.m.p, B.m.p);
        std::swap(A.p.p, B.p.p);
        std::swap(A.l.p, B.l.p);
        std::swap(A.c.p, B.c.p);
        std::swap(A.f.p, B.f.p);
        nact = a + kept;
        nL = np;
    }
    HFMM_LAUNCH(k_level1_self, nblocks(nact), TPB, 0, 0, A.l.p, nact, A.p.p);
    res.nb = nact;
    return res;
}

}  // namespace

// Positions as FP32 pairs: hi = fl32(x), lo = fl32(x - hi); hi + lo carries x to
// about 48 bits, and a separation formed as (hi - hi') + (lo - lo') in FP32 has the
// relative accuracy of an FP32 number however close the two points are.
__global__ void k_split_pos(const double* __restrict__ pos, int64_t m, float* out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    const double x = pos[i];
    const float hi = (float)x;
    out[i] = hi;
    out[m + i] = (float)(x - (double)hi);
}

void tree_build(hfmm_plan* P, const double* pos_dev) {
    const int64_t n = P->n;
    int* d_err = P->d_err.p;
    DevBuf<uint8_t> tmp;
    // bounding box (cubic.py:364-375)
    int nblk = (int)std::min<int64_t>(1024, nblocks(n));
    DevBuf<double> part, mm;
    part.alloc(nblk * 6);
    mm.alloc(6);
    DevBuf<int> bad;
    bad.alloc(1);
    bad.zero();
    HFMM_LAUNCH(k_minmax_partial, nblk, TPB, 0, 0, pos_dev, n, part.p, bad.p);
    HFMM_LAUNCH(k_minmax_final, 1, 32, 0, 0, part.p, nblk, mm.p);
    double h_mm[6];
    HFMM_CUDA(cudaMemcpy(h_mm, mm.p, sizeof(h_mm), cudaMemcpyDeviceToHost));
    if (scalar_to_host(bad.p)) throw Error{HFMM_ERR_ARG, "positions must be finite"};
    double extent = 0.0;
    if (P->domain_fixed) {   // every point inside the given cube, before the plan changes
        extent = P->extent;
        for (int a = 0; a < 3; ++a)
            if (!(h_mm[a] >= P->pmin[a] && h_mm[3 + a] <= P->pmin[a] + extent))
                throw Error{HFMM_ERR_CAPACITY, "points outside the plan's fixed domain"};
        for (int a = 0; a < 3; ++a) h_mm[a] = P->pmin[a];
    } else {
        for (int a = 0; a < 3; ++a) extent = std::max(extent, h_mm[3 + a] - h_mm[a]);
        P->extent = extent;
        for (int a = 0; a < 3; ++a) P->pmin[a] = h_mm[a];
    }

    // depth and buffer schedule of build_fmm_tree_auto (cubic.py:577-600)
    int md;
    if (P->md_given) md = P->md;
    else {
        double ratio = std::max((double)n / (double)std::max(P->n_max, 1), 1.0);
        md = std::max(2, (int)std::ceil(std::log(ratio) / std::log(8.0)));
    }
    int64_t mb = std::max<int64_t>(4 * n / P->n_max, 512) + 4096;

    DevBuf<uint64_t> keys, skeys;
    DevBuf<int32_t> vals, svals;
    keys.alloc(n);
    skeys.alloc(n);
    vals.alloc(n);
    svals.alloc(n);
    BoxArrays A, B;
    DevBuf<int32_t> w1, w2, child_tab;
    DevBuf<uint8_t> mergebuf;
    BuildResult res{};
    while (true) {
        if (md < 1 || md > 20) throw Error{HFMM_ERR_ARG, "max_depth out of range (1..20)"};
        HFMM_LAUNCH(k_morton, nblocks(n), TPB, 0, 0, pos_dev, n, h_mm[0], h_mm[1], h_mm[2],
                    extent, md, keys.p, vals.p);
        size_t bytes = 0;
        HFMM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys.p, skeys.p, vals.p, svals.p,
                                                  (int)n, 0, 3 * md));
        if (bytes > tmp.n) tmp.alloc(bytes);
        HFMM_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, keys.p, skeys.p, vals.p, svals.p,
                                                  (int)n, 0, 3 * md));
        res = build_depth(n, md, P->n_max, skeys, A, B, w1, w2, mergebuf, child_tab, tmp, d_err);
        int tries = 1;
        while (res.max_box_count >= mb) {   // the reference rebuilds with a doubled buffer
            if (tries >= 10)
                throw Error{HFMM_ERR_CAPACITY,
                            "build_fmm_tree_auto: box buffer kept overflowing; check max_depth/N_max"};
            mb *= 2;
            ++tries;
        }
        // realised max leaf occupancy
        std::vector<int32_t> hc, hl;
        std::vector<uint8_t> hf;
        to_host(hc, A.c.p, res.nb);
        to_host(hl, A.l.p, res.nb);
        to_host(hf, A.f.p, res.nb);
        int maxleaf = 0;
        for (int64_t b = 0; b < res.nb; ++b)
            if (hf[b] && hl[b] > 0) maxleaf = std::max(maxleaf, hc[b]);
        P->maxleaf = maxleaf;
        if (P->md_given || maxleaf <= 2 * P->n_max || md >= 10) break;
        md += 1;
    }
    P->md = md;
    P->ref_max_boxes = mb;
    const int64_t nb = res.nb;
    P->nb = nb;
    if (md >= MAX_LEVELS) throw Error{HFMM_ERR_CAPACITY, "tree deeper than supported"};

    // final box arrays (exact size)
    P->m_id.alloc(nb);
    P->p_id.alloc(nb);
    P->lvls.alloc(nb);
    P->counts.alloc(nb);
    P->is_leaf.alloc(nb);
    HFMM_CUDA(cudaMemcpy(P->m_id.p, A.m.p, nb * 8, cudaMemcpyDeviceToDevice));
    HFMM_CUDA(cudaMemcpy(P->p_id.p, A.p.p, nb * 4, cudaMemcpyDeviceToDevice));
    HFMM_CUDA(cudaMemcpy(P->lvls.p, A.l.p, nb * 4, cudaMemcpyDeviceToDevice));
    HFMM_CUDA(cudaMemcpy(P->counts.p, A.c.p, nb * 4, cudaMemcpyDeviceToDevice));
    HFMM_CUDA(cudaMemcpy(P->is_leaf.p, A.f.p, nb, cudaMemcpyDeviceToDevice));
    to_host(P->h_m_id, P->m_id.p, nb);
    to_host(P->h_lvls, P->lvls.p, nb);
    to_host(P->h_counts, P->counts.p, nb);
    to_host(P->h_p_id, P->p_id.p, nb);
    to_host(P->h_is_leaf, P->is_leaf.p, nb);
    for (int l = 0; l < MAX_LEVELS; ++l) P->level_lo[l] = P->level_hi[l] = 0;
    std::vector<int> seen(MAX_LEVELS, 0);
    int64_t nleaves = 0;
    std::vector<int32_t> leaf_levels;
    for (int64_t b = 0; b < nb; ++b) {
        int l = P->h_lvls[b];
        if (l < 0 || l >= MAX_LEVELS) throw Error{HFMM_ERR_STATE, "tree: bad level"};
        if (!seen[l]) {
            P->level_lo[l] = (int)b;
            seen[l] = 1;
        }
        P->level_hi[l] = (int)(b + 1);
        if (P->h_is_leaf[b] && l > 0) {
            ++nleaves;
            leaf_levels.push_back(l);
        }
    }
    // boxes of one level must be contiguous (fine-to-coarse packing)
    for (int64_t b = 1; b < nb; ++b)
        if (P->h_lvls[b] > P->h_lvls[b - 1]) throw Error{HFMM_ERR_STATE, "tree: levels not packed"};
    P->n_leaves = nleaves;
    std::sort(leaf_levels.begin(), leaf_levels.end());
    P->adaptive = !leaf_levels.empty() && leaf_levels.front() != leaf_levels.back();

    // particle layout
    P->sort_idx.alloc(n);
    HFMM_CUDA(cudaMemcpy(P->sort_idx.p, svals.p, n * 4, cudaMemcpyDeviceToDevice));
    P->rank.alloc(n);
    P->pos_s.alloc(3 * n);
    HFMM_LAUNCH(k_sorted_layout, nblocks(n), TPB, 0, 0, pos_dev, P->sort_idx.p, n, P->pos_s.p,
                P->rank.p);
    P->leaf_start.alloc(nb);
    HFMM_LAUNCH(k_leaf_start, nblocks(nb), TPB, 0, 0, P->m_id.p, P->lvls.p, P->is_leaf.p, skeys.p,
                n, nb, md, P->leaf_start.p);
    P->centre.alloc(3 * nb);
    P->hbox.alloc(nb);
    HFMM_LAUNCH(k_geometry, nblocks(nb), TPB, 0, 0, P->m_id.p, P->lvls.p, nb, extent, h_mm[0],
                h_mm[1], h_mm[2], P->centre.p, P->hbox.p);
    {   // the leaves must tile the sorted particle range exactly before any kernel indexes it
        std::vector<int32_t> ls;
        to_host(ls, P->leaf_start.p, nb);
        std::vector<std::pair<int64_t, int64_t>> seg;
        for (int64_t b = 0; b < nb; ++b)
            if (P->h_is_leaf[b] && P->h_lvls[b] > 0) {
                if (ls[b] < 0 || P->h_counts[b] <= 0 || ls[b] + (int64_t)P->h_counts[b] > n)
                    throw Error{HFMM_ERR_STATE, "tree: leaf slice out of range"};
                seg.push_back({ls[b], P->h_counts[b]});
            }
        std::sort(seg.begin(), seg.end());
        int64_t at = 0;
        for (auto& sg : seg) {
            if (sg.first != at) throw Error{HFMM_ERR_STATE, "tree: leaves do not tile the particles"};
            at += sg.second;
        }
        if (at != n) throw Error{HFMM_ERR_STATE, "tree: leaves do not cover every particle"};
    }
    P->pos_f.alloc(6 * (size_t)n);
    HFMM_LAUNCH(k_split_pos, nblocks(3 * n), TPB, 0, 0, P->pos_s.p, 3 * n, P->pos_f.p);
    P->rmax.alloc(nb);
    HFMM_LAUNCH(k_rmax, nblocks(nb), TPB, 0, 0, pos_dev, P->pos_s.p, P->leaf_start.p, P->counts.p,
                n, nb, P->maxleaf, P->rmax.p);
    HFMM_CUDA(cudaDeviceSynchronize());
}

}  // namespace hfmm
