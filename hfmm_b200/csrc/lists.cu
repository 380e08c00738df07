// Device interaction lists: the B200 form of the eager block builders of
// jaxfmm/trees/lists.py (818-931) and the near-pair assembly of core.py:138-140.
//
// One thread per candidate (target, neighbour[, child]) evaluates the same
// predicate as the reference (_v_block lists.py:619-661, _ua_block 664-738,
// _wx_block 741-802); a prefix sum over the candidate flags then writes the
// compact pair arrays in the reference's row order:
//   V: (target, neighbour, child) over all targets;
//   U: per block of 262144 targets: same-level, then coarser, then finer;
//   W: (target, neighbour, child); X: (target, neighbour).
// Box lookups use the sorted (level << 3*max_depth | morton) ids of
// _sorted_boxids / _blk_lookup (lists.py:583-599).
//
// The evaluate schedules built here (CSR near lists, M2L/M2M source tables, tile
// lists) are this library's own layout and have no reference counterpart.
#include "hfmm_internal.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>

namespace hfmm {

namespace {

constexpr int TPB = 256;
constexpr int64_t UBLOCK = 262144;   // lists.py:563

inline int nblocks(int64_t n) { return (int)std::max<int64_t>(1, ceil_div(n, TPB)); }

struct BoxView {
    const uint64_t* m;
    const int32_t* lvl;
    const uint8_t* leaf;
    const uint64_t* skey;   // sorted box ids
    const int32_t* sidx;    // box index of each sorted id
    int64_t nb;
    int shift;              // 3 * max_depth
};

__device__ __forceinline__ int32_t lookup(const BoxView& v, uint64_t id) {
    int64_t lo = 0, hi = v.nb;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (v.skey[mid] < id) lo = mid + 1;
        else hi = mid;
    }
    return (lo < v.nb && v.skey[lo] == id) ? v.sidx[lo] : -1;
}

__device__ __forceinline__ bool is_leaf_box(const BoxView& v, int32_t b) {
    return b >= 0 && v.leaf[b] && v.lvl[b] > 0;
}

__global__ void k_box_ids(const uint64_t* m, const int32_t* lvl, int64_t nb, int shift,
                          uint64_t* ids, int32_t* idx) {
    int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= nb) return;
    ids[b] = ((uint64_t)lvl[b] << shift) | m[b];
    idx[b] = (int32_t)b;
}

// Neighbour of (x, y, z) at level `l` in direction d; false when outside the grid.
__device__ __forceinline__ bool neighbour(int64_t x, int64_t y, int64_t z, int l, int d,
                                          uint64_t& code) {
    if (l < 0) return false;
    int dx, dy, dz;
    neigh_offset(d, dx, dy, dz);
    int64_t g = 1ll << l;
    int64_t nx = x + dx, ny = y + dy, nz = z + dz;
    if (nx < 0 || ny < 0 || nz < 0 || nx >= g || ny >= g || nz >= g) return false;
    code = morton3(nx, ny, nz);
    return true;
}

// V candidate (t, d, c): child c of the parent's neighbour d (lists.py:619-661).
__global__ void k_v_flags(BoxView v, int32_t* flag, int32_t* src) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= v.nb * 208) return;
    int64_t t = i / 208;
    int d = (int)((i / 8) % 26), c = (int)(i % 8);
    int l = v.lvl[t];
    int32_t s = -1;
    uint64_t pm = v.m[t] >> 3, pn;
    int64_t px, py, pz;
    demorton3(pm, px, py, pz);
    if (l > 0 && neighbour(px, py, pz, max(l - 1, 0), d, pn)) {
        uint64_t cm = pn * 8 + (uint64_t)c;
        int32_t o = lookup(v, ((uint64_t)l << v.shift) | cm);
        if (o >= 0 && cm != v.m[t]) {
            int64_t tx, ty, tz, cx, cy, cz;
            demorton3(v.m[t], tx, ty, tz);
            demorton3(cm, cx, cy, cz);
            bool na = (cx - tx > 1) || (tx - cx > 1) || (cy - ty > 1) || (ty - cy > 1) ||
                      (cz - tz > 1) || (tz - cz > 1);
            if (na) s = o;
        }
    }
    flag[i] = s >= 0 ? 1 : 0;
    src[i] = s;
}

__device__ __forceinline__ bool adj_coarse(int64_t b, int64_t c) { return (b <= 2 * c + 2) && (2 * c <= b + 1); }
__device__ __forceinline__ bool adj_fine(int64_t b, int64_t f) { return (2 * b <= f + 1) && (f <= 2 * b + 2); }

// kind 0: same-level neighbour, 1: parent colleague (coarser), 2: colleague child (finer)
// mode 0: U predicate (lists.py:664-738); 1: X (coarser, non-adjacent); 2: W (finer, non-adjacent)
__device__ int32_t cross_candidate(const BoxView& v, int64_t t, int kind, int d, int c, int mode) {
    int l = v.lvl[t];
    bool leaf_t = v.leaf[t] && l > 0;
    int64_t bx, by, bz;
    demorton3(v.m[t], bx, by, bz);
    if (kind == 0) {   // same level
        uint64_t nm;
        if (!leaf_t || !neighbour(bx, by, bz, l, d, nm)) return -1;
        int32_t o = lookup(v, ((uint64_t)l << v.shift) | nm);
        return is_leaf_box(v, o) ? o : -1;
    }
    if (kind == 1) {   // coarser: parent's neighbours at level l-1
        if (l <= 1) return -1;
        if (mode == 0 && !leaf_t) return -1;
        uint64_t pn;
        int64_t px, py, pz;
        demorton3(v.m[t] >> 3, px, py, pz);
        if (!neighbour(px, py, pz, l - 1, d, pn)) return -1;
        int32_t o = lookup(v, ((uint64_t)(l - 1) << v.shift) | pn);
        if (!is_leaf_box(v, o)) return -1;
        int64_t cx, cy, cz;
        demorton3(pn, cx, cy, cz);
        bool adj = adj_coarse(bx, cx) && adj_coarse(by, cy) && adj_coarse(bz, cz);
        return (mode == 0 ? adj : !adj) ? o : -1;
    }
    // finer: children of same-level neighbours
    if (!leaf_t) return -1;
    uint64_t nm;
    if (!neighbour(bx, by, bz, l, d, nm)) return -1;
    uint64_t cm = nm * 8 + (uint64_t)c;
    int32_t o = lookup(v, ((uint64_t)(l + 1) << v.shift) | cm);
    if (o < 0) return -1;
    if (mode == 0 && !is_leaf_box(v, o)) return -1;
    int64_t fx, fy, fz;
    demorton3(cm, fx, fy, fz);
    bool adj = adj_fine(bx, fx) && adj_fine(by, fy) && adj_fine(bz, fz);
    return (mode == 0 ? adj : !adj) ? o : -1;
}

// U flags of one target block [lo, hi): segments S (B*26), C (B*26), F (B*208)
__global__ void k_u_flags(BoxView v, int64_t lo, int64_t B, int32_t* flag, int32_t* tgt,
                          int32_t* src) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= B * 260) return;
    int kind, d, c = 0;
    int64_t t;
    if (i < B * 26) {
        kind = 0;
        t = lo + i / 26;
        d = (int)(i % 26);
    } else if (i < B * 52) {
        kind = 1;
        int64_t j = i - B * 26;
        t = lo + j / 26;
        d = (int)(j % 26);
    } else {
        kind = 2;
        int64_t j = i - B * 52;
        t = lo + j / 208;
        d = (int)((j / 8) % 26);
        c = (int)(j % 8);
    }
    int32_t s = cross_candidate(v, t, kind, d, c, 0);
    flag[i] = s >= 0 ? 1 : 0;
    tgt[i] = (int32_t)t;
    src[i] = s;
}

__global__ void k_x_flags(BoxView v, int32_t* flag, int32_t* src) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= v.nb * 26) return;
    int32_t s = cross_candidate(v, i / 26, 1, (int)(i % 26), 0, 1);
    if (v.lvl[i / 26] <= 0) s = -1;
    flag[i] = s >= 0 ? 1 : 0;
    src[i] = s;
}

__global__ void k_w_flags(BoxView v, int32_t* flag, int32_t* src) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= v.nb * 208) return;
    int32_t s = cross_candidate(v, i / 208, 2, (int)((i / 8) % 26), (int)(i % 8), 2);
    flag[i] = s >= 0 ? 1 : 0;
    src[i] = s;
}

// scatter flagged candidates to (pos, 2) pairs; tgt given per candidate or as i / per
__global__ void k_scatter_pairs(const int32_t* __restrict__ flag, const int32_t* __restrict__ incl,
                                const int32_t* __restrict__ tgt, const int32_t* __restrict__ src,
                                int64_t n, int64_t per, int64_t base, int32_t* out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n || !flag[i]) return;
    int64_t o = base + incl[i] - 1;
    out[2 * o] = tgt ? tgt[i] : (int32_t)(i / per);
    out[2 * o + 1] = src[i];
}

__global__ void k_self_pairs(const int32_t* __restrict__ leaves, int64_t nl, int64_t base,
                             int32_t* out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nl) return;
    out[2 * (base + i)] = leaves[i];
    out[2 * (base + i) + 1] = leaves[i];
}

void scan(const int32_t* in, int32_t* out, int64_t n, DevBuf<uint8_t>& tmp) {
    size_t bytes = 0;
    HFMM_CUDA(cub::DeviceScan::InclusiveSum(nullptr, bytes, in, out, (int)n));
    if (bytes > tmp.n) tmp.alloc(bytes);
    HFMM_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, bytes, in, out, (int)n));
}

int64_t last_of(const int32_t* d, int64_t n) {
    if (n == 0) return 0;
    int32_t v;
    HFMM_CUDA(cudaMemcpy(&v, d + n - 1, 4, cudaMemcpyDeviceToHost));
    return v;
}

// ---------------------------------------------------------------- schedules
__global__ void k_m2l_src(const int32_t* __restrict__ V, int64_t nV, const uint64_t* __restrict__ m,
                          int32_t* tab, int* err) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nV) return;
    int32_t t = V[2 * i], s = V[2 * i + 1];
    int64_t tx, ty, tz, sx, sy, sz;
    demorton3(m[t], tx, ty, tz);
    demorton3(m[s], sx, sy, sz);
    int64_t dx = tx - sx + 3, dy = ty - sy + 3, dz = tz - sz + 3;
    if (dx < 0 || dx > 6 || dy < 0 || dy > 6 || dz < 0 || dz > 6) {
        atomicOr(err, ERRF_BOUNDS);
        return;
    }
    tab[(int64_t)t * M2L_ENTRIES + dx * 49 + dy * 7 + dz] = s;
}

__global__ void k_l2l_src(const int32_t* __restrict__ p_id, const int32_t* __restrict__ lvl,
                          const uint64_t* __restrict__ m, int64_t nb, int32_t* tab,
                          int32_t* m2m_tab) {
    int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= nb) return;
    if (lvl[b] >= 3) {
        int o = (int)(m[b] & 7ull);
        tab[b * M2L_ENTRIES + N_DISP + o] = p_id[b];
        m2m_tab[(int64_t)p_id[b] * 8 + o] = (int32_t)b;
    }
}

__global__ void k_fill(int32_t* p, int64_t n, int32_t v) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// CSR by target of a (len x 2) pair list; tgt_map maps a target box to its row (or -1).
void build_csr(const int32_t* pairs, int64_t np, const std::vector<int32_t>& h_pairs,
               std::vector<int32_t>& rows, std::vector<int32_t>& off, std::vector<int32_t>& src,
               int64_t nb) {
    std::vector<int32_t> cnt(nb, 0);
    for (int64_t i = 0; i < np; ++i) cnt[h_pairs[2 * i]]++;
    std::vector<int32_t> row_of(nb, -1);
    rows.clear();
    for (int64_t b = 0; b < nb; ++b)
        if (cnt[b]) {
            row_of[b] = (int32_t)rows.size();
            rows.push_back((int32_t)b);
        }
    off.assign(rows.size() + 1, 0);
    for (size_t r = 0; r < rows.size(); ++r) off[r + 1] = off[r] + cnt[rows[r]];
    src.assign(np, 0);
    std::vector<int32_t> fillp(off.begin(), off.end() - 1);
    for (int64_t i = 0; i < np; ++i) {   // stable: pair order within a target
        int32_t r = row_of[h_pairs[2 * i]];
        src[fillp[r]++] = h_pairs[2 * i + 1];
    }
    (void)pairs;
}

template <typename T>
void upload(DevBuf<T>& d, const std::vector<T>& h) {
    d.alloc(h.size());
    if (!h.empty()) HFMM_CUDA(cudaMemcpy(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
}

template <typename T>
void download(std::vector<T>& h, const DevBuf<T>& d, size_t n) {
    h.resize(n);
    if (n) HFMM_CUDA(cudaMemcpy(h.data(), d.p, n * sizeof(T), cudaMemcpyDeviceToHost));
}

}  // namespace

void lists_build(hfmm_plan* P) {
    const int64_t nb = P->nb;
    DevBuf<uint8_t> tmp;
    DevBuf<uint64_t> ids, sids;
    DevBuf<int32_t> idx, sidx;
    ids.alloc(nb);
    sids.alloc(nb);
    idx.alloc(nb);
    sidx.alloc(nb);
    int shift = 3 * P->md;
    HFMM_LAUNCH(k_box_ids, nblocks(nb), TPB, 0, 0, P->m_id.p, P->lvls.p, nb, shift, ids.p, idx.p);
    size_t bytes = 0;
    HFMM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, ids.p, sids.p, idx.p, sidx.p, (int)nb));
    tmp.alloc(bytes);
    HFMM_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, ids.p, sids.p, idx.p, sidx.p, (int)nb));
    BoxView v{P->m_id.p, P->lvls.p, P->is_leaf.p, sids.p, sidx.p, nb, shift};

    DevBuf<int32_t> flag, incl, src, tgt;
    // V
    {
        int64_t n = nb * 208;
        flag.alloc(n);
        incl.alloc(n);
        src.alloc(n);
        HFMM_LAUNCH(k_v_flags, nblocks(n), TPB, 0, 0, v, flag.p, src.p);
        scan(flag.p, incl.p, n, tmp);
        P->nV = last_of(incl.p, n);
        P->V.alloc(2 * P->nV);
        HFMM_LAUNCH(k_scatter_pairs, nblocks(n), TPB, 0, 0, flag.p, incl.p, (const int32_t*)nullptr,
                    src.p, n, (int64_t)208, (int64_t)0, P->V.p);
    }
    // U, block by block
    {
        std::vector<std::pair<int64_t, int64_t>> parts;
        std::vector<DevBuf<int32_t>*> bufs;
        int64_t total = 0;
        std::vector<int32_t> hU;
        for (int64_t lo = 0; lo < nb; lo += UBLOCK) {
            int64_t B = std::min<int64_t>(UBLOCK, nb - lo);
            int64_t n = B * 260;
            flag.alloc(n);
            incl.alloc(n);
            src.alloc(n);
            tgt.alloc(n);
            HFMM_LAUNCH(k_u_flags, nblocks(n), TPB, 0, 0, v, lo, B, flag.p, tgt.p, src.p);
            scan(flag.p, incl.p, n, tmp);
            int64_t cnt = last_of(incl.p, n);
            DevBuf<int32_t> part;
            part.alloc(2 * cnt);
            HFMM_LAUNCH(k_scatter_pairs, nblocks(n), TPB, 0, 0, flag.p, incl.p, tgt.p, src.p, n,
                        (int64_t)1, (int64_t)0, part.p);
            std::vector<int32_t> h;
            download(h, part, 2 * cnt);
            hU.insert(hU.end(), h.begin(), h.end());
            total += cnt;
        }
        P->nU = total;
        upload(P->U, hU);
    }
    // leaves and near pairs = U + self pairs (core.py:138-140)
    std::vector<int32_t> h_leaves;
    for (int64_t b = 0; b < nb; ++b)
        if (P->h_is_leaf[b] && P->h_lvls[b] > 0) h_leaves.push_back((int32_t)b);
    upload(P->leaves, h_leaves);
    P->nNear = P->nU + (int64_t)h_leaves.size();
    P->near.alloc(2 * P->nNear);
    if (P->nU) HFMM_CUDA(cudaMemcpy(P->near.p, P->U.p, P->nU * 8, cudaMemcpyDeviceToDevice));
    HFMM_LAUNCH(k_self_pairs, nblocks(h_leaves.size()), TPB, 0, 0, P->leaves.p,
                (int64_t)h_leaves.size(), P->nU, P->near.p);
    // W and X only for adaptive trees (core.py:129-136)
    P->nW = P->nX = 0;
    if (P->adaptive) {
        int64_t n = nb * 208;
        flag.alloc(n);
        incl.alloc(n);
        src.alloc(n);
        HFMM_LAUNCH(k_w_flags, nblocks(n), TPB, 0, 0, v, flag.p, src.p);
        scan(flag.p, incl.p, n, tmp);
        P->nW = last_of(incl.p, n);
        P->W.alloc(2 * P->nW);
        HFMM_LAUNCH(k_scatter_pairs, nblocks(n), TPB, 0, 0, flag.p, incl.p, (const int32_t*)nullptr,
                    src.p, n, (int64_t)208, (int64_t)0, P->W.p);
        n = nb * 26;
        flag.alloc(n);
        incl.alloc(n);
        src.alloc(n);
        HFMM_LAUNCH(k_x_flags, nblocks(n), TPB, 0, 0, v, flag.p, src.p);
        scan(flag.p, incl.p, n, tmp);
        P->nX = last_of(incl.p, n);
        P->X.alloc(2 * P->nX);
        HFMM_LAUNCH(k_scatter_pairs, nblocks(n), TPB, 0, 0, flag.p, incl.p, (const int32_t*)nullptr,
                    src.p, n, (int64_t)26, (int64_t)0, P->X.p);
    }
    HFMM_CUDA(cudaDeviceSynchronize());
}

void schedules_build(hfmm_plan* P) {
    const int64_t nb = P->nb;
    // near CSR over leaves (pair order kept within a target)
    std::vector<int32_t> h_near, h_W, h_X;
    download(h_near, P->near, 2 * P->nNear);
    {
        std::vector<int32_t> rows, off, src;
        build_csr(P->near.p, P->nNear, h_near, rows, off, src, nb);
        // rows must be exactly the leaves (each leaf has its self pair)
        std::vector<int32_t> h_leaves;
        download(h_leaves, P->leaves, P->leaves.n);
        if (rows.size() != (size_t)P->n_leaves) throw Error{HFMM_ERR_STATE, "near CSR rows != leaves"};
        upload(P->near_off, off);
        upload(P->near_src, src);
    }
    if (P->nW) {
        download(h_W, P->W, 2 * P->nW);
        std::vector<int32_t> rows, off, src;
        build_csr(P->W.p, P->nW, h_W, rows, off, src, nb);
        upload(P->w_tgt, rows);
        upload(P->w_off, off);
        upload(P->w_src, src);
        P->n_w_tgt = (int64_t)rows.size();
    }
    if (P->nX) {
        download(h_X, P->X, 2 * P->nX);
        std::vector<int32_t> rows, off, src;
        build_csr(P->X.p, P->nX, h_X, rows, off, src, nb);
        upload(P->x_tgt, rows);
        upload(P->x_off, off);
        upload(P->x_src, src);
        P->n_x_tgt = (int64_t)rows.size();
    }
    // dense source tables for the GEMM phases
    P->m2l_src.alloc(nb * M2L_ENTRIES);
    P->m2m_src.alloc(nb * 8);
    HFMM_LAUNCH(k_fill, nblocks(nb * M2L_ENTRIES), TPB, 0, 0, P->m2l_src.p, nb * M2L_ENTRIES, -1);
    HFMM_LAUNCH(k_fill, nblocks(nb * 8), TPB, 0, 0, P->m2m_src.p, nb * 8, -1);
    if (P->nV)
        HFMM_LAUNCH(k_m2l_src, nblocks(P->nV), TPB, 0, 0, P->V.p, P->nV, P->m_id.p, P->m2l_src.p,
                    P->d_err.p);
    HFMM_LAUNCH(k_l2l_src, nblocks(nb), TPB, 0, 0, P->p_id.p, P->lvls.p, P->m_id.p, nb,
                P->m2l_src.p, P->m2m_src.p);
    // tile lists: TT = 64 targets (R = 1) or 32 (R = 2)
    for (int l = 2; l <= P->md; ++l) {
        int lo = P->level_lo[l], hi = P->level_hi[l];
        for (int r = 0; r < 2; ++r) {
            int TT = 64 / (r + 1);
            auto make = [&](std::vector<int32_t> boxes, hfmm_plan::Tiles& T) {
                std::vector<int32_t> t;
                for (size_t i = 0; i < boxes.size(); i += TT)
                    for (int j = 0; j < TT; ++j)
                        t.push_back(i + j < boxes.size() ? boxes[i + j] : -1);
                T.ntiles = (int)(t.size() / TT);
                upload(T.tgt, t);
            };
            std::vector<int32_t> all, nonleaf, leaf;
            for (int b = lo; b < hi; ++b) {
                all.push_back(b);
                (P->h_is_leaf[b] ? leaf : nonleaf).push_back(b);
            }
            make(all, P->dec_tiles[l][r]);
            make(nonleaf, P->m2m_tiles[l][r]);
            make(leaf, P->leaf_tiles[l][r]);
            // downward tiles: grouped by octant so the 189 active displacements and
            // the L2L matrix coincide within a tile
            std::vector<int32_t> byoct;
            for (int o = 0; o < 8; ++o) {
                std::vector<int32_t> g;
                for (int b = lo; b < hi; ++b)
                    if ((int)(P->h_m_id[b] & 7ull) == o) g.push_back(b);
                for (size_t i = 0; i < g.size(); i += TT)
                    for (int j = 0; j < TT; ++j) byoct.push_back(i + j < g.size() ? g[i + j] : -1);
            }
            P->dn_tiles[l][r].ntiles = (int)(byoct.size() / TT);
            upload(P->dn_tiles[l][r].tgt, byoct);
            // mixed M2L tiles: 128 columns = 128 / R targets, same octant grouping, and
            // the octants' tiles interleaved (tile k of octant 0..7, then tile k + 1):
            // consecutive CTAs then cover a compact block of the level, so the source
            // densities a wave gathers stay in L2 (the finest low-rank M2L of 1M points
            // read 8.7 GB from DRAM in octant-major order, 2.05 GB interleaved)
            const int TTM = 128 / (r + 1);
            std::vector<int32_t> mx;
            std::vector<std::vector<int32_t>> per(8);
            for (int o = 0; o < 8; ++o) {
                std::vector<int32_t> g;
                for (int b = lo; b < hi; ++b)
                    if ((int)(P->h_m_id[b] & 7ull) == o) g.push_back(b);
                for (size_t i = 0; i < g.size(); i += TTM)
                    for (int j = 0; j < TTM; ++j) per[o].push_back(i + j < g.size() ? g[i + j] : -1);
            }
            size_t most = 0;
            for (auto& v : per) most = std::max(most, v.size() / TTM);
            for (size_t k = 0; k < most; ++k)
                for (int o = 0; o < 8; ++o)
                    if ((k + 1) * TTM <= per[o].size())
                        mx.insert(mx.end(), per[o].begin() + k * TTM, per[o].begin() + (k + 1) * TTM);
            P->mx_tiles[l][r].ntiles = (int)(mx.size() / TTM);
            upload(P->mx_tiles[l][r].tgt, mx);
        }
        // grid tiles of a complete level (every one of its 8^l boxes present), for the
        // mixed M2L with complex charges: 64 targets = one octant o of a 4 x 4 x 4 block
        // of parents, target j = (x * 4 + y) * 4 + z at grid position
        // org + 2 (x, y, z), org = 8 (block) + o; the octants' tiles interleaved as above
        P->gx_tiles[l].ntiles = 0;
        const int64_t G = (int64_t)1 << l;
        if (l >= 3 && l <= GRID_MAX_LEVEL && (int64_t)(hi - lo) == G * G * G) {
            std::vector<int32_t> at((size_t)(G * G * G), -1);   // grid position -> box
            bool fits = true;
            for (int b = lo; b < hi && fits; ++b) {
                int64_t x, y, z;
                demorton3(P->h_m_id[b], x, y, z);
                if (x < 0 || y < 0 || z < 0 || x >= G || y >= G || z >= G ||
                    at[(size_t)((x * G + y) * G + z)] >= 0)
                    fits = false;   // not one box per grid cell: keep the gather
                else
                    at[(size_t)((x * G + y) * G + z)] = b;
            }
            if (!fits) continue;
            const int64_t nc = (G / 2 + 3) / 4;   // parent blocks per axis
            std::vector<int32_t> tg, org;
            for (int64_t c = 0; c < nc * nc * nc; ++c)
                for (int o = 0; o < 8; ++o) {
                    const int64_t ox = 8 * (c / (nc * nc)) + (o & 1);
                    const int64_t oy = 8 * ((c / nc) % nc) + ((o >> 1) & 1);
                    const int64_t oz = 8 * (c % nc) + ((o >> 2) & 1);
                    org.push_back((int32_t)ox);
                    org.push_back((int32_t)oy);
                    org.push_back((int32_t)oz);
                    for (int j = 0; j < 64; ++j) {
                        const int64_t x = ox + 2 * (j / 16), y = oy + 2 * ((j / 4) % 4), z = oz + 2 * (j % 4);
                        tg.push_back(x < G && y < G && z < G ? at[(size_t)((x * G + y) * G + z)] : -1);
                    }
                }
            P->gx_tiles[l].ntiles = (int)(tg.size() / 64);
            upload(P->gx_tiles[l].tgt, tg);
            upload(P->gx_org[l], org);
        }
    }
    HFMM_CUDA(cudaDeviceSynchronize());
}

}  // namespace hfmm
