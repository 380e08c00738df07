// C ABI of hfmm_b200 (include/hfmm_b200.h): plan life cycle, operator-table
// upload, schedules and the evaluate driver.
//
// The evaluate driver follows core.evaluate (jaxfmm/core.py:274-335) with the
// leveled KIFMM closures (kifmm/assemble.py:15-89):
//   S2M  P2M check potentials + level decode          (phases.py:79-125)
//   M2M  child -> parent check + decode, bottom-up     (phases.py:128-173)
//   M2L  V-list check, fused with P2L and L2L, decode  (phases.py:176-280, 1709-1770)
//   L2P  + near field P2P + W-list M2P                 (phases.py:1533-1582, near.py:48-312,
//                                                        phases.py:1064-1140)
// Both Helmholtz components (cos, sin) and the R charge columns run together.
// Levels 0 and 1 carry no far-field work: V, W and X pairs start at level 2, so
// their equivalent and local densities are never read.
#include "hfmm_internal.cuh"
#include "particles.cuh"
#include "mixed.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <memory>
#include <mutex>

namespace hfmm {

std::atomic<int64_t> g_launches{0};
static thread_local std::string t_last_error;

void set_error(int code, const std::string& msg) {
    (void)code;
    t_last_error = msg;
}
int fail(int code, const std::string& msg) {
    set_error(code, msg);
    return code;
}

namespace {

// dst[c][k][m] = (transpose ? src[map[c]][m][k] : src[map[c]][k][m]), zero padded to ld
__global__ void k_relayout(const double* __restrict__ src, const int32_t* __restrict__ map,
                           int count, int n_s, int ld, int transpose, double* dst) {
    __shared__ double tile[32][33];
    const int c = blockIdx.z;
    const int sc = map ? map[c] : c;
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;   // bx: m (dst column), by: k (dst row)
    const double* S = src + (int64_t)sc * n_s * n_s;
    double* D = dst + (int64_t)c * ld * ld;
    if (!transpose) {
        for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
            int k = by + yy, m = bx + threadIdx.x;
            tile[yy][threadIdx.x] = (k < n_s && m < n_s) ? S[(int64_t)k * n_s + m] : 0.0;
        }
    } else {
        // read S[m][k] coalesced along k: rows m = bx + yy, cols k = by + tx
        for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
            int m = bx + yy, k = by + threadIdx.x;
            tile[threadIdx.x][yy] = (m < n_s && k < n_s) ? S[(int64_t)m * n_s + k] : 0.0;
        }
    }
    __syncthreads();
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        int k = by + yy, m = bx + threadIdx.x;
        if (k < ld && m < ld) D[(int64_t)k * ld + m] = tile[yy][threadIdx.x];
    }
}

void relayout(const double* h_src, int src_count, const std::vector<int32_t>& map, int n_s,
              int ld, bool transpose, DevBuf<double>& dst) {
    int count = map.empty() ? src_count : (int)map.size();
    dst.alloc((size_t)count * ld * ld);
    DevBuf<double> staging;
    staging.alloc((size_t)src_count * n_s * n_s);
    HFMM_CUDA(cudaMemcpy(staging.p, h_src, (size_t)src_count * n_s * n_s * sizeof(double),
                         cudaMemcpyHostToDevice));
    DevBuf<int32_t> dmap;
    if (!map.empty()) {
        dmap.alloc(map.size());
        HFMM_CUDA(cudaMemcpy(dmap.p, map.data(), map.size() * 4, cudaMemcpyHostToDevice));
    }
    dim3 grid((unsigned)ceil_div(ld, 32), (unsigned)ceil_div(ld, 32), (unsigned)count);
    HFMM_LAUNCH(k_relayout, grid, dim3(32, 8), 0, 0, staging.p, map.empty() ? nullptr : dmap.p,
                count, n_s, ld, transpose ? 1 : 0, dst.p);
    HFMM_CUDA(cudaDeviceSynchronize());
}

void upload_vec(const double* h, int n_s, int ld, DevBuf<double>& dst) {
    std::vector<double> v(ld, 0.0);
    std::memcpy(v.data(), h, n_s * sizeof(double));
    dst.alloc(ld);
    HFMM_CUDA(cudaMemcpy(dst.p, v.data(), ld * sizeof(double), cudaMemcpyHostToDevice));
}

std::vector<int32_t> nonadjacent_map() {
    std::vector<int32_t> m;
    for (int d = 0; d < N_DISP; ++d) {
        int dx = d / 49 - 3, dy = (d / 7) % 7 - 3, dz = d % 7 - 3;
        if (std::max(std::abs(dx), std::max(std::abs(dy), std::abs(dz))) > 1) m.push_back(d);
    }
    return m;
}

// A-pointer sets of the GEMM calls: kind 0..3 decode (up U, up Vt, dn U, dn Vt),
// kind 4 M2M (8 entries), kind 5 downward M2L+L2L (351 entries), kind 6 L2L alone,
// kinds 7/8 compress / expand of the compressed M2L; per level, families adjacent.
enum { K_UPU, K_UPV, K_DNU, K_DNV, K_M2M, K_DN, K_L2L, K_CMP, K_EXP, K_M2MF, K_L2LF, K_COUNT };
const int k_entries[K_COUNT] = {1, 1, 1, 1, 8, M2L_ENTRIES, 8, 1, 1, 8, 8};

struct PtrIndex {
    size_t off[K_COUNT][MAX_LEVELS];
};

void build_a_ptrs(hfmm_plan* P, PtrIndex& ix) {
    std::vector<const double*> h;
    const size_t mat = (size_t)P->ld * P->ld;
    auto madj = nonadjacent_map();
    std::vector<int32_t> compact(N_DISP, -1);
    for (size_t i = 0; i < madj.size(); ++i) compact[madj[i]] = (int32_t)i;
    for (int kind = 0; kind < K_COUNT; ++kind)
        for (int l = 0; l < MAX_LEVELS; ++l) {
            ix.off[kind][l] = h.size();
            if (l < 2 || l > P->md) continue;
            for (int f = 0; f < P->n_fam; ++f) {
                LevelTables& T = P->tables[f][l];
                switch (kind) {
                    case K_UPU: h.push_back(T.up_U.p); break;
                    case K_UPV: h.push_back(T.up_Vt.p); break;
                    case K_DNU: h.push_back(T.dn_U.p); break;
                    case K_DNV: h.push_back(T.dn_Vt.p); break;
                    case K_M2M:
                        for (int o = 0; o < 8; ++o) h.push_back(T.m2m.p ? T.m2m.p + o * mat : nullptr);
                        break;
                    case K_DN: {
                        const double* m2l = P->streamed
                            ? static_cast<const double*>(P->ws) + (size_t)f * 316 * mat : T.m2l.p;
                        for (int d = 0; d < N_DISP; ++d)
                            h.push_back(compact[d] >= 0 && m2l ? m2l + compact[d] * mat : nullptr);
                        for (int o = 0; o < 8; ++o) h.push_back(T.l2l.p ? T.l2l.p + o * mat : nullptr);
                        break;
                    }
                    case K_L2L:
                        for (int o = 0; o < 8; ++o) h.push_back(T.l2l.p ? T.l2l.p + o * mat : nullptr);
                        break;
                    case K_CMP: h.push_back(T.cmp_f.p); break;   // folded (compress.cu)
                    case K_EXP: h.push_back(T.exp_f.p); break;
                    case K_M2MF:
                        for (int o = 0; o < 8; ++o) h.push_back(T.m2m_f.p ? T.m2m_f.p + o * mat : nullptr);
                        break;
                    case K_L2LF:
                        for (int o = 0; o < 8; ++o) h.push_back(T.l2l_f.p ? T.l2l_f.p + o * mat : nullptr);
                        break;
                }
            }
        }
    P->h_a_ptrs = h;
    P->a_ptrs.alloc(h.size());
    HFMM_CUDA(cudaMemcpy(P->a_ptrs.p, h.data(), h.size() * sizeof(void*), cudaMemcpyHostToDevice));
}

EvalView view(hfmm_plan* P) {
    EvalView v;
    v.n = P->n;
    v.nb = P->nb;
    v.n_s = P->n_s;
    v.ld = P->ld;
    v.k = P->k;
    v.yukawa = P->yukawa ? 1 : 0;
    v.pos_s = P->pos_s.p;
    v.pos_f = P->pos_f.p;
    v.q_s = P->q_s.p;
    v.leaf_start = P->leaf_start.p;
    v.counts = P->counts.p;
    v.lvls = P->lvls.p;
    v.centre = P->centre.p;
    v.hbox = P->hbox.p;
    v.rmax = P->rmax.p;
    return v;
}

struct PlanExtra {
    PtrIndex ix;
    bool profiling = false;
    std::vector<cudaEvent_t> ev;     // pairs (start, end)
    std::vector<int> ev_phase;
    size_t used = 0;
    ~PlanExtra() {
        for (auto e : ev) cudaEventDestroy(e);
    }
};

// Records a start/end event pair around one phase instance when profiling is on.
struct PhaseTimer {
    PlanExtra* X;
    cudaStream_t s;
    size_t slot = (size_t)-1;
    PhaseTimer(PlanExtra* x, cudaStream_t st, int phase) : X(x), s(st) {
        if (!X || !X->profiling || X->used >= X->ev_phase.size()) return;
        slot = X->used++;
        X->ev_phase[slot] = phase;
        HFMM_CUDA(cudaEventRecord(X->ev[2 * slot], s));
    }
    ~PhaseTimer() {
        if (slot != (size_t)-1) cudaEventRecord(X->ev[2 * slot + 1], s);
    }
};

std::mutex g_extra_mu;
std::vector<std::pair<hfmm_plan*, PlanExtra*>> g_extra;

PlanExtra* extra(hfmm_plan* P, bool create) {
    std::lock_guard<std::mutex> g(g_extra_mu);
    for (auto& e : g_extra)
        if (e.first == P) return e.second;
    if (!create) return nullptr;
    g_extra.push_back({P, new PlanExtra()});
    return g_extra.back().second;
}

void drop_extra(hfmm_plan* P) {
    std::lock_guard<std::mutex> g(g_extra_mu);
    for (size_t i = 0; i < g_extra.size(); ++i)
        if (g_extra[i].first == P) {
            delete g_extra[i].second;
            g_extra.erase(g_extra.begin() + i);
            return;
        }
}

}  // namespace

void upload_level(hfmm_plan* P, int fam, int l, const double* const* h) {
    LevelTables& T = P->tables[fam][l];
    const int n_s = P->n_s, ld = P->ld;
    std::vector<int32_t> none;
    relayout(h[0], 1, none, n_s, ld, false, T.up_U);   // A = U^T  -> A^T = U
    upload_vec(h[1], n_s, ld, T.up_d);
    relayout(h[2], 1, none, n_s, ld, false, T.up_Vt);  // A = Vt^T -> A^T = Vt
    relayout(h[3], 1, none, n_s, ld, false, T.dn_U);
    upload_vec(h[4], n_s, ld, T.dn_d);
    relayout(h[5], 1, none, n_s, ld, false, T.dn_Vt);
    if (P->streamed && h[8])
        throw Error{HFMM_ERR_STATE, "streamed M2L tables are generated on the device: pass no M2L table"};
    if (!h[8]) {   // kernel matrices generated on the device
        generate_tables(P, fam, l);
        T.set = true;
        return;
    }
    if (h[6] && l < P->md) relayout(h[6], 8, none, n_s, ld, true, T.m2m);
    else T.m2m.release();
    if (h[7] && l >= 3) relayout(h[7], 8, none, n_s, ld, true, T.l2l);
    else T.l2l.release();
    relayout(h[8], N_DISP, nonadjacent_map(), n_s, ld, true, T.m2l);
    T.set = true;
}

// Tensor maps of the streamed TF32 tables: every level reads the same workspace
// (hi halves of both families, then the lo halves; [fam][316][m][k] each).
void stream_maps(hfmm_plan* P) {
    if (!P->mx_maps) P->mx_maps = new MixedMaps[MAX_LEVELS];
    MixedMaps* maps = static_cast<MixedMaps*>(P->mx_maps);
    std::memset(maps, 0, sizeof(MixedMaps) * MAX_LEVELS);
    const size_t fam = (size_t)316 * P->ld * P->ld;
    const float* hi = static_cast<const float*>(P->ws);
    const float* lo = hi + (size_t)P->n_fam * fam;
    for (int l = 2; l <= P->md; ++l)
        for (int f = 0; f < P->n_fam; ++f) {
            make_table_map(&maps[l].a_hi[f], hi + f * fam, P->ld, 316);
            make_table_map(&maps[l].a_lo[f], lo + f * fam, P->ld, 316);
        }
}

// The low-rank mixed M2L of one level and family (R charge columns): the call of
// m2l_tf32x3 / one entry of the batch's M2L queue.
MixedCall cx_call(hfmm_plan* P, int l, int f, int R) {
    LevelTables& T = P->tables[f][l];
    auto lb = [&](auto* buf, int cld) { return buf - (int64_t)P->level_lo[l] * R * cld; };
    MixedCall mc{};
    mc.tile_tgt = P->mx_tiles[l][R - 1].tgt.p;
    mc.ntiles = P->mx_tiles[l][R - 1].ntiles;
    mc.src_tab = P->m2l_src.p;
    mc.disp_compact = P->disp_compact.p;
    mc.Bhi = lb(T.xc_hi.p, T.ckld);
    mc.Blo = lb(T.xc_lo.p, T.ckld);
    mc.Lhi = nullptr;
    mc.Llo = nullptr;
    mc.out = lb(T.yc.p, T.cmld);
    mc.src_lo = P->level_lo[l];   // the level's buffers hold its own boxes only
    mc.src_hi = P->level_hi[l];
    mc.R = R;
    mc.ld = T.cmld;
    mc.ldk = T.ckld;
    mc.ldm = T.cmld;
    mc.m_valid = T.cr;   // rows r..cmld of the C_d tables are zero
    mc.n_fam = 1;
    mc.has_l2l = 0;
    mc.fam_stride = 0;
    mc.out_fam_stride = 0;
    mc.nb = P->nb;
    mc.err = P->d_err.p;
    if (R == 2 && T.grid && g_m2l_grid.load()) {   // sources from the dense grid by TMA
        mc.grid = 1;
        mc.tile_tgt = P->gx_tiles[l].tgt.p;
        mc.ntiles = P->gx_tiles[l].ntiles;
        mc.tile_org = P->gx_org[l].p;
    }
    return mc;
}

std::string queue_items(hfmm_plan* const* plans, int n_plans, int R, std::vector<MixedCall>& calls,
                        std::vector<MixedMaps>& maps, std::vector<M2LItem>& items) {
    struct Keyed {
        double cost;
        M2LItem it;
    };
    std::vector<Keyed> list;
    calls.clear();
    maps.clear();
    items.clear();
    for (int i = 0; i < n_plans; ++i) {
        hfmm_plan* P = plans[i];
        for (int l = 2; l <= P->md; ++l)
            for (int f = 0; f < P->n_fam; ++f) {
                MixedCall c = cx_call(P, l, f, R);
                if (c.ntiles == 0) continue;
                c.wait_ns = 0;
                c.starve = 0;
                if ((int64_t)c.nb * R * c.ldk >= ((int64_t)1 << 31))
                    return "a level's densities exceed 32-bit gather offsets";
                const int id = (int)calls.size();
                calls.push_back(c);
                maps.push_back(static_cast<MixedMaps*>(P->cx_maps)[f * MAX_LEVELS + l]);
                const int blocks = (c.ldm + 127) / 128;
                const int valid = c.m_valid > 0 ? c.m_valid : c.ldm;
                for (int t = 0; t < c.ntiles; ++t)
                    for (int b = 0; b < blocks; ++b) {
                        const double cost = (double)(c.ldk / 32) * (valid - 128 * b <= 64 ? 0.6 : 1.0);
                        list.push_back({cost, M2LItem{id, t, b}});
                    }
            }
    }
    if (list.empty()) return "no M2L work";
    std::stable_sort(list.begin(), list.end(), [](const Keyed& a, const Keyed& b) { return a.cost > b.cost; });
    for (auto& k : list) items.push_back(k.it);
    return "";
}

void plan_queue_release(hfmm_plan* P) {
    for (auto*& q : P->cxq) {
        delete static_cast<PlanQueue*>(q);
        q = nullptr;
    }
}

void plan_queue_build(hfmm_plan* P) {
    plan_queue_release(P);
    if (!P->compressed || !P->mixed_ready) return;
    for (int R = 1; R <= 2; ++R) {
        std::vector<MixedCall> calls;
        std::vector<MixedMaps> maps;
        std::vector<M2LItem> items;
        if (!queue_items(&P, 1, R, calls, maps, items).empty()) continue;
        auto* q = new PlanQueue;
        P->cxq[R - 1] = q;
        q->calls.alloc(calls.size());
        q->maps.alloc(maps.size());
        q->items.alloc(items.size());
        q->next.alloc(1);
        HFMM_CUDA(cudaMemcpy(q->calls.p, calls.data(), calls.size() * sizeof(MixedCall), cudaMemcpyHostToDevice));
        HFMM_CUDA(cudaMemcpy(q->maps.p, maps.data(), maps.size() * sizeof(MixedMaps), cudaMemcpyHostToDevice));
        HFMM_CUDA(cudaMemcpy(q->items.p, items.data(), items.size() * sizeof(M2LItem), cudaMemcpyHostToDevice));
        q->n_items = (int)items.size();
    }
}

namespace {
// The far-field chain (every phase but the near field) runs on the plan's own stream of
// the highest priority, forked from the caller's stream and joined back on every exit:
// the block scheduler then serves the chain first and the near field, on its default-
// priority side stream, fills the SMs the chain leaves free.
struct CritStream {
    cudaStream_t caller, s;
    hfmm_plan* P;
    CritStream(hfmm_plan* p, cudaStream_t c) : caller(c), s(c), P(p) {
        if (!P->crit) return;
        HFMM_CUDA(cudaEventRecord(P->crit_fork, caller));
        HFMM_CUDA(cudaStreamWaitEvent(P->crit, P->crit_fork, 0));
        s = P->crit;
    }
    ~CritStream() {
        if (s == caller) return;
        cudaEventRecord(P->crit_join, s);
        cudaStreamWaitEvent(caller, P->crit_join, 0);
    }
};
}  // namespace

// On an error part-way through an evaluate, the side streams may still run work that
// was enqueued before it (the near field writes the outputs, the compressed M2Ls the
// local expansions). While the exception unwinds, the far-field stream waits for all
// of it, and CritStream's join then carries that wait to the caller's stream: no
// kernel of the call outlives its error return on the caller's stream.
struct SideJoin {
    hfmm_plan* P;
    cudaStream_t s;
    int unwinding;
    SideJoin(hfmm_plan* p, cudaStream_t st) : P(p), s(st), unwinding(std::uncaught_exceptions()) {}
    ~SideJoin() {
        if (std::uncaught_exceptions() <= unwinding) return;
        auto join = [&](cudaStream_t side, cudaEvent_t ev) {
            if (side && ev && side != s && cudaEventRecord(ev, side) == cudaSuccess)
                cudaStreamWaitEvent(s, ev, 0);
        };
        join(P->nf_side, P->nf_join);
        for (int k = 0; k < hfmm_plan::CX_STREAMS; ++k) join(P->cx_side[k], P->cx_join[k]);
    }
};

void evaluate_fp64(hfmm_plan* P, const double* q_re, const double* q_im, double* phi, double* E,
                   cudaStream_t s_caller, bool mixed, int phase) {
    const bool up = phase & EVAL_UP, down = phase & EVAL_DOWN;
    if (down && P->rot_P > 0 && !(mixed && P->mixed_ready))
        rot_check(P);   // before anything is enqueued
    CritStream crit(P, s_caller);
    cudaStream_t s = crit.s;
    SideJoin side_join(P, s);   // destroyed before crit: the sides join s, then s the caller
    const int R = q_im ? 2 : 1;
    const int NF = P->n_fam;
    const bool field = E != nullptr;
    PlanExtra* X = extra(P, false);
    const int64_t fs = P->nb * (int64_t)R * P->ld;   // family stride of expansion arrays
    if (up) {
        PhaseTimer pt(X, s, 0);
        gather_charges(P->n, P->sort_idx.p, q_re, q_im, P->q_s.p, s);
    }
    EvalView v = view(P);

    // Particle phases. On the mixed path only the near field runs in FP32: P2M and P2L
    // feed the damped decodes and L2P/M2P read their output; for the sin component
    // (eps_rel 1e-12) FP32 noise there is amplified along near-null singular
    // directions, so those phases stay FP64.
    auto particles = [&](const ParticlePass& p, cudaStream_t st) {
        if (mixed && p.op == ParticleOp::P2P) particles_mixed(p, st);
        else particles_f64(p, st);
    };
    ParticlePass base;
    base.v = v;
    base.nf = NF;
    base.R = R;
    base.field = field;
    base.fam_stride = fs;
    base.pot = P->pot.p;
    base.fld = P->fld.p;

    // The near field needs only the gathered charges: it runs on the plan's side
    // stream beside the whole far field and joins before L2P, which adds into the
    // potentials and fields P2P stores. It is enqueued after P2M (below), so that the
    // far field's first kernel takes the SMs first.
    if (up) HFMM_CUDA(cudaEventRecord(P->nf_fork, s));
    auto launch_near_field = [&]() {
        HFMM_CUDA(cudaStreamWaitEvent(P->nf_side, P->nf_fork, 0));
        ParticlePass p = base;
        p.op = ParticleOp::P2P;
        p.rows = P->leaves.p;
        p.nrows = P->n_leaves;
        p.off = P->near_off.p;
        p.srcs = P->near_src.p;
        {
            PhaseTimer pt(X, P->nf_side, 7);
            particles(p, P->nf_side);
        }
        HFMM_CUDA(cudaEventRecord(P->nf_join, P->nf_side));
    };

    // scale_up / scale_dn: multiply row m of family f's result by the level's decode
    // scale d (the folded low-rank plan's GEMMs end in scaled SVD coordinates)
    enum { NO_SCALE, SCALE_UP, SCALE_DN };
    auto gemm = [&](int kind, int l, const hfmm_plan::Tiles& tiles, const int32_t* src_tab,
                    int src_ld, const double* B0, const double* B1, double* out,
                    int scale_kind = NO_SCALE, int accumulate = -1) {
        const int phase = (kind == K_M2M || kind == K_M2MF) ? 2
                          : kind == K_DN                    ? 4
                          : (kind == K_L2L || kind == K_L2LF) ? 13
                          : kind <= K_UPV                   ? 3
                                                            : 6;
        PhaseTimer pt(X, s, phase);
        GemmCall c{};
        c.tile_tgt = tiles.tgt.p;
        c.ntiles = tiles.ntiles;
        c.src_tab = src_tab;
        c.src_ld = src_ld;
        c.n_entries = k_entries[kind];
        c.b_split = kind == K_DN ? N_DISP : c.n_entries;
        c.accumulate = accumulate >= 0 ? accumulate : (kind == K_L2L ? 1 : 0);
        c.A = P->a_ptrs.p + X->ix.off[kind][l];
        c.B0 = B0;
        c.B1 = B1;
        c.out = out;
        if (scale_kind != NO_SCALE) {
            auto pick = [&](int f) {
                return scale_kind == SCALE_UP ? P->tables[f][l].up_d.p : P->tables[f][l].dn_d.p;
            };
            c.scale = pick(0);
            c.scale_f1 = NF > 1 ? pick(1) : nullptr;
        }
        c.R = R;
        c.ld = P->ld;
        c.n_s = P->n_s;
        c.k_valid = P->n_s;   // every table's rows past n_s are zero
        c.fam_stride = fs;
        c.a_fam_stride = k_entries[kind];
        c.n_fam = NF;
        c.nb = P->nb;
        c.part = P->gemm_part.p;   // coarse levels' small grids split their entries
        c.part_cap = P->gemm_part.n;
        gemm_f64(c, P->d_err.p, s);
    };
    // The decode scale vector differs per family: run the first decode step once per family.
    auto decode = [&](int l, bool up, const double* in, double* out) {
        const hfmm_plan::Tiles& tiles = P->dec_tiles[l][R - 1];
        for (int f = 0; f < NF; ++f) {
            PhaseTimer pt(X, s, up ? 3 : 6);
            GemmCall c{};
            c.tile_tgt = tiles.tgt.p;
            c.ntiles = tiles.ntiles;
            c.src_tab = nullptr;
            c.src_ld = 0;
            c.n_entries = 1;
            c.b_split = 1;
            c.A = P->a_ptrs.p + X->ix.off[up ? K_UPU : K_DNU][l] + f;
            c.B0 = in + f * fs;
            c.B1 = nullptr;
            c.out = P->tmp.p + f * fs;
            c.scale = up ? P->tables[f][l].up_d.p : P->tables[f][l].dn_d.p;
            c.accumulate = 0;
            c.R = R;
            c.ld = P->ld;
            c.n_s = P->n_s;
            c.k_valid = P->n_s;
            c.fam_stride = 0;
            c.a_fam_stride = 0;
            c.n_fam = 1;
            c.nb = P->nb;
            gemm_f64(c, P->d_err.p, s);
        }
        gemm(up ? K_UPV : K_DNV, l, tiles, nullptr, 0, P->tmp.p, nullptr, out);
    };

    // ---- upward pass
    const bool use_mx = mixed && P->mixed_ready;
    const bool use_cx = use_mx && P->compressed;
    if (up) {
        ParticlePass p = base;
        p.op = ParticleOp::P2M;
        p.rows = P->leaves.p;
        p.nrows = P->n_leaves;
        p.surf = P->check_pts.p;
        p.out = P->check.p;
        {
            PhaseTimer pt(X, s, 1);
            particles(p, s);
        }
        launch_near_field();
    }
    if (!up) {
    } else if (use_cx) {
        // folded tables (compress.cu): P->equiv holds y = d .* (U^T x) per box, from the
        // leaf check potentials (U, leaves) or the children's y (folded M2M, the rest)
        for (int l = P->md; l >= 2; --l) {
            gemm(K_UPU, l, P->leaf_tiles[l][R - 1], nullptr, 0, P->check.p, nullptr, P->equiv.p,
                 SCALE_UP);
            if (l < P->md)
                gemm(K_M2MF, l, P->m2m_tiles[l][R - 1], P->m2m_src.p, 8, P->equiv.p, nullptr,
                     P->equiv.p, SCALE_UP);
            if (P->nW)   // the W list's M2P reads the equivalent densities themselves
                gemm(K_UPV, l, P->dec_tiles[l][R - 1], nullptr, 0, P->equiv.p, nullptr, P->tmp.p);
        }
    } else {
        for (int l = P->md; l >= 2; --l) {
            if (l < P->md)
                gemm(K_M2M, l, P->m2m_tiles[l][R - 1], P->m2m_src.p, 8, P->equiv.p, nullptr,
                     P->check.p);
            decode(l, true, P->check.p, P->equiv.p);
        }
    }
    // A level's compressed buffers hold [box - level_lo][R][cld]; the GEMMs index boxes
    // absolutely, so they get the buffer's address shifted back by level_lo rows.
    auto level_base = [&](auto* buf, int l, int cld) {
        return buf - (int64_t)P->level_lo[l] * R * cld;
    };
    // one-entry GEMM over every box of level l between layouts of different widths
    auto gemm_1 = [&](int kind, int l, int f, const double* in, int ldk, double* out, int ldm,
                      cudaStream_t st, const double* scale = nullptr) {
        GemmCall c{};
        c.scale = scale;
        c.k_valid = kind == K_EXP ? P->tables[f][l].cr : P->n_s;   // compress reads y (n_s)
        c.tile_tgt = P->dec_tiles[l][R - 1].tgt.p;
        c.ntiles = P->dec_tiles[l][R - 1].ntiles;
        c.src_tab = nullptr;
        c.n_entries = 1;
        c.b_split = 1;
        c.A = P->a_ptrs.p + X->ix.off[kind][l] + f;
        c.B0 = in;
        c.out = out;
        c.accumulate = 0;
        c.R = R;
        c.ld = P->ld;
        c.ldk = ldk;
        c.ldm = ldm;
        c.n_s = P->n_s;
        c.n_fam = 1;
        c.nb = P->nb;
        gemm_f64(c, P->d_err.p, st);
    };
    if (up && use_cx) {   // compress every level's densities (x' = y Vt_up U_c), then split them
        PhaseTimer pt(X, s, 14);
        for (int l = 2; l <= P->md; ++l)
            for (int f = 0; f < NF; ++f) {
                LevelTables& T = P->tables[f][l];
                gemm_1(K_CMP, l, f, P->equiv.p + f * fs, P->ld, level_base(T.xc.p, l, T.ckld), T.ckld,
                       s);
                const int64_t nbl = P->level_hi[l] - P->level_lo[l];
                if (R == 2 && T.grid && g_m2l_grid.load())   // complete level: into the dense grid
                    split_tf32_grid(T.xc.p, P->m_id.p + P->level_lo[l], nbl, T.grid, T.ckld,
                                    T.xg_hi.p, T.xg_lo.p, s);
                else
                    split_tf32(T.xc.p, T.xc_hi.p, T.xc_lo.p, nbl * R * T.ckld, s);
            }
    } else if (up && use_mx) {   // TF32 hi/lo halves of every equivalent density (B operand)
        PhaseTimer pt(X, s, 11);
        split_tf32(P->equiv.p, P->e_hi.p, P->e_lo.p, (int64_t)NF * fs, s);
    }
    // split evaluate (a batch's queued M2L): the upward half ends here; the downward half
    // starts with every level's expansion of the queue's check potentials
    if (!down) return;
    if (!up && use_cx) {
        for (int l = 2; l <= P->md; ++l)
            for (int f = 0; f < NF; ++f) {
                LevelTables& T = P->tables[f][l];
                PhaseTimer pt(X, s, 14);
                gemm_1(K_EXP, l, f, level_base(T.yc.p, l, T.cmld), T.cmld, P->loc.p + f * fs, P->ld,
                       s, T.dn_d.p);
            }
    }
    // The plan's own queued M2L (every level and family in one persistent launch, the
    // largest items first) in place of the per-level launches on side streams; the test
    // switches of the M2L kernels (grid mode off) take the per-level path.
    PlanQueue* pq = (up && use_cx && g_m2l_grid.load() && P->queue_m2l) ? static_cast<PlanQueue*>(P->cxq[R - 1])
                                                                 : nullptr;
    if (pq) {
        {
            PhaseTimer pt(X, s, 4);
            m2l_queue(pq->calls.p, pq->maps.p, pq->items.p, pq->n_items, pq->next.p, R, sm_count(), s,
                      g_m2l_starve.load());
        }
        for (int l = 2; l <= P->md; ++l)
            for (int f = 0; f < NF; ++f) {
                LevelTables& T = P->tables[f][l];
                PhaseTimer pt(X, s, 14);
                gemm_1(K_EXP, l, f, level_base(T.yc.p, l, T.cmld), T.cmld, P->loc.p + f * fs, P->ld,
                       s, T.dn_d.p);
            }
    }
    const bool cx_side = up && use_cx && !pq;   // the per-level M2L launches on side streams
    std::unique_ptr<PhaseTimer> m2l_timer;
    if (cx_side) {
        // A level's M2L reads only the compressed densities of the upward pass, so the
        // M2Ls of every level and family run at once on the plan's side streams (the
        // coarse levels have a handful of tiles each and would otherwise run alone on
        // a few SMs); each expands into its own level's check potentials. The finest
        // level takes streams 0 and 1; the coarse levels queue on streams 2 and 3,
        // coarsest first, so the downward chain below can start on them while the
        // finest level's M2L still runs: it waits for each level's events in turn.
        m2l_timer.reset(new PhaseTimer(X, s, 4));   // until the finest level has joined
        HFMM_CUDA(cudaEventRecord(P->cx_fork, s));
        for (int k = 0; k < hfmm_plan::CX_STREAMS; ++k)
            HFMM_CUDA(cudaStreamWaitEvent(P->cx_side[k], P->cx_fork, 0));
        auto launch = [&](int l, int f, cudaStream_t ss) {
            LevelTables& T = P->tables[f][l];
            MixedCall mc = cx_call(P, l, f, R);
            m2l_tf32x3(static_cast<MixedMaps*>(P->cx_maps)[f * MAX_LEVELS + l], mc, ss);
            // expand into the level's downward coordinates: y_dn = d_dn .* (y' U_c^T U_dn)
            // (overwrites; the L2L and X list add to it on the main stream)
            gemm_1(K_EXP, l, f, level_base(T.yc.p, l, T.cmld), T.cmld, P->loc.p + f * fs, P->ld,
                   ss, T.dn_d.p);
            HFMM_CUDA(cudaEventRecord(P->cx_level[l][f], ss));
        };
        for (int f = 0; f < NF; ++f) launch(P->md, f, P->cx_side[f]);
        for (int l = 2; l < P->md; ++l)
            for (int f = 0; f < NF; ++f) launch(l, f, P->cx_side[2 + f]);
        for (int k = 0; k < hfmm_plan::CX_STREAMS; ++k)   // every side stream rejoins
            HFMM_CUDA(cudaEventRecord(P->cx_join[k], P->cx_side[k]));
    }
    // ---- downward pass (M2L + L2L in one GEMM, then X-list P2L, then decode)
    for (int l = 2; l <= P->md; ++l) {
        if (P->streamed && !use_cx) {
            PhaseTimer pt(X, s, 12);
            generate_m2l_stream(P, l, use_mx, P->ws, s);
        }
        if (use_cx) {   // this level's M2L ran above: on a side stream, or queued
            if (cx_side)
                for (int f = 0; f < NF; ++f) HFMM_CUDA(cudaStreamWaitEvent(s, P->cx_level[l][f], 0));
            if (cx_side && l == P->md) {
                for (int k = 0; k < hfmm_plan::CX_STREAMS; ++k)
                    HFMM_CUDA(cudaStreamWaitEvent(s, P->cx_join[k], 0));
                m2l_timer.reset();
            }
            if (l >= 3)   // folded L2L (phases.py:273-278): y_dn += d_dn .* (y_dn(parent) F_o)
                gemm(K_L2LF, l, P->dn_tiles[l][R - 1], P->m2l_src.p + N_DISP, M2L_ENTRIES,
                     P->loc.p, nullptr, P->loc.p, SCALE_DN, 1);
        } else if (use_mx) {
            MixedCall mc{};
            mc.tile_tgt = P->mx_tiles[l][R - 1].tgt.p;
            mc.ntiles = P->mx_tiles[l][R - 1].ntiles;
            mc.src_tab = P->m2l_src.p;
            mc.disp_compact = P->disp_compact.p;
            mc.Bhi = P->e_hi.p;
            mc.Blo = P->e_lo.p;
            mc.Lhi = nullptr;
            mc.Llo = nullptr;
            mc.out = P->check.p;
            mc.R = R;
            mc.ld = P->ld;
            mc.n_fam = NF;
            mc.has_l2l = 0;   // L2L stays FP64 (below): the downward locals are ill-conditioned
            mc.fam_stride = fs;
            mc.out_fam_stride = fs;
            mc.nb = P->nb;
            mc.err = P->d_err.p;
            {
                PhaseTimer pt(X, s, 4);
                m2l_tf32x3(static_cast<MixedMaps*>(P->mx_maps)[l], mc, s);
            }
            if (l >= 3)   // L2L (phases.py:273-278) in FP64, added to the check potential
                gemm(K_L2L, l, P->dn_tiles[l][R - 1], P->m2l_src.p + N_DISP, M2L_ENTRIES, P->loc.p,
                     nullptr, P->check.p);
        } else if (P->rot_P > 0) {   // rotation-based M2L (m2l_rotation.cu), then the L2L GEMM
            {
                PhaseTimer pt(X, s, 4);
                rot_m2l(P, l, R, fs, s);
            }
            if (l >= 3)
                gemm(K_L2L, l, P->dn_tiles[l][R - 1], P->m2l_src.p + N_DISP, M2L_ENTRIES, P->loc.p,
                     nullptr, P->check.p);
        } else {
            gemm(K_DN, l, P->dn_tiles[l][R - 1], P->m2l_src.p, M2L_ENTRIES, P->equiv.p, P->loc.p,
                 P->check.p);
        }
        if (P->nX) {
            if (use_cx)   // the X list's check potentials alone, decoded into y_dn below
                for (int f = 0; f < NF; ++f)
                    HFMM_CUDA(cudaMemsetAsync(
                        P->check.p + f * fs + (int64_t)P->level_lo[l] * R * P->ld, 0,
                        (size_t)(P->level_hi[l] - P->level_lo[l]) * R * P->ld * sizeof(double), s));
            ParticlePass p = base;
            p.op = ParticleOp::P2L;
            p.rows = P->x_tgt.p;
            p.nrows = P->n_x_tgt;
            p.off = P->x_off.p;
            p.srcs = P->x_src.p;
            p.surf = P->equiv_pts.p;
            p.out = P->check.p;
            p.level = l;
            {
                PhaseTimer pt(X, s, 5);
                particles(p, s);
            }
            if (use_cx)
                gemm(K_DNU, l, P->dec_tiles[l][R - 1], nullptr, 0, P->check.p, nullptr, P->loc.p,
                     SCALE_DN, 1);
        }
        if (use_cx)   // leaves leave the coordinates: local densities for L2P, into P->check
            gemm(K_DNV, l, P->leaf_tiles[l][R - 1], nullptr, 0, P->loc.p, nullptr, P->check.p);
        else
            decode(l, false, P->check.p, P->loc.p);
    }
    // ---- particle outputs: the near field (above) stores, far field and W list add
    HFMM_CUDA(cudaStreamWaitEvent(s, P->nf_join, 0));
    {
        ParticlePass p = base;
        p.op = ParticleOp::L2P;
        p.rows = P->leaves.p;
        p.nrows = P->n_leaves;
        p.surf = P->check_pts.p;
        p.dens = use_cx ? P->check.p : P->loc.p;
        {
            PhaseTimer pt(X, s, 8);
            particles(p, s);
        }
        if (P->nW) {
            p = base;
            p.op = ParticleOp::M2P;
            p.rows = P->w_tgt.p;
            p.nrows = P->n_w_tgt;
            p.off = P->w_off.p;
            p.srcs = P->w_src.p;
            p.surf = P->equiv_pts.p;
            p.dens = use_cx ? P->tmp.p : P->equiv.p;
            PhaseTimer pt(X, s, 9);
            particles(p, s);
        }
        p = base;
        p.op = ParticleOp::COMBINE;
        p.rows = P->sort_idx.p;
        p.phi = phi;
        p.E = E;
        PhaseTimer pt(X, s, 10);
        particles(p, s);
    }
}

}  // namespace hfmm

using namespace hfmm;

#define API_BEGIN try {
#define API_END                                              \
    }                                                        \
    catch (const hfmm::Error& e) {                           \
        return fail(e.code, e.msg);                          \
    }                                                        \
    catch (const std::exception& e) {                        \
        return fail(HFMM_ERR_STATE, e.what());               \
    }                                                        \
    catch (...) {                                            \
        return fail(HFMM_ERR_STATE, "unknown error");        \
    }

extern "C" {

const char* hfmm_last_error(void) { return t_last_error.c_str(); }

int64_t hfmm_launch_count(void) { return g_launches.load(); }

int hfmm_tree_build(const double* pos_dev, int64_t n, int32_t n_max, int32_t max_depth,
                    hfmm_plan** out) {
    if (!out) return fail(HFMM_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!pos_dev || n <= 0) return fail(HFMM_ERR_ARG, "positions must be a nonempty (N,3) array");
    if (n_max < 1) return fail(HFMM_ERR_ARG, "N_max must be a positive integer");
    if (n > (int64_t)INT32_MAX) return fail(HFMM_ERR_CAPACITY, "more than 2^31-1 points");
    hfmm_plan* P = new hfmm_plan();
    API_BEGIN
    HFMM_CUDA(cudaGetDevice(&P->device));
    require_device_ptr(pos_dev, "positions");
    P->n = n;
    P->n_max = n_max;
    P->md_given = max_depth > 0;
    P->md = max_depth;
    P->d_err.alloc(1);
    P->d_err.zero();
    tree_build(P, pos_dev);
    *out = P;
    return HFMM_OK;
    }
    catch (const hfmm::Error& e) {
        delete P;
        return fail(e.code, e.msg);
    }
    catch (...) {
        delete P;
        return fail(HFMM_ERR_STATE, "tree build failed");
    }
}

int hfmm_tree_build_in_domain(const double* pos_dev, int64_t n, int32_t n_max, int32_t max_depth,
                              const double* pmin, double extent, hfmm_plan** out) {
    if (!out) return fail(HFMM_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!pos_dev || n <= 0) return fail(HFMM_ERR_ARG, "positions must be a nonempty (N,3) array");
    if (n_max < 1) return fail(HFMM_ERR_ARG, "N_max must be a positive integer");
    if (max_depth < 1) return fail(HFMM_ERR_ARG, "a fixed domain needs a fixed max_depth >= 1");
    if (!pmin || !std::isfinite(pmin[0]) || !std::isfinite(pmin[1]) || !std::isfinite(pmin[2]) ||
        !std::isfinite(extent) || !(extent > 0))
        return fail(HFMM_ERR_ARG, "the domain needs a finite corner and a positive extent");
    if (n > (int64_t)INT32_MAX) return fail(HFMM_ERR_CAPACITY, "more than 2^31-1 points");
    hfmm_plan* P = new hfmm_plan();
    API_BEGIN
    HFMM_CUDA(cudaGetDevice(&P->device));
    require_device_ptr(pos_dev, "positions");
    P->n = n;
    P->n_max = n_max;
    P->md_given = true;
    P->md = max_depth;
    P->domain_fixed = true;
    P->extent = extent;
    for (int a = 0; a < 3; ++a) P->pmin[a] = pmin[a];
    P->d_err.alloc(1);
    P->d_err.zero();
    tree_build(P, pos_dev);
    *out = P;
    return HFMM_OK;
    }
    catch (const hfmm::Error& e) {
        delete P;
        return fail(e.code, e.msg);
    }
    catch (...) {
        delete P;
        return fail(HFMM_ERR_STATE, "tree build failed");
    }
}

int hfmm_plan_rebuild(hfmm_plan* P, const double* pos_dev) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    if (!P->domain_fixed) return fail(HFMM_ERR_STATE, "rebuild needs a plan built in a fixed domain");
    if (!P->finalized) return fail(HFMM_ERR_STATE, "finalize the plan first");
    if (P->batch_owner) return fail(HFMM_ERR_STATE, "the plan belongs to a batch (its graph holds the old tree)");
    if (!pos_dev) return fail(HFMM_ERR_ARG, "positions are NULL");
    API_BEGIN
    require_device_ptr(pos_dev, "positions");
    HFMM_CUDA(cudaDeviceSynchronize());   // no evaluate of the old tree in flight
    tree_build(P, pos_dev);               // checks the domain before it changes anything
    // lists, schedules and every tree-sized buffer follow the new tree; the operator
    // tables (same depth, same domain, same level scales) are kept
    P->finalized = false;
    P->V.release();
    const int rc = hfmm_plan_finalize(P);
    return rc;
    API_END
}

int hfmm_plan_info(const hfmm_plan* P, hfmm_info* o) {
    if (!P || !o) return fail(HFMM_ERR_ARG, "NULL argument");
    std::memset(o, 0, sizeof(*o));
    o->n_points = P->n;
    o->max_depth = P->md;
    o->maxleaf = P->maxleaf;
    o->max_boxes = P->ref_max_boxes;
    o->n_boxes = P->nb;
    o->n_leaves = P->n_leaves;
    o->adaptive = P->adaptive ? 1 : 0;
    for (int l = 0; l < MAX_LEVELS; ++l) {
        o->level_lo[l] = P->level_lo[l];
        o->level_hi[l] = P->level_hi[l];
    }
    o->domain_extent = P->extent;
    for (int a = 0; a < 3; ++a) o->pmin[a] = P->pmin[a];
    o->n_v = P->nV;
    o->n_u = P->nU;
    o->n_w = P->nW;
    o->n_x = P->nX;
    o->n_near = P->nNear;
    o->n_s = P->n_s;
    o->p = P->p;
    return HFMM_OK;
}

int hfmm_plan_set_kernel_kind(hfmm_plan* P, int32_t kind) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    if (kind != HFMM_KERNEL_HELMHOLTZ && kind != HFMM_KERNEL_YUKAWA)
        return fail(HFMM_ERR_ARG, "kind must be HFMM_KERNEL_HELMHOLTZ or HFMM_KERNEL_YUKAWA");
    P->yukawa = kind == HFMM_KERNEL_YUKAWA;
    P->n_s = 0;   // hfmm_plan_set_kernel comes next
    P->finalized = false;
    return HFMM_OK;
}

int hfmm_plan_set_kernel(hfmm_plan* P, double k, int32_t p, int32_t n_families,
                         const double* equiv_pts, const double* check_pts) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    if (!std::isfinite(k)) return fail(HFMM_ERR_ARG, "k must be a finite real number");
    if (P->yukawa && (n_families != 1 || k < 0))
        return fail(HFMM_ERR_ARG, "the screened-Coulomb kernel has one family and kappa >= 0");
    if (p < 2) return fail(HFMM_ERR_ARG, "p must be an integer >= 2");
    if (n_families != 1 && n_families != 2) return fail(HFMM_ERR_ARG, "n_families must be 1 or 2");
    if (!equiv_pts || !check_pts) return fail(HFMM_ERR_ARG, "surfaces are NULL");
    API_BEGIN
    P->k = k;
    P->p = p;
    P->n_s = 6 * p * p - 12 * p + 8;
    P->ld = round_up(P->n_s, 32);
    P->n_fam = n_families;
    for (int f = 0; f < 2; ++f)
        for (int l = 0; l < MAX_LEVELS; ++l) P->tables[f][l].reset();
    std::vector<double> soa(3 * P->n_s);
    for (int which = 0; which < 2; ++which) {
        const double* src = which == 0 ? equiv_pts : check_pts;
        for (int j = 0; j < P->n_s; ++j)
            for (int a = 0; a < 3; ++a) soa[a * P->n_s + j] = src[j * 3 + a];
        DevBuf<double>& d = which == 0 ? P->equiv_pts : P->check_pts;
        d.alloc(soa.size());
        HFMM_CUDA(cudaMemcpy(d.p, soa.data(), soa.size() * 8, cudaMemcpyHostToDevice));
    }
    P->finalized = false;
    return HFMM_OK;
    API_END
}

int hfmm_plan_set_streaming(hfmm_plan* P, int32_t enable) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    if (P->n_s == 0) return fail(HFMM_ERR_STATE, "set the kernel first");
    for (int f = 0; f < 2; ++f)
        for (int l = 0; l < MAX_LEVELS; ++l)
            if (P->tables[f][l].set)
                return fail(HFMM_ERR_STATE, "choose the table mode before the level tables");
    P->streamed = enable != 0;
    if (!P->streamed) {
        P->ws_own.release();
        P->ws = nullptr;
        P->ws_bytes = 0;
    }
    return HFMM_OK;
}

int hfmm_plan_workspace_bytes(const hfmm_plan* P, int64_t* bytes) {
    if (!P || !bytes) return fail(HFMM_ERR_ARG, "plan or output is NULL");
    if (P->n_s == 0) return fail(HFMM_ERR_STATE, "set the kernel first");
    *bytes = (int64_t)stream_ws_bytes(P);
    return HFMM_OK;
}

int hfmm_plan_bind_workspace(hfmm_plan* P, void* ws_dev, int64_t bytes) {
    if (!P || !ws_dev) return fail(HFMM_ERR_ARG, "plan or workspace is NULL");
    if (!P->streamed) return fail(HFMM_ERR_STATE, "the plan does not stream its M2L tables");
    if (bytes < (int64_t)stream_ws_bytes(P)) return fail(HFMM_ERR_CAPACITY, "workspace too small");
    if ((uintptr_t)ws_dev % 256) return fail(HFMM_ERR_ARG, "workspace must be 256-byte aligned");
    API_BEGIN
    require_device_ptr(ws_dev, "workspace");
    P->ws_own.release();
    P->ws = ws_dev;
    P->ws_bytes = (size_t)bytes;
    if (P->finalized) {
        build_a_ptrs(P, extra(P, true)->ix);
        if (P->mixed_ready) stream_maps(P);
    }
    return HFMM_OK;
    API_END
}

int hfmm_plan_set_level(hfmm_plan* P, int32_t family, int32_t level, const double* F_up_U,
                        const double* F_up_d, const double* F_up_Vt, const double* F_dn_U,
                        const double* F_dn_d, const double* F_dn_Vt, const double* M2M_K,
                        const double* L2L_K, const double* M2L_K) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    if (P->n_s == 0) return fail(HFMM_ERR_STATE, "set the kernel first");
    if (family < 0 || family >= P->n_fam) return fail(HFMM_ERR_ARG, "family out of range");
    if (level < 2 || level > P->md) return fail(HFMM_ERR_ARG, "level must be in [2, max_depth]");
    if (!F_up_U || !F_up_d || !F_up_Vt || !F_dn_U || !F_dn_d || !F_dn_Vt || !M2L_K)
        return fail(HFMM_ERR_ARG, "decode and M2L tables are required");
    if (level < P->md && !M2M_K) return fail(HFMM_ERR_ARG, "M2M_K required below max_depth");
    if (level >= 3 && !L2L_K) return fail(HFMM_ERR_ARG, "L2L_K required from level 3");
    API_BEGIN
    const double* h[9] = {F_up_U, F_up_d, F_up_Vt, F_dn_U, F_dn_d, F_dn_Vt, M2M_K, L2L_K, M2L_K};
    upload_level(P, family, level, h);
    P->finalized = false;
    return HFMM_OK;
    API_END
}

int hfmm_plan_set_level_decode(hfmm_plan* P, int32_t family, int32_t level, const double* F_up_U,
                               const double* F_up_d, const double* F_up_Vt, const double* F_dn_U,
                               const double* F_dn_d, const double* F_dn_Vt) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    if (P->n_s == 0) return fail(HFMM_ERR_STATE, "set the kernel first");
    if (family < 0 || family >= P->n_fam) return fail(HFMM_ERR_ARG, "family out of range");
    if (level < 2 || level > P->md) return fail(HFMM_ERR_ARG, "level must be in [2, max_depth]");
    if (!F_up_U || !F_up_d || !F_up_Vt || !F_dn_U || !F_dn_d || !F_dn_Vt)
        return fail(HFMM_ERR_ARG, "decode factors are required");
    API_BEGIN
    const double* h[9] = {F_up_U, F_up_d, F_up_Vt, F_dn_U, F_dn_d, F_dn_Vt, nullptr, nullptr, nullptr};
    upload_level(P, family, level, h);
    P->finalized = false;
    return HFMM_OK;
    API_END
}

int hfmm_plan_finalize(hfmm_plan* P) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    if (P->n_s == 0) return fail(HFMM_ERR_STATE, "set the kernel first");
    for (int f = 0; f < P->n_fam; ++f)
        for (int l = 2; l <= P->md; ++l)
            if (!P->tables[f][l].set)
                return fail(HFMM_ERR_STATE, "tables missing for family " + std::to_string(f) +
                                                " level " + std::to_string(l));
    API_BEGIN
    if (!P->V.p) {
        lists_build(P);
        schedules_build(P);
    }
    // mixed path: the low-rank M2L's buffers and folded tables (compress.cu), before the
    // A pointer table that points at them
    P->mixed_ready = false;
    compressed_prepare(P);
    PlanExtra* X = extra(P, true);
    build_a_ptrs(P, X->ix);   // streamed plans without a workspace yet: see evaluate
    if (!P->crit) {
        int lo = 0, hi = 0;
        HFMM_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        HFMM_CUDA(cudaStreamCreateWithPriority(&P->crit, cudaStreamNonBlocking, hi));
        HFMM_CUDA(cudaEventCreateWithFlags(&P->crit_fork, cudaEventDisableTiming));
        HFMM_CUDA(cudaEventCreateWithFlags(&P->crit_join, cudaEventDisableTiming));
    }
    if (!P->nf_side) {
        HFMM_CUDA(cudaStreamCreateWithFlags(&P->nf_side, cudaStreamNonBlocking));
        HFMM_CUDA(cudaEventCreateWithFlags(&P->nf_fork, cudaEventDisableTiming));
        HFMM_CUDA(cudaEventCreateWithFlags(&P->nf_join, cudaEventDisableTiming));
    }
    const size_t exp = (size_t)P->n_fam * P->nb * 2 * P->ld;
    P->check.alloc(exp);
    P->gemm_part.alloc(GEMM_PART_CAP);
    P->equiv.alloc(exp);
    P->loc.alloc(exp);
    P->tmp.alloc(exp);
    P->check.zero();
    P->equiv.zero();
    P->loc.zero();
    P->tmp.zero();
    // mixed path: TF32 hi/lo tables, tensor maps, split density buffers (needs ld >= 128);
    // with a compressed M2L on every level the dense TF32 tables are not needed
    if (P->ld >= 128) {
        std::vector<int32_t> dc(N_DISP, -1);
        auto madj = nonadjacent_map();
        for (size_t i = 0; i < madj.size(); ++i) dc[madj[i]] = (int32_t)i;
        P->disp_compact.alloc(N_DISP);
        HFMM_CUDA(cudaMemcpy(P->disp_compact.p, dc.data(), N_DISP * 4, cudaMemcpyHostToDevice));
        const size_t mat = (size_t)P->ld * P->ld;
        if (!P->mx_maps) P->mx_maps = new MixedMaps[MAX_LEVELS];
        MixedMaps* maps = static_cast<MixedMaps*>(P->mx_maps);
        std::memset(maps, 0, sizeof(MixedMaps) * MAX_LEVELS);
        if (P->compressed) {
            // the mixed M2L runs on the compressed tables (compress.cu)
        } else if (P->streamed) {
            if (P->ws) stream_maps(P);
        } else {
            for (int f = 0; f < P->n_fam; ++f)
                for (int l = 2; l <= P->md; ++l) {
                    LevelTables& T = P->tables[f][l];
                    const int nm = (int)madj.size();
                    T.m2l_hi.alloc(nm * mat);
                    T.m2l_lo.alloc(nm * mat);
                    split_transpose_tables(T.m2l.p, T.m2l_hi.p, T.m2l_lo.p, P->ld, nm);
                    make_table_map(&maps[l].a_hi[f], T.m2l_hi.p, P->ld, nm);
                    make_table_map(&maps[l].a_lo[f], T.m2l_lo.p, P->ld, nm);
                }
        }
        P->e_hi.alloc(exp);
        P->e_lo.alloc(exp);
        P->e_hi.zero();
        P->e_lo.zero();
        P->mixed_ready = true;
    }
    plan_queue_build(P);
    P->q_s.alloc(2 * P->n);
    P->pot.alloc((size_t)P->n_fam * 2 * P->n);
    P->fld.alloc((size_t)P->n_fam * 2 * 3 * P->n);
    HFMM_CUDA(cudaDeviceSynchronize());
    P->finalized = true;
    return HFMM_OK;
    API_END
}

int hfmm_evaluate(hfmm_plan* P, const double* q_re, const double* q_im, double* phi, double* E,
                  int32_t precision, void* stream) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    if (!P->finalized) return fail(HFMM_ERR_STATE, "plan not finalized");
    if (!q_re || !phi) return fail(HFMM_ERR_ARG, "charges and output are required");
    if (precision != HFMM_PREC_FP64 && precision != HFMM_PREC_MIXED)
        return fail(HFMM_ERR_ARG, "precision must be HFMM_PREC_FP64 or HFMM_PREC_MIXED");
    API_BEGIN
    require_device_ptr(q_re, "q_re");
    if (q_im) require_device_ptr(q_im, "q_im");
    require_device_ptr(phi, "phi_out");
    if (E) require_device_ptr(E, "field_out");
    if (P->streamed && !P->ws) {   // first evaluate without a bound workspace: the plan's own
        P->ws_bytes = stream_ws_bytes(P);
        P->ws_own.alloc(P->ws_bytes / sizeof(double));
        P->ws = P->ws_own.p;
        build_a_ptrs(P, extra(P, true)->ix);
        if (P->mixed_ready) stream_maps(P);
    }
    evaluate_fp64(P, q_re, q_im, phi, E, (cudaStream_t)stream, precision == HFMM_PREC_MIXED);
    return HFMM_OK;
    API_END
}

int hfmm_plan_set_m2l_queue(hfmm_plan* P, int32_t on) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    P->queue_m2l = on != 0;
    return HFMM_OK;
}

int hfmm_plan_check(hfmm_plan* P, void* stream) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    API_BEGIN
    int v = 0;
    HFMM_CUDA(cudaMemcpyAsync(&v, P->d_err.p, sizeof(int), cudaMemcpyDeviceToHost,
                              (cudaStream_t)stream));
    HFMM_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (v) {
        HFMM_CUDA(cudaMemsetAsync(P->d_err.p, 0, sizeof(int), (cudaStream_t)stream));
        HFMM_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
        return fail(HFMM_ERR_DEVICE, "device error flag " + std::to_string(v) +
                                         " (1 = index out of bounds, 2 = capacity, 4 = a bounded wait timed out)");
    }
    return HFMM_OK;
    API_END
}

}  // extern "C"

namespace hfmm {
bool plan_profiling(hfmm_plan* P) {
    PlanExtra* X = extra(P, false);
    return X && X->profiling;
}
}  // namespace hfmm

extern "C" {

int hfmm_plan_set_profiling(hfmm_plan* P, int32_t enable) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    API_BEGIN
    PlanExtra* X = extra(P, true);
    if (enable && X->ev.empty()) {
        const size_t slots = 8192;
        X->ev.resize(2 * slots);
        for (auto& e : X->ev) HFMM_CUDA(cudaEventCreate(&e));
        X->ev_phase.assign(slots, -1);
    }
    X->profiling = enable != 0;
    X->used = 0;
    return HFMM_OK;
    API_END
}

int hfmm_plan_phase_times(hfmm_plan* P, double* ms) {
    if (!P || !ms) return fail(HFMM_ERR_ARG, "NULL argument");
    API_BEGIN
    for (int i = 0; i < HFMM_N_PHASES; ++i) ms[i] = 0.0;
    PlanExtra* X = extra(P, false);
    if (!X || !X->profiling) return fail(HFMM_ERR_STATE, "profiling is off");
    for (size_t i = 0; i < X->used; ++i) {
        HFMM_CUDA(cudaEventSynchronize(X->ev[2 * i + 1]));
        float t = 0;
        HFMM_CUDA(cudaEventElapsedTime(&t, X->ev[2 * i], X->ev[2 * i + 1]));
        if (X->ev_phase[i] >= 0 && X->ev_phase[i] < HFMM_N_PHASES) ms[X->ev_phase[i]] += t;
    }
    X->used = 0;   // the next read covers the evaluates issued after this one
    return HFMM_OK;
    API_END
}

void hfmm_plan_destroy(hfmm_plan* P) {
    if (!P) return;
    if (P->batch_owner) batch_forget_plan(P->batch_owner, P);
    drop_extra(P);
    delete[] static_cast<MixedMaps*>(P->mx_maps);
    P->mx_maps = nullptr;
    plan_queue_release(P);
    delete[] static_cast<MixedMaps*>(P->cx_maps);
    P->cx_maps = nullptr;
    compressed_release(P);
    if (P->nf_side) cudaStreamDestroy(P->nf_side);
    if (P->crit) cudaStreamDestroy(P->crit);
    if (P->crit_fork) cudaEventDestroy(P->crit_fork);
    if (P->crit_join) cudaEventDestroy(P->crit_join);
    if (P->nf_fork) cudaEventDestroy(P->nf_fork);
    if (P->nf_join) cudaEventDestroy(P->nf_join);
    delete P;
}

int hfmm_export_tree(const hfmm_plan* P, uint64_t* m_id, int32_t* p_id, int32_t* lvls,
                     int32_t* counts, uint8_t* is_leaf, int32_t* sort_idx) {
    if (!P) return fail(HFMM_ERR_ARG, "plan is NULL");
    API_BEGIN
    const int64_t nb = P->nb;
    if (m_id) HFMM_CUDA(cudaMemcpy(m_id, P->m_id.p, nb * 8, cudaMemcpyDeviceToHost));
    if (p_id) HFMM_CUDA(cudaMemcpy(p_id, P->p_id.p, nb * 4, cudaMemcpyDeviceToHost));
    if (lvls) HFMM_CUDA(cudaMemcpy(lvls, P->lvls.p, nb * 4, cudaMemcpyDeviceToHost));
    if (counts) HFMM_CUDA(cudaMemcpy(counts, P->counts.p, nb * 4, cudaMemcpyDeviceToHost));
    if (is_leaf) HFMM_CUDA(cudaMemcpy(is_leaf, P->is_leaf.p, nb, cudaMemcpyDeviceToHost));
    if (sort_idx) HFMM_CUDA(cudaMemcpy(sort_idx, P->sort_idx.p, P->n * 4, cudaMemcpyDeviceToHost));
    return HFMM_OK;
    API_END
}

int hfmm_export_pil(const hfmm_plan* P, int32_t* pil) {
    if (!P || !pil) return fail(HFMM_ERR_ARG, "NULL argument");
    API_BEGIN
    std::vector<int32_t> ls(P->nb), sidx(P->n);
    HFMM_CUDA(cudaMemcpy(ls.data(), P->leaf_start.p, P->nb * 4, cudaMemcpyDeviceToHost));
    HFMM_CUDA(cudaMemcpy(sidx.data(), P->sort_idx.p, P->n * 4, cudaMemcpyDeviceToHost));
    const int w = P->maxleaf;
    for (int64_t b = 0; b < P->nb; ++b) {
        int32_t* row = pil + b * w;
        for (int j = 0; j < w; ++j) row[j] = -1;
        if (ls[b] < 0) continue;
        int c = std::min(P->h_counts[b], w);
        for (int j = 0; j < c; ++j) row[j] = sidx[ls[b] + j];
    }
    return HFMM_OK;
    API_END
}

int hfmm_export_list(const hfmm_plan* P, int32_t which, int32_t* pairs, int64_t cap) {
    if (!P || !pairs) return fail(HFMM_ERR_ARG, "NULL argument");
    API_BEGIN
    const DevBuf<int32_t>* b;
    int64_t len;
    switch (which) {
        case 0: b = &P->V; len = P->nV; break;
        case 1: b = &P->U; len = P->nU; break;
        case 2: b = &P->W; len = P->nW; break;
        case 3: b = &P->X; len = P->nX; break;
        case 4: b = &P->near; len = P->nNear; break;
        default: return fail(HFMM_ERR_ARG, "which must be 0..4");
    }
    if (cap < len) return fail(HFMM_ERR_CAPACITY, "pairs buffer too small");
    if (len) HFMM_CUDA(cudaMemcpy(pairs, b->p, len * 8, cudaMemcpyDeviceToHost));
    return HFMM_OK;
    API_END
}

int hfmm_export_densities(const hfmm_plan* P, int32_t which, int32_t columns, double* out,
                          int64_t cap) {
    if (!P || !out) return fail(HFMM_ERR_ARG, "NULL argument");
    if (!P->finalized) return fail(HFMM_ERR_STATE, "plan not finalized");
    if (which != 0 && which != 1) return fail(HFMM_ERR_ARG, "which must be 0 (up) or 1 (down)");
    if (columns != 1 && columns != 2) return fail(HFMM_ERR_ARG, "columns must be 1 or 2");
    // [family][box][column][ld], the family stride being n_boxes x columns x ld (evaluate
    // lays the arrays out for its own column count; finalize sized them for two columns)
    const int64_t rows = (int64_t)P->n_fam * P->nb * columns;
    if (cap < rows * P->n_s) return fail(HFMM_ERR_CAPACITY, "densities buffer too small");
    API_BEGIN
    HFMM_CUDA(cudaDeviceSynchronize());
    std::vector<double> h((size_t)(rows * P->ld));
    const DevBuf<double>& b = which == 0 ? P->equiv : P->loc;
    if (rows)
        HFMM_CUDA(cudaMemcpy(h.data(), b.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int64_t r = 0; r < rows; ++r)
        std::copy(h.data() + r * P->ld, h.data() + r * P->ld + P->n_s, out + r * P->n_s);
    return HFMM_OK;
    API_END
}

int64_t hfmm_direct_scratch_bytes(int64_t n, int64_t n_t) {
    if (n <= 0 || n_t < 0) return fail(HFMM_ERR_ARG, "invalid direct-sum sizes");
    return (int64_t)direct_splits(n, n_t) * std::max<int64_t>(n_t, 1) * 8 * (int64_t)sizeof(double);
}

int hfmm_direct_async(const double* pos, const double* q_re, const double* q_im, int64_t n,
                      const int32_t* targets, int64_t n_t, double k, double* phi, double* fld,
                      double* scratch, int64_t scratch_bytes, int* err_dev, void* stream) {
    if (!pos || !q_re || !targets || !phi || !scratch || !err_dev || n <= 0 || n_t < 0)
        return fail(HFMM_ERR_ARG, "invalid direct-sum arguments");
    if (!std::isfinite(k)) return fail(HFMM_ERR_ARG, "k must be finite");
    const int splits = direct_splits(n, n_t);
    if (scratch_bytes < (int64_t)splits * std::max<int64_t>(n_t, 1) * 8 * (int64_t)sizeof(double))
        return fail(HFMM_ERR_CAPACITY, "direct-sum scratch too small (hfmm_direct_scratch_bytes)");
    API_BEGIN
    require_device_ptr(pos, "positions");
    require_device_ptr(q_re, "q_re");
    if (q_im) require_device_ptr(q_im, "q_im");
    require_device_ptr(targets, "targets");
    require_device_ptr(phi, "phi_out");
    if (fld) require_device_ptr(fld, "field_out");
    require_device_ptr(scratch, "scratch");
    require_device_ptr(err_dev, "err");
    direct_sum(pos, q_re, q_im, n, targets, n_t, k, phi, fld, scratch, splits,
               (cudaStream_t)stream, err_dev);
    return HFMM_OK;
    API_END
}

int hfmm_direct_kernel(int32_t kind, const double* pos, const double* q_re, const double* q_im,
                       int64_t n, const int32_t* targets, int64_t n_t, double k, double* phi,
                       double* fld, void* stream);

int hfmm_direct(const double* pos, const double* q_re, const double* q_im, int64_t n,
                const int32_t* targets, int64_t n_t, double k, double* phi, double* fld,
                void* stream) {
    return hfmm_direct_kernel(HFMM_KERNEL_HELMHOLTZ, pos, q_re, q_im, n, targets, n_t, k, phi, fld,
                              stream);
}

int hfmm_direct_kernel(int32_t kind, const double* pos, const double* q_re, const double* q_im,
                       int64_t n, const int32_t* targets, int64_t n_t, double k, double* phi,
                       double* fld, void* stream) {
    if (kind != HFMM_KERNEL_HELMHOLTZ && kind != HFMM_KERNEL_YUKAWA)
        return fail(HFMM_ERR_ARG, "kind must be HFMM_KERNEL_HELMHOLTZ or HFMM_KERNEL_YUKAWA");
    if (!pos || !q_re || !targets || !phi || n <= 0 || n_t < 0)
        return fail(HFMM_ERR_ARG, "invalid direct-sum arguments");
    if (!std::isfinite(k)) return fail(HFMM_ERR_ARG, "k must be finite");
    API_BEGIN
    require_device_ptr(pos, "positions");
    require_device_ptr(q_re, "q_re");
    if (q_im) require_device_ptr(q_im, "q_im");
    require_device_ptr(targets, "targets");
    require_device_ptr(phi, "phi_out");
    if (fld) require_device_ptr(fld, "field_out");
    int splits = direct_splits(n, n_t);
    DevBuf<double> scratch;
    scratch.alloc((size_t)splits * std::max<int64_t>(n_t, 1) * 8);
    DevBuf<int> err;
    err.alloc(1);
    err.zero((cudaStream_t)stream);
    direct_sum(pos, q_re, q_im, n, targets, n_t, k, phi, fld, scratch.p, splits,
               (cudaStream_t)stream, err.p, kind == HFMM_KERNEL_YUKAWA ? 1 : 0);
    int h = 0;
    HFMM_CUDA(cudaMemcpyAsync(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    HFMM_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (h) return fail(HFMM_ERR_ARG, "target index out of range");
    return HFMM_OK;
    API_END
}

}  // extern "C"
