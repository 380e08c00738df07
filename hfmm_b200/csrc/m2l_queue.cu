// Persistent mixed-precision M2L over a work queue: the batched evaluate's M2L.
//
// A batch of plans (batch.cu) runs every plan's upward pass, then ONE launch of this
// kernel for the M2L of every plan, level and kernel family, then every plan's
// downward pass. Each work item is one target tile x one 128-row block of one
// (plan, level, family) M2L -- the unit one CTA of k_m2l_tf32x3 computes -- and the
// items are queued by decreasing cost, so large levels start first and the small
// problems' few coarse tiles fill the tail. One CTA per SM stays resident and takes
// the next item with an atomic counter until the queue is empty: tensor memory is
// allocated, mbarriers initialised and registers split once per CTA, and the stage
// and accumulation-unit counters run on across items, so consecutive items keep the
// pipeline's barrier phases. The per-item arithmetic is k_m2l_tf32x3's (3xTF32
// products, FP32 units of 24 MMAs folded into FP64 sums held in registers), the call
// parameters (MixedCall) and the TMA tensor maps of every (plan, level, family) come
// from global memory. Every wait is bounded as in k_m2l_tf32x3; a timeout stops the
// CTA after the item, drains what it issued and frees tensor memory.
#include "hfmm_internal.cuh"
#include "m2l_common.cuh"
#include "mixed.cuh"

#include <algorithm>

namespace hfmm {

using namespace mxk;

namespace {

struct __align__(8) QueueCtl {
    uint64_t full[STAGES];
    uint64_t tfull[STAGES];
    uint64_t empty[STAGES];
    uint64_t acc_full[NACC];
    uint64_t acc_empty[NACC];
    uint64_t done;
    uint32_t tmem;
    int abort_flag;
    int item;                 // the item this CTA works on (-1: queue empty)
    int n_act;
    int tgt[BN];
    short act[M2L_ENTRIES + 1];
    short zidx[M2L_ENTRIES + 1];
    unsigned char used[M2L_ENTRIES + 1];
    short ztab[M2L_ENTRIES + 1];
    MixedCall c;              // the item's call parameters
};

// Start of an item, called by every thread of the CTA in the same order (four block
// barriers): the first fold warp takes the next item and copies its call parameters,
// the fold warps (which hold the most registers) load the tile's targets and find its
// active entries. Returns false, for every thread at once, when the queue is empty or
// the CTA has timed out. FOLDER: compiled for the fold warps, which do the work.
template <int R, bool FOLDER>
__device__ __forceinline__ bool next_item(QueueCtl& ctl, const MixedCall* __restrict__ calls,
                                          const M2LItem* __restrict__ items, int n_items, int* next,
                                          int warp, int lane, int tid) {
    constexpr int TT = BN / R;
    if (FOLDER && warp == FOLD_WARP0 && lane == 0) {
        const int it = ctl.abort_flag ? n_items : atomicAdd(next, 1);
        ctl.item = it < n_items ? it : -1;
        if (it < n_items) ctl.c = calls[items[it].call];
    }
    __syncthreads();
    if (ctl.item < 0) return false;
    const int ft = tid - FOLD_WARP0 * 32;   // 0..511 in the fold warps
    if (FOLDER) {
        const MixedCall& c = ctl.c;
        const int tile = items[ctl.item].tile;
        if (ft < TT) {
            int t = c.tile_tgt[(int64_t)tile * TT + ft];
            const int64_t lo = c.src_hi > 0 ? c.src_lo : 0, hi = c.src_hi > 0 ? c.src_hi : c.nb;
            if (t >= 0 && (t < lo || t >= hi)) {
                atomicOr(c.err, ERRF_BOUNDS);
                t = -1;
            }
            ctl.tgt[ft] = t;
        }
        for (int e = ft; e < M2L_ENTRIES; e += 32 * N_FOLD_WARPS) {
            ctl.used[e] = 0;
            ctl.ztab[e] = (short)(e < N_DISP ? c.disp_compact[e] : (c.has_l2l ? e - N_DISP : -1));
        }
    }
    __syncthreads();
    if (FOLDER) {
        const MixedCall& c = ctl.c;
        constexpr int BATCH = 4;
        constexpr int PAIRS = TT * M2L_ENTRIES;
        constexpr int NT = 32 * N_FOLD_WARPS;
        for (int i0 = ft; i0 < PAIRS; i0 += NT * BATCH) {
            int src[BATCH];
#pragma unroll
            for (int u = 0; u < BATCH; ++u) {
                const int i = i0 + u * NT;
                src[u] = -1;
                if (i < PAIRS) {
                    const int t = ctl.tgt[i / M2L_ENTRIES];
                    if (t >= 0) src[u] = __ldg(c.src_tab + (int64_t)t * M2L_ENTRIES + i % M2L_ENTRIES);
                }
            }
#pragma unroll
            for (int u = 0; u < BATCH; ++u)
                if (src[u] >= 0) ctl.used[(i0 + u * NT) % M2L_ENTRIES] = 1;
        }
    }
    __syncthreads();
    if (FOLDER && warp == FOLD_WARP0) {
        int base = 0;
        for (int e0 = 0; e0 < M2L_ENTRIES; e0 += 32) {
            int e = e0 + lane;
            const bool act = e < M2L_ENTRIES && ctl.used[e] && ctl.ztab[e] >= 0;
            unsigned bal = __ballot_sync(0xffffffffu, act);
            if (act) {
                const int slot = base + __popc(bal & ((1u << lane) - 1));
                ctl.act[slot] = (short)e;
                ctl.zidx[slot] = ctl.ztab[e];
            }
            base += __popc(bal);
        }
        if (lane == 0) ctl.n_act = base;
    }
    __syncthreads();
    return true;
}

template <int R>
__global__ void __launch_bounds__(THREADS, 1)
    k_m2l_queue(const MixedCall* __restrict__ calls, const MixedMaps* __restrict__ maps,
                const M2LItem* __restrict__ items, int n_items, int* next, uint64_t wait_ns_in,
                int starve) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* sm = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    QueueCtl& ctl = *reinterpret_cast<QueueCtl*>(sm + STAGES * STAGE_BYTES);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    volatile int* abort_flag = &ctl.abort_flag;
    const uint64_t wait_ns = wait_ns_in ? wait_ns_in : WAIT_NS;

    if (tid == 0) {
        ctl.abort_flag = 0;
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&ctl.full[s]), 128);
            mbar_init(smem_u32(&ctl.tfull[s]), 1);
            mbar_init(smem_u32(&ctl.empty[s]), 1);
        }
        for (int b = 0; b < NACC; ++b) {
            mbar_init(smem_u32(&ctl.acc_full[b]), 1);
            mbar_init(smem_u32(&ctl.acc_empty[b]), N_FOLD_WARPS);
        }
        mbar_init(smem_u32(&ctl.done), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&ctl.tmem)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = ctl.tmem;
    if (warp < 4)
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(REG_GATHER));
    else if (warp < FOLD_WARP0)
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(REG_CTRL));
    else
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(REG_FOLD));

    // Every role runs its own loop over the items; the loops meet at the same block
    // barriers (four in next_item, one at each item's end). q_total and u_total are the
    // stages and accumulation units this CTA has issued before the current item.
    int q_total = 0, u_total = 0;
    if (warp < 4) {
        // ---------------- B gathers (k_m2l_tf32x3's, for items that are not in grid mode)
        while (next_item<R, false>(ctl, calls, items, n_items, next, warp, lane, tid)) {
            const MixedCall& c = ctl.c;
            const int kch = c.ldk / BK, nq = ctl.n_act * kch;
            if (!c.grid) {
                constexpr int RSTEP = 128 / CPR;
                const int ch = tid % CPR;
                uint32_t soff[CPR];
                int goff[CPR];   // element offsets: the host keeps nb x R x ldk below 2^31
#pragma unroll
                for (int i = 0; i < CPR; ++i) {
                    const int n = tid / CPR + RSTEP * i;
                    const int sw = BK == 32 ? (n & 7) : ((n & 7) >> 1);
                    soff[i] = (uint32_t)((n >> 3) * 8 * ROW_BYTES + (n & 7) * ROW_BYTES + ((ch ^ sw) << 4));
                    goff[i] = -1;
                }
                const int64_t src_lo = c.src_hi > 0 ? c.src_lo : 0;
                const int64_t src_hi = c.src_hi > 0 ? c.src_hi : c.nb;
                int cur_entry = -1;
                for (int q = 0; q < nq; ++q) {
                    const int qg = q_total + q, st = qg % STAGES;
                    const int ai = q / kch;
                    if (ai != cur_entry) {
                        cur_entry = ai;
                        const int e = ctl.act[ai];
#pragma unroll
                        for (int i = 0; i < CPR; ++i) {
                            const int n = tid / CPR + RSTEP * i;
                            const int t = ctl.tgt[n / R];
                            int s_ = t >= 0 ? c.src_tab[(int64_t)t * M2L_ENTRIES + e] : -1;
                            if (s_ >= 0 && (s_ < src_lo || s_ >= src_hi)) {
                                atomicOr(c.err, ERRF_BOUNDS);
                                s_ = -1;
                            }
                            goff[i] = s_ >= 0 ? (s_ * R + (n % R)) * c.ldk + ch * 4 : -1;
                        }
                    }
                    if (!mbar_wait(smem_u32(&ctl.empty[st]), ((qg / STAGES) & 1) ^ 1, abort_flag, wait_ns)) break;
                    const int k0 = (q % kch) * BK;
                    const uint32_t sbh = smem_u32(sm + st * STAGE_BYTES + 2 * TILE_BYTES);
                    const uint32_t sbl = sbh + TILE_BYTES;
#pragma unroll
                    for (int i = 0; i < CPR; ++i) {
                        const bool ok = goff[i] >= 0;
                        const int o = ok ? goff[i] + k0 : 0;
                        cp_async16(sbh + soff[i], c.Bhi + o, ok);
                        cp_async16(sbl + soff[i], c.Blo + o, ok);
                    }
                    if (!(starve && qg == 0))   // (test: the CTA's first stage never fills)
                        asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(
                                         smem_u32(&ctl.full[st]))
                                     : "memory");
                }
                asm volatile("cp.async.wait_all;\n" ::: "memory");
            }
            q_total += nq;
            __syncthreads();
        }
    } else if (warp >= FOLD_WARP0) {
        // ---------------- fold into FP64 sums in registers; store at each item's end
        const int quad = warp & 3;
        const int c_lo = ((warp - FOLD_WARP0) >> 2) * COLS_PER_FOLD_WARP;
        const uint32_t lane_base = tmem + ((uint32_t)(quad * 32) << 16);
        while (next_item<R, true>(ctl, calls, items, n_items, next, warp, lane, tid)) {
            const MixedCall& c = ctl.c;
            const int m0 = items[ctl.item].mblock * BM;
            const bool half = (c.m_valid > 0 ? c.m_valid : c.ldm) - m0 <= 64;
            const int kch = c.ldk / BK, nq = ctl.n_act * kch;
            const int n_units = (nq + FOLD - 1) / FOLD;
            const int m = half ? m0 + quad * 16 + lane : m0 + quad * 32 + lane;
            const bool row_ok = half ? (lane < 16 && m < c.ldm) : (m0 + quad * 32 < c.ldm);
            double sum[COLS_PER_FOLD_WARP];
#pragma unroll
            for (int j = 0; j < COLS_PER_FOLD_WARP; ++j) sum[j] = 0.0;
            bool ok = true;
            for (int u = 0; u < n_units; ++u) {
                const int ug = u_total + u, b = ug & (NACC - 1);
                const bool got = mbar_wait(smem_u32(&ctl.acc_full[b]), (ug / NACC) & 1, abort_flag, wait_ns);
                if (!__all_sync(0xffffffffu, got)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    uint32_t v[16];
                    tmem_ld16(lane_base + b * BN + c_lo + 16 * h, v);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int j = 0; j < 16; ++j) sum[16 * h + j] += (double)__uint_as_float(v[j]);
                }
                asm volatile("tcgen05.fence::before_thread_sync;");
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&ctl.acc_empty[b]));
            }
            const bool aborted = !__all_sync(0xffffffffu, ok && !*abort_flag);
            if (aborted) {
                if (lane == 0) atomicOr(c.err, ERRF_TIMEOUT);
            } else if (row_ok) {
#pragma unroll
                for (int j = 0; j < COLS_PER_FOLD_WARP; ++j) {
                    const int n = c_lo + j;
                    const int t = ctl.tgt[n / R];
                    if (t >= 0) c.out[((int64_t)t * R + (n % R)) * c.ldm + m] = sum[j];
                }
            }
            u_total += n_units;
            __syncthreads();
        }
    } else if (warp == 4) {
        // ---------------- A (and, in grid mode, B) tiles by TMA
        int last_q[STAGES];   // the last stage index loaded into each stage
#pragma unroll
        for (int st = 0; st < STAGES; ++st) last_q[st] = -1;
        int* err = nullptr;
        while (next_item<R, false>(ctl, calls, items, n_items, next, warp, lane, tid)) {
            const MixedCall& c = ctl.c;
            const int kch = c.ldk / BK, nq = ctl.n_act * kch;
            if (lane == 0) {
                err = c.err;
                const int tile = items[ctl.item].tile, m0 = items[ctl.item].mblock * BM;
                const MixedMaps* mp = maps + items[ctl.item].call;
                const CUtensorMap* mh = &mp->a_hi[0];
                const CUtensorMap* ml = &mp->a_lo[0];
                const CUtensorMap* bh = &mp->b_hi[0];
                const CUtensorMap* bl = &mp->b_lo[0];
                // the maps were written through the generic proxy (a host copy): make them
                // visible to the tensor-map proxy before their use in this item
                asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(mh) : "memory");
                asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(ml) : "memory");
                int ox = 0, oy = 0, oz = 0;
                if (c.grid) {
                    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(bh) : "memory");
                    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(bl) : "memory");
                    ox = c.tile_org[3 * (int64_t)tile];
                    oy = c.tile_org[3 * (int64_t)tile + 1];
                    oz = c.tile_org[3 * (int64_t)tile + 2];
                }
                for (int q = 0; q < nq; ++q) {
                    const int qg = q_total + q, st = qg % STAGES;
                    if (!mbar_wait(smem_u32(&ctl.empty[st]), ((qg / STAGES) & 1) ^ 1, abort_flag, wait_ns)) break;
                    if (c.grid && starve && qg == 0) continue;   // (test: stage 0 never fills)
                    const int e = ctl.act[q / kch];
                    const int z = ctl.zidx[q / kch];
                    const int k0 = (q % kch) * BK;
                    const uint32_t fb = smem_u32(&ctl.tfull[st]);
                    const uint32_t sa = smem_u32(sm + st * STAGE_BYTES);
                    mbar_arrive_tx(fb, (c.grid ? 4 : 2) * TILE_BYTES);
                    tma_load_3d(sa, mh, k0, m0, z, fb);
                    tma_load_3d(sa + TILE_BYTES, ml, k0, m0, z, fb);
                    if (c.grid) {
                        const int sx = ox - (e / 49 - 3), sy = oy - ((e / 7) % 7 - 3), sz = oz - (e % 7 - 3);
                        tma_load_5d(sa + 2 * TILE_BYTES, bh, k0, 0, sz, sy, sx, fb);
                        tma_load_5d(sa + 3 * TILE_BYTES, bl, k0, 0, sz, sy, sx, fb);
                    }
#pragma unroll
                    for (int j = 0; j < STAGES; ++j)
                        if (j == st) last_q[j] = qg;
                }
            }
            q_total += nq;
            __syncthreads();
        }
        if (lane == 0) {   // drain: every stage's last load has landed
            bool drained = true;
#pragma unroll
            for (int j = 0; j < STAGES; ++j)
                if (last_q[j] >= 0) drained &= mbar_drain(smem_u32(&ctl.tfull[j]), (last_q[j] / STAGES) & 1, wait_ns);
            if (!drained && err) atomicOr(err, ERRF_TIMEOUT);
        }
    } else if (warp == 5) {
        // ---------------- MMA issue
        bool issued = false;
        int* err = nullptr;
        // The gather warps complete a stage's full barrier only for items that are not in
        // grid mode, so its phase is not the stage counter's: bit st holds the parity of
        // full[st]'s next phase.
        uint32_t full_par = 0;
        while (next_item<R, false>(ctl, calls, items, n_items, next, warp, lane, tid)) {
            const MixedCall& c = ctl.c;
            const int kch = c.ldk / BK, nq = ctl.n_act * kch;
            const int n_units = (nq + FOLD - 1) / FOLD;
            if (lane == 0) {
                err = c.err;
                const int m0 = items[ctl.item].mblock * BM;
                const bool half = (c.m_valid > 0 ? c.m_valid : c.ldm) - m0 <= 64;
                const uint32_t idesc = half ? IDESC64 : IDESC;
                for (int q = 0; q < nq; ++q) {
                    const int qg = q_total + q, st = qg % STAGES;
                    const int u = q / FOLD, uq = q % FOLD;
                    const int ug = u_total + u, b = ug & (NACC - 1);
                    if (uq == 0 && ug >= NACC) {
                        if (!mbar_wait(smem_u32(&ctl.acc_empty[b]), ((ug / NACC) & 1) ^ 1, abort_flag, wait_ns))
                            break;
                        asm volatile("tcgen05.fence::after_thread_sync;");
                    }
                    if (!c.grid) {
                        if (!mbar_wait(smem_u32(&ctl.full[st]), (full_par >> st) & 1u, abort_flag, wait_ns))
                            break;
                        full_par ^= 1u << st;
                    }
                    if (!mbar_wait(smem_u32(&ctl.tfull[st]), (qg / STAGES) & 1, abort_flag, wait_ns)) break;
                    if (!c.grid) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    const uint32_t base = smem_u32(sm + st * STAGE_BYTES);
                    const uint64_t ah = sw_desc(base), al = sw_desc(base + TILE_BYTES);
                    const uint64_t bh = sw_desc(base + 2 * TILE_BYTES), bl = sw_desc(base + 3 * TILE_BYTES);
                    const uint32_t dt = tmem + b * BN;
#pragma unroll
                    for (int ks = 0; ks < BK / 8; ++ks) {
                        const uint64_t d = (uint64_t)(ks * 2);
                        umma_tf32(dt, ah + d, bh + d, idesc, (uq > 0 || ks > 0) ? 1u : 0u);
                        umma_tf32(dt, ah + d, bl + d, idesc, 1u);
                        umma_tf32(dt, al + d, bh + d, idesc, 1u);
                    }
                    issued = true;
                    umma_commit(smem_u32(&ctl.empty[st]));
                    if (uq == FOLD - 1 || q == nq - 1) umma_commit(smem_u32(&ctl.acc_full[b]));
                }
            }
            q_total += nq;
            u_total += n_units;
            __syncthreads();
        }
        if (lane == 0 && issued) {   // drain: the commit tracks every MMA issued
            umma_commit(smem_u32(&ctl.done));
            if (!mbar_drain(smem_u32(&ctl.done), 0, wait_ns) && err) atomicOr(err, ERRF_TIMEOUT);
        }
    } else {
        // warps 6 and 7: no role; they keep the item barriers' count
        while (next_item<R, false>(ctl, calls, items, n_items, next, warp, lane, tid)) __syncthreads();
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 5) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

void check_queue_split() {
    static int verdict = 0;
    if (verdict == 0) {
        int fits = 1;
        for (int r = 0; r < 2; ++r) {
            cudaFuncAttributes a{};
            HFMM_CUDA(cudaFuncGetAttributes(&a, r ? (const void*)k_m2l_queue<2> : (const void*)k_m2l_queue<1>));
            const long need = 128L * REG_GATHER + 128L * REG_CTRL + 32L * N_FOLD_WARPS * REG_FOLD;
            if ((long)a.numRegs * THREADS < need || a.maxThreadsPerBlock < THREADS) fits = 0;
        }
        verdict = fits ? 1 : -1;
    }
    if (verdict < 0)
        throw Error{HFMM_ERR_STATE, "m2l_queue: the warp roles' register split exceeds the launch's registers"};
}

}  // namespace

size_t m2l_queue_smem() { return (size_t)STAGES * STAGE_BYTES + sizeof(QueueCtl) + 1024; }

void m2l_queue(const MixedCall* calls, const MixedMaps* maps, const M2LItem* items, int n_items,
               int* next, int R, int n_ctas, cudaStream_t s, int starve) {
    if (n_items <= 0) return;
    check_queue_split();
    const size_t smem = m2l_queue_smem();
    const int grid = std::max(1, std::min(n_ctas, n_items));
    HFMM_CUDA(cudaMemsetAsync(next, 0, sizeof(int), s));
    if (R == 1) {
        HFMM_CUDA(cudaFuncSetAttribute(k_m2l_queue<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        HFMM_LAUNCH(k_m2l_queue<1>, grid, THREADS, smem, s, calls, maps, items, n_items, next, g_m2l_wait_ns.load(),
                    starve);
    } else {
        HFMM_CUDA(cudaFuncSetAttribute(k_m2l_queue<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        HFMM_LAUNCH(k_m2l_queue<2>, grid, THREADS, smem, s, calls, maps, items, n_items, next, g_m2l_wait_ns.load(),
                    starve);
    }
}

}  // namespace hfmm
