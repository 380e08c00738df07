// Mixed-precision M2L (+ L2L) on the 5th-generation tensor cores: split 3xTF32.
//
// Same contraction as the FP64 output-stationary GEMM (gemm_f64.cu; M2L of
// phases.py:211-236 and L2L of phases.py:273-278 summed into one check
// potential), with every product A*B evaluated as
//     A_hi*B_hi + A_hi*B_lo + A_lo*B_hi,   x_hi = tf32(x), x_lo = tf32(x - x_hi)
// by tcgen05.mma kind::tf32 into one FP32 accumulator in tensor memory.
//
// CTA = one tile of target boxes (same level and octant) x one 128-row block of
// the n_s check points x one kernel family; accumulator 128 lanes x 128 columns
// (targets x charge columns) FP32 in TMEM. Per k-chunk of 32 (128-byte rows):
//   * warp 4 (one lane) loads A_hi and A_lo with TMA (3-D tensor maps over the
//     level's tables, SWIZZLE_128B, K-major) -> mbarrier complete_tx;
//   * warps 0-3 gather the B columns (source boxes' equivalent densities) with
//     16-byte cp.async into the same SWIZZLE_128B K-major layout; each thread's
//     cp.async.mbarrier.arrive counts on the stage's mbarrier once its copies land
//     (the MMA warp fences the generic->async proxy after its wait);
//   * warp 5 (one lane) issues 4 k-steps x 3 tcgen05.mma and commits the stage
//     back to its "empty" mbarrier;
// three stages in flight.
// Grid mode (a complete level with complex charges, the uniform workloads): the
// level's densities sit in a dense box grid and a tile is one octant of a 4 x 4 x 4
// block of parents, so its 64 targets' sources at one displacement form a stride-2
// 4 x 4 x 4 box of that grid: warp 4 then loads B hi/lo with two 5-D TMA copies per
// stage as well (element strides 2, out-of-domain sources read the zero fill), the
// gather warps idle, and the stage's only barrier is the TMA transaction count.
// Accumulation precision: the error of an FP32 accumulator grows with the
// length of its chain of MMAs (measured: about linearly), and the damped decode
// amplifies it. So every FOLD k-chunks (24 MMAs) accumulate into a fresh FP32
// buffer in TMEM (four buffers in turn, 4 x 128 columns = all 512), and the fold
// warps (16: four per TMEM lane quadrant, each taking 32 of the 128 columns) add each
// finished buffer into FP64 running sums held in their own registers, 32 doubles a
// thread, while the tensor core fills the next buffers. The FP64 sums are stored as
// the check potentials. (Folding every 4 k-chunks instead was 22 % faster but
// doubled the M2L error: 8.3e-7 against 4.6e-7 for the potential at p = 8.)
// Registers: the block launches with 768 threads; setmaxnreg moves registers from
// the gather and control warpgroups (warps 0-7) to the four fold warpgroups (8-23),
// and the host checks that the split fits the launch's register file before the
// first launch.
// Every mbarrier wait is bounded (2 s of %globaltimer by default); a timeout sets
// the CTA's abort flag and the device error flag, and every role stops issuing.
// Before TMEM is freed and the CTA exits, nothing it issued may still be in flight:
// the TMA thread waits for the bytes of every stage it loaded (their own tx-only
// barriers, so the wait does not depend on the other roles), the MMA thread commits
// its issued MMAs to a drain barrier and waits for it, and the gather threads wait
// for their own copies. These drain waits ignore the abort flag and are bounded by
// time only.
#include "hfmm_internal.cuh"
#include "m2l_common.cuh"
#include "mixed.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

namespace hfmm {

namespace {

using namespace mxk;

template <int R>
__global__ void __launch_bounds__(THREADS, 1) k_m2l_tf32x3(const __grid_constant__ MixedMaps maps,
                                                            MixedCall c) {
    constexpr int TT = BN / R;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* sm = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    Ctl& ctl = *reinterpret_cast<Ctl*>(sm + STAGES * STAGE_BYTES);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile = blockIdx.x, m0 = blockIdx.y * BM, fam = blockIdx.z;
    volatile int* abort_flag = &ctl.abort_flag;
    const uint64_t wait_ns = c.wait_ns ? c.wait_ns : WAIT_NS;
    const bool half = (c.m_valid > 0 ? c.m_valid : c.ldm) - m0 <= 64;
    const uint32_t idesc = half ? IDESC64 : IDESC;

    if (tid < TT) {   // targets share the sources' box range (a level's own buffers)
        int t = c.tile_tgt[(int64_t)tile * TT + tid];
        const int64_t lo = c.src_hi > 0 ? c.src_lo : 0, hi = c.src_hi > 0 ? c.src_hi : c.nb;
        if (t >= 0 && (t < lo || t >= hi)) {
            atomicOr(c.err, ERRF_BOUNDS);
            t = -1;
        }
        ctl.tgt[tid] = t;
    }
    for (int e = tid; e < M2L_ENTRIES; e += THREADS) {
        ctl.used[e] = 0;
        ctl.ztab[e] = (short)(e < N_DISP ? c.disp_compact[e] : (c.has_l2l ? e - N_DISP : -1));
    }
    if (tid == 0) {
        ctl.abort_flag = 0;
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&ctl.full[s]), 128);   // each gather thread's copies
            mbar_init(smem_u32(&ctl.tfull[s]), 1);    // the TMA thread's arrive + its bytes
            mbar_init(smem_u32(&ctl.empty[s]), 1);    // MMA commit
        }
        for (int b = 0; b < NACC; ++b) {
            mbar_init(smem_u32(&ctl.acc_full[b]), 1);
            mbar_init(smem_u32(&ctl.acc_empty[b]), N_FOLD_WARPS);   // one per fold warp
        }
        mbar_init(smem_u32(&ctl.done), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 5) {   // tensor memory: the FP32 accumulation buffers
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&ctl.tmem)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    // active entries: every thread tests (target, entry) pairs, entries fastest (the
    // source table's rows are read coalesced) and the loads of a batch independent of
    // each other; warp 0 then compacts the flags with ballots
    {
        constexpr int BATCH = 16;
        constexpr int PAIRS = TT * M2L_ENTRIES;
        for (int i0 = tid; i0 < PAIRS; i0 += THREADS * BATCH) {
            int src[BATCH];
#pragma unroll
            for (int u = 0; u < BATCH; ++u) {
                const int i = i0 + u * THREADS;
                src[u] = -1;
                if (i < PAIRS) {
                    const int t = ctl.tgt[i / M2L_ENTRIES];
                    if (t >= 0) src[u] = __ldg(c.src_tab + (int64_t)t * M2L_ENTRIES + i % M2L_ENTRIES);
                }
            }
#pragma unroll
            for (int u = 0; u < BATCH; ++u)
                if (src[u] >= 0) ctl.used[(i0 + u * THREADS) % M2L_ENTRIES] = 1;
        }
    }
    __syncthreads();
    if (warp == 0) {
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
    const int n_act = ctl.n_act;
    const int kch = c.ldk / BK;
    const int nq = n_act * kch;
    const uint32_t tmem = ctl.tmem;
    const int64_t fs = (int64_t)fam * c.fam_stride;
    // per warpgroup: the fold warps take the registers the other roles do not need
    if (warp < 4)
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(REG_GATHER));
    else if (warp < FOLD_WARP0)
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(REG_CTRL));
    else
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(REG_FOLD));

    if (warp < 4) {
        if (!c.grid) {   // (grid mode: B comes by TMA, warp 4)
            // ---------------- B gathers (cp.async, manual SWIZZLE_128B placement)
            const float* Bh = c.Bhi + fs;
            const float* Bl = c.Blo + fs;
            // Each thread always serves chunk ch of the same CPR rows (columns) of the B
            // tile: rows n_i = tid / CPR + (128 / CPR) i. Their swizzled shared-memory
            // offsets are fixed (the 16-byte chunk index XORs with the row's bits: all three
            // for 128-byte rows, the upper two for 64-byte rows, as TMA and the MMA read them);
            // their global sources change only when the displacement entry changes.
            constexpr int RSTEP = 128 / CPR;
            const int ch = tid % CPR;
            uint32_t soff[CPR];
            int64_t goff[CPR];
    #pragma unroll
            for (int i = 0; i < CPR; ++i) {
                const int n = tid / CPR + RSTEP * i;
                const int sw = BK == 32 ? (n & 7) : ((n & 7) >> 1);
                soff[i] = (uint32_t)((n >> 3) * 8 * ROW_BYTES + (n & 7) * ROW_BYTES + ((ch ^ sw) << 4));
                goff[i] = -1;
            }
            // The source boxes of the next entry are loaded while the current one streams,
            // so the table lookups' latency stays off the copy pipeline.
            int nsrc[CPR];
            auto load_sources = [&](int ai) {
                const int e = ctl.act[ai];
    #pragma unroll
                for (int i = 0; i < CPR; ++i) {
                    const int t = ctl.tgt[(tid / CPR + RSTEP * i) / R];
                    nsrc[i] = t >= 0 ? c.src_tab[(int64_t)t * M2L_ENTRIES + e] : -1;
                }
            };
            const int64_t src_lo = c.src_hi > 0 ? c.src_lo : 0;
            const int64_t src_hi = c.src_hi > 0 ? c.src_hi : c.nb;
            if (nq > 0) load_sources(0);
            int cur_entry = -1;
            for (int q = 0; q < nq; ++q) {
                const int st = q % STAGES;
                const int ai = q / kch;
                if (ai != cur_entry) {   // new displacement entry: this thread's 8 sources
                    cur_entry = ai;
    #pragma unroll
                    for (int i = 0; i < CPR; ++i) {
                        const int n = tid / CPR + RSTEP * i;
                        int s_ = nsrc[i];
                        if (s_ >= 0 && (s_ < src_lo || s_ >= src_hi)) {
                            atomicOr(c.err, ERRF_BOUNDS);
                            s_ = -1;
                        }
                        goff[i] = s_ >= 0 ? ((int64_t)s_ * R + (n % R)) * c.ldk + ch * 4 : -1;
                    }
                    if (ai + 1 < n_act) load_sources(ai + 1);
                }
                if (!mbar_wait(smem_u32(&ctl.empty[st]), ((q / STAGES) & 1) ^ 1, abort_flag, wait_ns)) break;
                const int k0 = (q % kch) * BK;
                const uint32_t sbh = smem_u32(sm + st * STAGE_BYTES + 2 * TILE_BYTES);
                const uint32_t sbl = sbh + TILE_BYTES;
    #pragma unroll
                for (int i = 0; i < CPR; ++i) {
                    const bool ok = goff[i] >= 0;
                    const int64_t o = ok ? goff[i] + k0 : 0;
                    cp_async16(sbh + soff[i], Bh + o, ok);
                    cp_async16(sbl + soff[i], Bl + o, ok);
                }
                // the stage's barrier counts this thread's arrival when its copies have
                // landed: no thread waits for its own copies, so every stage can be in flight
                // (c.starve: a test leaves stage 0 without its arrivals, so the MMA thread's
                // bounded wait runs out)
                if (!(c.starve && q == 0))
                    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(
                                     smem_u32(&ctl.full[st]))
                                 : "memory");
            }
            // drain: this thread's copies (and the arrivals they trigger) complete
            asm volatile("cp.async.wait_all;\n" ::: "memory");
        }
    } else if (warp >= FOLD_WARP0) {
        // ---------------- fold each finished buffer into FP64 sums in registers
        // Warp w may touch TMEM lanes 32 (w % 4) .. + 31 only: four fold warps cover
        // each lane quadrant, each folding 32 of the 128 columns.
        const int quad = warp & 3;                 // TMEM lane quadrant of this warp
        const int c_lo = ((warp - FOLD_WARP0) >> 2) * COLS_PER_FOLD_WARP;
        // the row of this lane (M = 64 blocks: lanes 16-31 of a quadrant hold none)
        const int m = half ? m0 + quad * 16 + lane : m0 + quad * 32 + lane;
        const bool row_ok = half ? (lane < 16 && m < c.ldm) : (m0 + quad * 32 < c.ldm);
        const uint32_t lane_base = tmem + ((uint32_t)(quad * 32) << 16);
        double* out = c.out + (int64_t)fam * c.out_fam_stride;
        double sum[COLS_PER_FOLD_WARP];
#pragma unroll
        for (int j = 0; j < COLS_PER_FOLD_WARP; ++j) sum[j] = 0.0;
        bool ok = true;
        const int n_units = (nq + FOLD - 1) / FOLD;
        for (int i = 0; i < n_units; ++i) {
            const int b = i & (NACC - 1);
            // the TMEM loads below are warp-collective: agree on the wait's outcome
            const bool got = mbar_wait(smem_u32(&ctl.acc_full[b]), (i / NACC) & 1, abort_flag, wait_ns);
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
            __syncwarp();   // one arrive per fold warp
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
                if (t >= 0) out[((int64_t)t * R + (n % R)) * c.ldm + m] = sum[j];
            }
        }
    } else if (warp == 4) {
        // ---------------- A tiles by TMA
        if (lane == 0) {
            const CUtensorMap* mh = &maps.a_hi[fam];
            const CUtensorMap* ml = &maps.a_lo[fam];
            const CUtensorMap* lh = &maps.l_hi[fam];
            const CUtensorMap* ll = &maps.l_lo[fam];
            const CUtensorMap* bh = &maps.b_hi[fam];
            const CUtensorMap* bl = &maps.b_lo[fam];
            int ox = 0, oy = 0, oz = 0;   // grid mode: the tile's grid origin
            if (c.grid) {
                ox = c.tile_org[3 * (int64_t)tile];
                oy = c.tile_org[3 * (int64_t)tile + 1];
                oz = c.tile_org[3 * (int64_t)tile + 2];
            }
            int last_q[STAGES];   // the last q loaded into each stage (-1: none)
#pragma unroll
            for (int st = 0; st < STAGES; ++st) last_q[st] = -1;
            for (int q = 0; q < nq; ++q) {
                const int st = q % STAGES;
                if (!mbar_wait(smem_u32(&ctl.empty[st]), ((q / STAGES) & 1) ^ 1, abort_flag, wait_ns)) break;
                if (c.grid && c.starve && q == 0) continue;   // test: stage 0 never fills
                const int e = ctl.act[q / kch];
                const int z = ctl.zidx[q / kch];
                const int k0 = (q % kch) * BK;
                const uint32_t fb = smem_u32(&ctl.tfull[st]);
                const uint32_t sa = smem_u32(sm + st * STAGE_BYTES);
                mbar_arrive_tx(fb, (c.grid ? 4 : 2) * TILE_BYTES);
                if (e < N_DISP) {
                    tma_load_3d(sa, mh, k0, m0, z, fb);
                    tma_load_3d(sa + TILE_BYTES, ml, k0, m0, z, fb);
                } else {
                    tma_load_3d(sa, lh, k0, m0, z, fb);
                    tma_load_3d(sa + TILE_BYTES, ll, k0, m0, z, fb);
                }
                if (c.grid) {   // sources at target - d, d = (e / 49 - 3, (e / 7) % 7 - 3, e % 7 - 3)
                    const int sx = ox - (e / 49 - 3), sy = oy - ((e / 7) % 7 - 3), sz = oz - (e % 7 - 3);
                    tma_load_5d(sa + 2 * TILE_BYTES, bh, k0, 0, sz, sy, sx, fb);
                    tma_load_5d(sa + 3 * TILE_BYTES, bl, k0, 0, sz, sy, sx, fb);
                }
#pragma unroll
                for (int j = 0; j < STAGES; ++j)
                    if (j == st) last_q[j] = q;
            }
            // drain: every stage's last load has landed (earlier loads of a stage were
            // consumed by the MMA thread before the stage was loaded again)
            bool drained = true;
#pragma unroll
            for (int j = 0; j < STAGES; ++j)
                if (last_q[j] >= 0)
                    drained &= mbar_drain(smem_u32(&ctl.tfull[j]), (last_q[j] / STAGES) & 1, wait_ns);
            if (!drained) atomicOr(c.err, ERRF_TIMEOUT);
        }
    } else if (warp == 5) {
        // ---------------- MMA issue (warp 5, one lane; warps 6 and 7 have no role)
        if (lane == 0) {
            bool ok = true, issued = false;
            for (int q = 0; q < nq && ok; ++q) {
                const int st = q % STAGES;
                const int unit = q / FOLD, uq = q % FOLD;
                const int b = unit & (NACC - 1);
                if (uq == 0 && unit >= NACC) {   // buffer b must have been folded (unit - NACC)
                    if (!mbar_wait(smem_u32(&ctl.acc_empty[b]), ((unit / NACC) & 1) ^ 1, abort_flag, wait_ns)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;");
                }
                if ((!c.grid && !mbar_wait(smem_u32(&ctl.full[st]), (q / STAGES) & 1, abort_flag, wait_ns)) ||
                    !mbar_wait(smem_u32(&ctl.tfull[st]), (q / STAGES) & 1, abort_flag, wait_ns)) {
                    ok = false;
                    break;
                }
                // the gathered B halves were written by cp.async (generic proxy): order them
                // before the tensor core's (async proxy) reads of the stage
                if (!c.grid) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t base = smem_u32(sm + st * STAGE_BYTES);
                const uint64_t ah = sw_desc(base), al = sw_desc(base + TILE_BYTES);
                const uint64_t bh = sw_desc(base + 2 * TILE_BYTES),
                               bl = sw_desc(base + 3 * TILE_BYTES);
                const uint32_t dt = tmem + b * BN;
#pragma unroll
                for (int ks = 0; ks < BK / 8; ++ks) {   // 8 tf32 = 32 bytes per k-step
                    const uint64_t d = (uint64_t)(ks * 2);
                    umma_tf32(dt, ah + d, bh + d, idesc, (uq > 0 || ks > 0) ? 1u : 0u);
                    umma_tf32(dt, ah + d, bl + d, idesc, 1u);
                    umma_tf32(dt, al + d, bh + d, idesc, 1u);
                }
                issued = true;
                umma_commit(smem_u32(&ctl.empty[st]));
                if (uq == FOLD - 1 || q == nq - 1) umma_commit(smem_u32(&ctl.acc_full[b]));
            }
            // drain, on every exit path: the commit tracks every MMA this thread issued
            if (issued) {
                umma_commit(smem_u32(&ctl.done));
                if (!mbar_drain(smem_u32(&ctl.done), 0, wait_ns)) atomicOr(c.err, ERRF_TIMEOUT);
            }
        }
    }
    // nothing this CTA issued is in flight into shared or tensor memory from here on
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 5) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// Round an FP32 value to TF32 (10 explicit mantissa bits, ties away from zero) and
// clear the 13 low bits, so the container holds exactly the value the tensor core
// multiplies, however it treats the low bits.
__device__ __forceinline__ float tf32_exact(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// x -> (hi, lo) with hi = tf32(x), lo = tf32(x - hi), both exact TF32 in FP32 containers
__device__ __forceinline__ void split2(double x, float& hi, float& lo) {
    hi = tf32_exact((float)x);
    lo = tf32_exact((float)(x - (double)hi));
}

__global__ void k_split_tf32(const double* __restrict__ src, float* hi, float* lo, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float h, l;
    split2(src[i], h, l);
    hi[i] = h;
    lo[i] = l;
}

// densities [box][2][ckld] of a complete level -> TF32 halves at the box's grid position
__global__ void k_split_tf32_grid(const double* __restrict__ src, const uint64_t* __restrict__ m_id,
                                  int64_t n, int G, int ckld, float* hi, float* lo) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t row = 2 * (int64_t)ckld;
    const int64_t b = i / row, within = i % row;
    int64_t x, y, z;
    demorton3(m_id[b], x, y, z);
    if (x >= G || y >= G || z >= G) return;
    const int64_t o = ((x * G + y) * G + z) * row + within;
    float h, l;
    split2(src[i], h, l);
    hi[o] = h;
    lo[o] = l;
}

// FP64 A^T tables ([k][m], ld x ld) -> TF32 hi/lo A tables ([m][k]), count matrices
__global__ void k_split_transpose(const double* __restrict__ at, float* hi, float* lo, int ld) {
    __shared__ double tile[32][33];
    const int c = blockIdx.z;
    const int bk = blockIdx.x * 32, bm = blockIdx.y * 32;
    const double* S = at + (int64_t)c * ld * ld;
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        int k = bk + yy, m = bm + threadIdx.x;
        tile[yy][threadIdx.x] = (k < ld && m < ld) ? S[(int64_t)k * ld + m] : 0.0;
    }
    __syncthreads();
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        int m = bm + yy, k = bk + threadIdx.x;
        if (m < ld && k < ld) {
            float h, l;
            split2(tile[threadIdx.x][yy], h, l);
            int64_t o = (int64_t)c * ld * ld + (int64_t)m * ld + k;
            hi[o] = h;
            lo[o] = l;
        }
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    if (!fn) throw Error{HFMM_ERR_CUDA, "cuTensorMapEncodeTiled is not available"};
    return fn;
}

}  // namespace

void make_table_map(CUtensorMap* map, const float* base, int ld, int count, int ldm) {
    // [count][ldm][ld] fp32 (ldm = 0: square), boxes of BK k x 128 m
    if (!ldm) ldm = ld;
    if (((uintptr_t)base & 15) || (ld * 4) % 16 || ld < BK || ldm < BM)
        throw Error{HFMM_ERR_STATE, "tensor map: table not 16-byte aligned or smaller than a box"};
    cuuint64_t dims[3] = {(cuuint64_t)ld, (cuuint64_t)ldm, (cuuint64_t)count};
    cuuint64_t strides[2] = {(cuuint64_t)ld * 4, (cuuint64_t)ld * ldm * 4};
    cuuint32_t box[3] = {BK, BM, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode_fn()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)base, dims, strides,
                             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             BK == 32 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error{HFMM_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r)};
}

void make_grid_map(CUtensorMap* map, const float* base, int ckld, int G) {
    // dense grid [x][y][z][2][ckld] fp32: dims (k, r, z, y, x); a box is one k-chunk of both
    // charge columns of 4 x 4 x 4 boxes two grid steps apart (element strides 2: a box of
    // 8 elements loads 4 of them), 128 rows of ROW_BYTES in the tile layout of the A maps
    if (((uintptr_t)base & 15) || (ckld * 4) % 16 || ckld < BK || G < 1)
        throw Error{HFMM_ERR_STATE, "grid map: grid not 16-byte aligned or smaller than a box"};
    cuuint64_t dims[5] = {(cuuint64_t)ckld, 2, (cuuint64_t)G, (cuuint64_t)G, (cuuint64_t)G};
    cuuint64_t strides[4] = {(cuuint64_t)ckld * 4, (cuuint64_t)ckld * 8, (cuuint64_t)G * ckld * 8,
                             (cuuint64_t)G * G * ckld * 8};
    cuuint32_t box[5] = {BK, 2, 8, 8, 8};
    cuuint32_t estr[5] = {1, 1, 2, 2, 2};
    CUresult r = encode_fn()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, (void*)base, dims, strides,
                             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             BK == 32 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        throw Error{HFMM_ERR_CUDA, "cuTensorMapEncodeTiled (grid) failed: " + std::to_string((int)r)};
}

void split_tf32_grid(const double* src, const uint64_t* m_id, int64_t n_boxes, int G, int ckld,
                     float* hi, float* lo, cudaStream_t s) {
    const int64_t n = n_boxes * 2 * ckld;
    if (n <= 0) return;
    HFMM_LAUNCH(k_split_tf32_grid, (unsigned)ceil_div(n, 256), 256, 0, s, src, m_id, n, G, ckld, hi, lo);
}

void split_tf32(const double* src, float* hi, float* lo, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    HFMM_LAUNCH(k_split_tf32, (unsigned)ceil_div(n, 256), 256, 0, s, src, hi, lo, n);
}

void split_transpose_tables(const double* at, float* hi, float* lo, int ld, int count) {
    dim3 grid((unsigned)ceil_div(ld, 32), (unsigned)ceil_div(ld, 32), (unsigned)count);
    HFMM_LAUNCH(k_split_transpose, grid, dim3(32, 8), 0, 0, at, hi, lo, ld);
}

// setmaxnreg.inc draws on the registers the block was launched with: the split of the
// three warp roles must fit THREADS x (registers per thread at launch), or the fold
// warps' increase would wait forever. Checked once, before the first launch.
void check_register_split() {
    static int verdict = 0;   // 0 unknown, 1 fits, -1 does not
    static std::mutex mu;
    std::lock_guard<std::mutex> g(mu);
    if (verdict == 0) {
        int fits = 1;
        for (int r = 0; r < 2; ++r) {
            cudaFuncAttributes a{};
            HFMM_CUDA(cudaFuncGetAttributes(&a, r ? (const void*)k_m2l_tf32x3<2> : (const void*)k_m2l_tf32x3<1>));
            const long need = 128L * REG_GATHER + 128L * REG_CTRL + 32L * N_FOLD_WARPS * REG_FOLD;
            if ((long)a.numRegs * THREADS < need || a.maxThreadsPerBlock < THREADS) fits = 0;
        }
        verdict = fits ? 1 : -1;
    }
    if (verdict < 0)
        throw Error{HFMM_ERR_STATE, "m2l_tf32x3: the warp roles' register split exceeds the launch's registers"};
}

std::atomic<uint64_t> g_m2l_wait_ns{0};
std::atomic<int> g_m2l_grid{1};
std::atomic<int> g_m2l_starve{0};

size_t m2l_tf32x3_smem() { return (size_t)STAGES * STAGE_BYTES + sizeof(Ctl) + 1024; }

void m2l_tf32x3(const MixedMaps& maps, const MixedCall& call, cudaStream_t s) {
    if (call.ntiles == 0) return;
    MixedCall c = call;
    c.wait_ns = g_m2l_wait_ns.load();
    c.starve = g_m2l_starve.load();
    if (!c.ldk) c.ldk = c.ld;
    if (!c.ldm) c.ldm = c.ld;
    if (c.ldk % BK || c.ldm % BK)
        throw Error{HFMM_ERR_STATE, "m2l_tf32x3: ld must be a multiple of 32"};
    const size_t smem = m2l_tf32x3_smem();
    dim3 grid(c.ntiles, (c.ldm + BM - 1) / BM, c.n_fam);
    check_register_split();
    if (c.R == 1) {
        HFMM_CUDA(cudaFuncSetAttribute(k_m2l_tf32x3<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        HFMM_LAUNCH(k_m2l_tf32x3<1>, grid, THREADS, smem, s, maps, c);
    } else {
        HFMM_CUDA(cudaFuncSetAttribute(k_m2l_tf32x3<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        HFMM_LAUNCH(k_m2l_tf32x3<2>, grid, THREADS, smem, s, maps, c);
    }
}

}  // namespace hfmm

extern "C" int hfmm_debug_m2l_grid(int on) {
    hfmm::g_m2l_grid = on ? 1 : 0;
    return HFMM_OK;
}

extern "C" int hfmm_debug_m2l_wait(uint64_t wait_ns, int starve) {
    hfmm::g_m2l_wait_ns = wait_ns;
    hfmm::g_m2l_starve = starve ? 1 : 0;
    return HFMM_OK;
}
