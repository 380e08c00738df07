// Shared pieces of the tcgen05 M2L kernels (m2l_tf32x3.cu: one launch per level and
// family; m2l_queue.cu: one persistent launch over a queue of such work): tile and
// stage geometry, warp roles and their register split, the bounded mbarrier waits,
// the TMA / UMMA / TMEM instruction wrappers and the per-CTA control block.
#pragma once
#include "hfmm_internal.cuh"
#include "mixed.cuh"

#include <cuda.h>

namespace hfmm {
namespace mxk {

constexpr int BM = 128;          // UMMA M (check points per CTA)
constexpr int BN = 128;          // UMMA N (target columns per CTA)
// fp32 elements per k-chunk: 32 (128-byte rows, SWIZZLE_128B, three 64 KiB stages) or
// 16 (64-byte rows, SWIZZLE_64B, six 32 KiB stages), the same 192 KiB of operands in
// flight. Same results bit for bit; on the 1M-point p = 8 low-rank M2L 32 took 11.5 ms
// and 16 took 14.0: each stage carries a fixed cost of about 0.3 us that the MMAs do
// not hide, so fewer, larger stages win.
#ifndef HFMM_MX_BK
#define HFMM_MX_BK 32
#endif
constexpr int BK = HFMM_MX_BK;
static_assert(BK == 16 || BK == 32, "k-chunk");
constexpr int ROW_BYTES = BK * 4;           // one K-major row of a tile
constexpr int CPR = ROW_BYTES / 16;         // 16-byte chunks per row
constexpr int TILE_BYTES = BM * ROW_BYTES;  // one operand half
constexpr int STAGE_BYTES = 4 * TILE_BYTES;
constexpr int STAGES = (3 * 64 * 1024) / STAGE_BYTES;
constexpr int N_FOLD_WARPS = 16;                  // four per TMEM lane quadrant
constexpr int FOLD_WARP0 = 8;                     // warps 0-3 gather, 4 TMA, 5 MMA, 6-7 idle
constexpr int THREADS = (FOLD_WARP0 + N_FOLD_WARPS) * 32;
constexpr int COLS_PER_FOLD_WARP = BN * 4 / N_FOLD_WARPS;   // 32
constexpr int NACC = 4;                           // FP32 accumulation buffers in TMEM
constexpr int TMEM_COLS = NACC * BN;              // 512
// registers per thread after setmaxnreg: gather warpgroup, control warpgroup, fold
constexpr int REG_GATHER = 64, REG_CTRL = 32, REG_FOLD = 96;
static_assert(128 * REG_GATHER + 128 * REG_CTRL + 32 * N_FOLD_WARPS * REG_FOLD <= THREADS * 80,
              "register split exceeds an 80-register launch");
constexpr int FOLD = 64 / BK;   // k-chunks per FP32 accumulation unit: 64 K values, 24 MMAs
constexpr uint64_t WAIT_NS = 2000000000ull;   // bounded waits: 2 s

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false on timeout (which sets the abort flag) or when another role
// has aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                          uint64_t limit_ns) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = gtimer();
    while (true) {
        if (mbar_try(bar, parity)) return true;
        if (*abort_flag) return false;
        if (gtimer() - t0 > limit_ns) {
            *abort_flag = 1;
            return false;
        }
    }
}
// Drain wait: for work this thread has already issued, so it ignores the abort flag;
// bounded by time only.
__device__ __forceinline__ bool mbar_drain(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
    const uint64_t t0 = gtimer();
    while (!mbar_try(bar, parity))
        if (gtimer() - t0 > limit_ns) return false;
    return true;
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src),
                 "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, int c3, int c4, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
        : "memory");
}
// UMMA shared-memory descriptor: K-major, swizzled rows of ROW_BYTES (layout type 2 =
// SWIZZLE_128B, 4 = SWIZZLE_64B), 8-row groups 8 * ROW_BYTES apart.
__device__ __forceinline__ uint64_t sw_desc(uint32_t addr) {
    constexpr uint64_t layout = BK == 32 ? 2 : 4;
    return (uint64_t)((addr & 0x3FFFF) >> 4) | (1ull << 16) |
           ((uint64_t)(8 * ROW_BYTES / 16) << 32) | (1ull << 46) | (layout << 61);
}
__device__ __forceinline__ void umma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
          "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}
// Instruction descriptor: D = F32, A = B = TF32, both K-major, M = 128 (or 64), N = BN.
constexpr uint32_t idesc_m(int m) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}
constexpr uint32_t IDESC = idesc_m(BM);
// A row block with at most 64 rows that can be nonzero (the last block of a level whose
// rank r leaves r - m0 <= 64, e.g. r = 185 in two blocks, or a low-rank sin table)
// runs the M = 64 shape: half the tensor work. Its accumulator occupies TMEM lanes
// 0-15 of each 32-lane quadrant (row i at lane 32 (i / 16) + i % 16), the layout
// CUTLASS's 1-SM UMMA fragments give M = 64.
constexpr uint32_t IDESC64 = idesc_m(64);

struct __align__(8) Ctl {
    uint64_t full[STAGES];   // the gather threads' copies of a stage have landed
    uint64_t tfull[STAGES];  // the stage's TMA bytes have landed (tx-only)
    uint64_t empty[STAGES];
    uint64_t acc_full[NACC];    // a unit's FP32 sum is complete in buffer b (MMA commit)
    uint64_t acc_empty[NACC];   // buffer b has been folded into the FP64 sums (one per fold warp)
    uint64_t done;
    uint32_t tmem;
    int abort_flag;
    int n_act;
    int tgt[BN];
    short act[M2L_ENTRIES + 1];
    short zidx[M2L_ENTRIES + 1];   // A-table index of each active entry (M2L or L2L table)
    unsigned char used[M2L_ENTRIES + 1];   // entry has a source for some target of the tile
    short ztab[M2L_ENTRIES + 1];           // A-table index of every entry (-1: none)
};


}  // namespace mxk
}  // namespace hfmm
