// Mixed-precision (3xTF32 on tcgen05) M2L: shared declarations.
#pragma once
#include "hfmm_internal.cuh"

#include <cuda.h>

#include <atomic>

#include <string>
#include <vector>

namespace hfmm {

// TMA descriptors of one level's TF32 hi/lo tables, per kernel family:
// M2L (316 non-adjacent displacements) and L2L (8 octants), each [z][m][k] fp32.
struct MixedMaps {
    CUtensorMap a_hi[2], a_lo[2], l_hi[2], l_lo[2];
    CUtensorMap b_hi[2], b_lo[2];   // grid mode: the level's dense density grid (5-D)
};

struct MixedCall {
    const int32_t* tile_tgt;       // ntiles x (128 / R) target boxes, -1 padded
    int ntiles;
    const int32_t* src_tab;        // nb x 351 source boxes (-1 = none)
    const int32_t* disp_compact;   // 343: displacement -> M2L table index (-1 = adjacent)
    const float* Bhi;              // equivalent densities, split, [fam][box][R][ld]
    const float* Blo;
    const float* Lhi;              // parent local densities, split (L2L entries)
    const float* Llo;
    double* out;                   // check potentials [fam][box][R][ld], FP64
    int R, ld, n_fam, has_l2l;
    int ldk, ldm;                  // rectangular tables: K extent (B rows) and M extent (out
                                   // rows); 0 = ld. A tables are [count][ldm][ldk]
    int m_valid;                   // rows of A that can be nonzero (0 = ldm): a row block
                                   // with at most 64 of them runs the M = 64 MMA shape
    int64_t fam_stride, out_fam_stride, nb;
    int64_t src_lo, src_hi;        // valid source boxes [src_lo, src_hi) (0, nb when unset)
    int* err;
    uint64_t wait_ns;              // limit of each bounded wait (0: 2 s); set by m2l_tf32x3
    int starve;                    // test only: leave stage 0 without its gather arrivals
    // grid mode (complete level, R = 2): B comes from the dense density grid by TMA, one
    // strided 4 x 4 x 4 box per displacement; tile_tgt then holds grid tiles and
    // tile_org each tile's grid origin (x, y, z)
    int grid;
    const int32_t* tile_org;
};

// Wait limit and starvation switch of the next M2L launches (hfmm_debug_m2l_wait):
// a test makes a bounded wait run out on purpose and checks the error status. Atomic:
// a hook call may come from another thread than the evaluate that reads it.
extern std::atomic<uint64_t> g_m2l_wait_ns;
extern std::atomic<int> g_m2l_starve;

void make_table_map(CUtensorMap* map, const float* base, int ld, int count, int ldm = 0);
void split_tf32(const double* src, float* hi, float* lo, int64_t n, cudaStream_t s);
// a complete level's densities [box][2][ckld] (boxes in level order from m_id) -> TF32
// halves in the dense grid [x][y][z][2][ckld] of side G
void split_tf32_grid(const double* src, const uint64_t* m_id, int64_t n_boxes, int G, int ckld,
                     float* hi, float* lo, cudaStream_t s);
void make_grid_map(CUtensorMap* map, const float* base, int ckld, int G);
// process-wide: 1 (default) lets complete levels use grid mode, 0 forces the gather
extern std::atomic<int> g_m2l_grid;
void split_transpose_tables(const double* at, float* hi, float* lo, int ld, int count);
void m2l_tf32x3(const MixedMaps& maps, const MixedCall& c, cudaStream_t s);

// the low-rank mixed M2L call of one plan, level and family for R charge columns
MixedCall cx_call(hfmm_plan* P, int l, int f, int R);

// One work item of the queued M2L: a tile x one 128-row block of calls[call].
struct M2LItem {
    int call, tile, mblock;
};
// Persistent M2L over items (sorted by the caller), n_ctas resident CTAs; `next` is a
// device int the launch resets. calls, maps and items live in device memory. The wait
// limit comes from g_m2l_wait_ns at launch; starve (a test switch) leaves every CTA's
// first stage unfilled.
void m2l_queue(const MixedCall* calls, const MixedMaps* maps, const M2LItem* items, int n_items,
               int* next, int R, int n_ctas, cudaStream_t s, int starve = 0);
// The work list of a queued M2L over the plans given: every (plan, level, family)
// low-rank call with its tensor maps, one item per tile and 128-row block, largest
// first (cost: k-chunks per entry, 0.6 for a block of at most 64 live rows). Returns
// "" when it applies, else why not (32-bit gather offsets would overflow).
std::string queue_items(hfmm_plan* const* plans, int n_plans, int R, std::vector<MixedCall>& calls,
                        std::vector<MixedMaps>& maps, std::vector<M2LItem>& items);
// A plan's own queued M2L for R charge columns, built and uploaded at finalize.
struct PlanQueue {
    DevBuf<MixedCall> calls;
    DevBuf<MixedMaps> maps;
    DevBuf<M2LItem> items;
    DevBuf<int> next;
    int n_items = 0;
};
void plan_queue_build(hfmm_plan* P);     // both charge-column counts
void plan_queue_release(hfmm_plan* P);
size_t m2l_queue_smem();
size_t m2l_tf32x3_smem();

}  // namespace hfmm
