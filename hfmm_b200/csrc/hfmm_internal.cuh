// Internal declarations of the hfmm_b200 library: the plan object, error
// plumbing, launch accounting and device helpers shared by the .cu files.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include <atomic>

#include "../../include/hfmm_b200.h"

namespace hfmm {

// ---------------------------------------------------------------- errors
struct Error {
    int code;
    std::string msg;
};

void set_error(int code, const std::string& msg);
int fail(int code, const std::string& msg);           // set_error + return code
extern std::atomic<int64_t> g_launches;

#define HFMM_CUDA(call)                                                                  \
    do {                                                                                 \
        cudaError_t _e = (call);                                                         \
        if (_e != cudaSuccess)                                                           \
            throw hfmm::Error{HFMM_ERR_CUDA, std::string(#call) + ": " +                 \
                                                 cudaGetErrorString(_e)};                \
    } while (0)

// Every kernel launch goes through this: counts it and checks launch errors.
#define HFMM_LAUNCH(kernel, grid, block, smem, stream, ...)                              \
    do {                                                                                 \
        kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);                      \
        hfmm::g_launches.fetch_add(1, std::memory_order_relaxed);                        \
        cudaError_t _e = cudaGetLastError();                                             \
        if (_e != cudaSuccess)                                                           \
            throw hfmm::Error{HFMM_ERR_CUDA, std::string("launch ") + #kernel + ": " +   \
                                                 cudaGetErrorString(_e)};                \
    } while (0)

// Device error flag bits (kernels OR these into plan->d_err).
enum : int {
    ERRF_BOUNDS = 1,      // an index left its buffer (access skipped)
    ERRF_CAPACITY = 2,    // a device-side capacity was exceeded
    ERRF_TIMEOUT = 4,     // a bounded wait gave up (the kernel drained and returned)
};

// ---------------------------------------------------------------- device memory
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        HFMM_CUDA(cudaMalloc((void**)&p, count * sizeof(T)));
        n = count;
    }
    void zero(cudaStream_t s = 0) { HFMM_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

constexpr int MAX_LEVELS = 16;
constexpr int N_DISP = 343;        // (dx, dy, dz) in [-3, 3]^3
constexpr int M2L_ENTRIES = N_DISP + 8;   // 343 displacement slots + 8 L2L octant slots
constexpr int GRID_MAX_LEVEL = 5;  // densest level kept as a dense box grid (32^3 boxes)

// Per-level, per-family operator tables in the GEMM layout (A^T, k-major,
// leading dimension ld, zero padded): out_col = A @ in_col.
struct LevelTables {
    DevBuf<double> up_U, up_d, up_Vt;   // decode: y = d .* (U^T x); z = Vt^T y
    DevBuf<double> dn_U, dn_d, dn_Vt;
    DevBuf<double> m2m;                 // 8 x (A^T) for this level as PARENT
    DevBuf<double> l2l;                 // 8 x (A^T) for this level as CHILD
    DevBuf<double> m2l;                 // 316 x (A^T), non-adjacent displacements
    // rotation-based M2L (m2l_rotation.cu): multipole-from-equivalent Q, check-from-local
    // E (complex, interleaved) and the coaxial shift matrices of every distance
    DevBuf<double> rot_Q, rot_E, rot_C;
    double rot_pref = 0.0;
    // mixed path: TF32 hi/lo halves of M2L and L2L as A[m][k] (fp32 containers)
    DevBuf<float> m2l_hi, m2l_lo, l2l_hi, l2l_lo;
    // compressed M2L of the mixed path, K_d ~ U C_d U^T (rank cr): the K side padded
    // to ckld (>= 32), the M side to cmld (>= 128, the MMA tile), both multiples of 32
    int cr = 0, ckld = 0, cmld = 0;
    DevBuf<double> c_cmp, c_exp;   // A^T of U^T (ld -> ckld) and of U (cmld -> ld)
    DevBuf<float> c_hi, c_lo;      // C_d halves as A [316][cmld][ckld]
    DevBuf<double> xc, yc;         // the level's compressed densities [.][R][ckld] and
    DevBuf<float> xc_hi, xc_lo;    // check potentials [.][R][cmld] (box - level_lo first)
    // a complete level's split densities as a dense box grid [x][y][z][2][ckld] (complex
    // charges): a target tile's sources at one displacement are then one strided TMA box
    int grid = 0;                  // grid side 2^level when the grid is in use, else 0
    DevBuf<float> xg_hi, xg_lo;
    // the low-rank plan's folded tables (row-major right multipliers, zero padded):
    // the decodes' Vt and U taken into the operators next to them, so a box keeps its
    // densities as scaled SVD coordinates (d .* (U^T x)) through both passes
    DevBuf<double> m2m_f;          // 8 x Vt_up(l+1) M2M^T U_up(l), this level as PARENT
    DevBuf<double> l2l_f;          // 8 x Vt_dn(l-1) L2L^T U_dn(l), this level as CHILD
    DevBuf<double> cmp_f, exp_f;   // Vt_up(l) c_cmp (ld x ckld); c_exp U_dn(l) (cmld x ld)
    bool set = false;
    void reset() {
        up_U.release(); up_d.release(); up_Vt.release();
        dn_U.release(); dn_d.release(); dn_Vt.release();
        m2m.release(); l2l.release(); m2l.release();
        m2l_hi.release(); m2l_lo.release(); l2l_hi.release(); l2l_lo.release();
        cr = ckld = cmld = 0;
        c_cmp.release(); c_exp.release(); c_hi.release(); c_lo.release();
        rot_Q.release(); rot_E.release(); rot_C.release();
        xc.release(); yc.release(); xc_hi.release(); xc_lo.release();
        grid = 0;
        xg_hi.release(); xg_lo.release();
        m2m_f.release(); l2l_f.release(); cmp_f.release(); exp_f.release();
        set = false;
    }
};

struct hfmm_plan_impl;

}  // namespace hfmm

struct hfmm_plan {
    int device = 0;
    // problem
    int64_t n = 0;
    int n_max = 0, md = 0, maxleaf = 0;
    bool md_given = false;
    // moving geometry: the domain cube [pmin, pmin + extent]^3 is given, not measured, so
    // the level scales (and the operator tables) stay valid when the points move
    bool domain_fixed = false;
    // the kernel seam: false, the Helmholtz components cos|sin(kr)/r (one or two
    // families); true, the screened-Coulomb kernel exp(-k r) / (4 pi r), k = kappa >= 0
    // (one family; kappa = 0: Laplace)
    bool yukawa = false;
    double extent = 0, pmin[3] = {0, 0, 0};
    int64_t ref_max_boxes = 0;     // the reference's buffer size (reporting only)
    int64_t nb = 0;                // active boxes
    int64_t n_leaves = 0;
    bool adaptive = false;
    int level_lo[hfmm::MAX_LEVELS] = {0}, level_hi[hfmm::MAX_LEVELS] = {0};

    // particles (Morton-sorted order == leaf-major order)
    hfmm::DevBuf<double> pos_s;       // 3 x n SoA (x | y | z)
    hfmm::DevBuf<float> pos_f;        // 6 x n: hi(x|y|z) then lo(x|y|z), pos = hi + lo
    hfmm::DevBuf<int32_t> sort_idx;   // sorted slot -> original index
    hfmm::DevBuf<int32_t> rank;       // original index -> sorted slot

    // boxes
    hfmm::DevBuf<uint64_t> m_id;
    hfmm::DevBuf<int32_t> p_id, lvls, counts, leaf_start;
    hfmm::DevBuf<uint8_t> is_leaf;
    hfmm::DevBuf<double> centre;      // 3 x nb SoA
    hfmm::DevBuf<double> hbox;        // nb
    hfmm::DevBuf<double> rmax;        // per box: sqrt(max |x|^2 over its padded slots)
    std::vector<uint64_t> h_m_id;     // host copies of small box metadata
    std::vector<int32_t> h_lvls, h_counts, h_p_id;
    std::vector<uint8_t> h_is_leaf;

    // kernel + tables
    double k = 0;
    int p = 0, n_s = 0, ld = 0, n_fam = 0;
    hfmm::DevBuf<double> equiv_pts, check_pts;   // unit surfaces, 3 x n_s SoA
    hfmm::LevelTables tables[2][hfmm::MAX_LEVELS];   // [family][level]

    // lists (device, (len x 2) int32)
    hfmm::DevBuf<int32_t> V, U, W, X, near;
    int64_t nV = 0, nU = 0, nW = 0, nX = 0, nNear = 0;

    // schedules
    hfmm::DevBuf<int32_t> leaves;                 // leaf box ids
    hfmm::DevBuf<int32_t> near_off, near_src;     // CSR over leaves (index into `leaves`)
    hfmm::DevBuf<int32_t> w_tgt, w_off, w_src;    // W CSR: target leaves with W sources
    hfmm::DevBuf<int32_t> x_tgt, x_off, x_src;    // X CSR: target boxes with X sources
    int64_t n_w_tgt = 0, n_x_tgt = 0;
    hfmm::DevBuf<int32_t> m2l_src;                // nb x M2L_ENTRIES source boxes (-1 = none)
    hfmm::DevBuf<int32_t> m2m_src;                // nb x 8 child boxes (-1 = none)
    // per level tile lists (targets, -1 padded) for the GEMM phases
    struct Tiles {
        hfmm::DevBuf<int32_t> tgt;
        int ntiles = 0;
    };
    Tiles m2m_tiles[hfmm::MAX_LEVELS][2];   // [level][R-1]
    Tiles dn_tiles[hfmm::MAX_LEVELS][2];
    Tiles dec_tiles[hfmm::MAX_LEVELS][2];
    Tiles leaf_tiles[hfmm::MAX_LEVELS][2];  // the level's leaves only
    Tiles mx_tiles[hfmm::MAX_LEVELS][2];    // mixed M2L tiles: 128 / R targets, by octant
    // complete levels, complex charges: tiles of one octant of a 4 x 4 x 4 block of
    // parents (target j = (x * 4 + y) * 4 + z at grid org + 2 (x, y, z)), origins per tile
    Tiles gx_tiles[hfmm::MAX_LEVELS];
    hfmm::DevBuf<int32_t> gx_org[hfmm::MAX_LEVELS];
    hfmm::DevBuf<int32_t> disp_compact;     // 343 -> M2L table index or -1
    hfmm::DevBuf<float> e_hi, e_lo, l_hi, l_lo;   // split densities [fam][box][R][ld]
    void* mx_maps = nullptr;                // MixedMaps per level (host array)
    bool compressed = false;                // every level has a compressed M2L (mixed path)
    void* cx_maps = nullptr;                // MixedMaps [2][MAX_LEVELS] of the C_d tables
    void* cxq[2] = {nullptr, nullptr};      // PlanQueue per charge-column count (finalize)
    bool queue_m2l = true;                  // run the low-rank M2L as the plan's queue
    cudaStream_t nf_side = nullptr;         // the near field's stream (runs beside the far field)
    cudaStream_t crit = nullptr;            // highest-priority stream of the far-field chain
    cudaEvent_t crit_fork = nullptr, crit_join = nullptr;
    cudaEvent_t nf_fork = nullptr, nf_join = nullptr;
    static constexpr int CX_STREAMS = 4;    // side streams of the concurrent compressed M2L
    cudaStream_t cx_side[CX_STREAMS] = {};
    cudaEvent_t cx_fork = nullptr, cx_join[CX_STREAMS] = {};
    cudaEvent_t cx_level[hfmm::MAX_LEVELS][2] = {};   // a level's M2L + expansion is done
    bool mixed_ready = false;
    // streamed M2L tables: regenerated per level and evaluate into a workspace
    // (the plan's own, or one bound by the caller and shared by plans that run in turn)
    bool streamed = false;
    void* ws = nullptr;
    size_t ws_bytes = 0;
    hfmm::DevBuf<double> ws_own;
    struct hfmm_batch* batch_owner = nullptr;   // the batch whose workspace and graph use this plan
    hfmm::DevBuf<const double*> a_ptrs;     // device arrays of A pointers per GEMM call
    std::vector<const double*> h_a_ptrs;
    size_t a_ptr_cursor = 0;

    // evaluate scratch (allocated at finalize for R = 2)
    hfmm::DevBuf<double> q_s;        // R x n sorted charges
    hfmm::DevBuf<double> check, equiv, loc, tmp;   // [fam][box][R][ld]
    hfmm::DevBuf<double> gemm_part;  // partial tiles of the main stream's split GEMMs
    int rot_P = 0, rot_n_dist = 0, rot_n_theta = 0;   // rotation-based M2L of the FP64 evaluate (0: dense)
    hfmm::DevBuf<double> rot_D;      // real y-rotation blocks per polar angle, then transposed
    hfmm::DevBuf<int32_t> rot_theta; // polar angle index per slot
    hfmm::DevBuf<double> rot_phase;  // e^{i m phi} per slot (complex)
    hfmm::DevBuf<int32_t> rot_dist;  // coaxial matrix per slot
    hfmm::DevBuf<double> rot_M;      // multipole work array of one level
    hfmm::DevBuf<double> pot;        // per sorted particle: [fam][R] potentials
    hfmm::DevBuf<double> fld;        // per sorted particle: [fam][R][3]
    hfmm::DevBuf<int> d_err;
    bool finalized = false;
};

namespace hfmm {

// ---------------------------------------------------------------- host entry points
void tree_build(hfmm_plan* P, const double* pos_dev);
void lists_build(hfmm_plan* P);
void schedules_build(hfmm_plan* P);
void upload_level(hfmm_plan* P, int fam, int level, const double* const* h);
void generate_tables(hfmm_plan* P, int fam, int level);
size_t stream_ws_bytes(const hfmm_plan* P);
bool plan_profiling(hfmm_plan* P);
void batch_forget_plan(struct hfmm_batch* B, hfmm_plan* P);
void generate_m2l_stream(hfmm_plan* P, int level, bool mixed, void* ws, cudaStream_t s);
void compressed_prepare(hfmm_plan* P);   // finalize: buffers, tensor maps, side streams
void compressed_release(hfmm_plan* P);   // plan destroy: side streams and events
// phase: EVAL_ALL; or the two halves of a batch whose low-rank M2L runs from one queue
// (m2l_queue): EVAL_UP ends after the levels' compressed densities, EVAL_DOWN starts
// with the expansions of the queue's check potentials
enum { EVAL_UP = 1, EVAL_DOWN = 2, EVAL_ALL = 3 };
void evaluate_fp64(hfmm_plan* P, const double* q_re, const double* q_im, double* phi,
                   double* fld, cudaStream_t s, bool mixed = false, int phase = EVAL_ALL);
void direct_sum(const double* pos, const double* q_re, const double* q_im, int64_t n,
                const int32_t* targets, int64_t n_t, double k, double* phi, double* fld,
                double* scratch, int n_split, cudaStream_t s, int* err, int yukawa = 0);
int direct_splits(int64_t n, int64_t n_t);

// ---------------------------------------------------------------- GEMM launcher
// out[t][r][m] (+)= scale[m] * sum_e sum_k A_e[m][k] * B_e[src(t,e)][r][k]
struct GemmCall {
    const int32_t* tile_tgt;   // ntiles x TT target boxes (-1 = empty slot)
    int ntiles;
    const int32_t* src_tab;    // nullptr: src = target (one entry); else src_tab[t*src_ld + e]
    int src_ld;
    int n_entries;
    int b_split;               // entries >= b_split read B1, others B0
    const double* const* A;    // device array of n_entries A^T pointers (nullptr = skip entry)
    const double* B0;
    const double* B1;
    double* out;
    const double* scale;       // nullable, length ld
    const double* scale_f1;    // family 1's scale when it differs (nullable: scale)
    int accumulate;            // 1: out += result, 0: out = result
    int R;
    int ld;                    // padded n_s (multiple of 16)
    int ldk, ldm;              // rectangular calls: K extent / B row length and M extent /
                               // out row length (0: both ld); A^T is ldk x ldm
    int k_valid;               // rows of A^T that can be nonzero (0: ldk); the K loop stops
                               // after the last chunk that holds one
    int n_s;
    int64_t fam_stride;        // elements between the families' B/out arrays
    int64_t a_fam_stride;      // entries between the families' A pointer sets
    int n_fam;
    int64_t nb;                // box count (bounds checks)
    double* part;              // nullable: scratch for entry splits of small grids
    int64_t part_cap;          // its size in doubles
    int n_split;               // set by gemm_f64: CTAs per output tile (entry ranges)
};
void gemm_f64(const GemmCall& c, int* d_err, cudaStream_t s);
int sm_count();   // multiprocessors of the current device (read once)
// rotation-based M2L of level l into the check potentials (m2l_rotation.cu)
void rot_m2l(hfmm_plan* P, int l, int R, int64_t fam_stride, cudaStream_t s);
void rot_check(const hfmm_plan* P);   // throws when the rotation M2L cannot run
size_t rot_workspace_doubles(const hfmm_plan* P);
constexpr int64_t GEMM_PART_CAP = 768LL * 64 * 64;   // doubles: 768 partial 64 x 64 tiles

// ---------------------------------------------------------------- device helpers
__host__ __device__ inline uint64_t expand_bits(uint64_t v) {
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}
__host__ __device__ inline uint64_t compact_bits(uint64_t v) {
    v &= 0x1249249249249249ull;
    v = (v | (v >> 2)) & 0x10C30C30C30C30C3ull;
    v = (v | (v >> 4)) & 0x100F00F00F00F00Full;
    v = (v | (v >> 8)) & 0x1F0000FF0000FFull;
    v = (v | (v >> 16)) & 0x1F00000000FFFFull;
    v = (v | (v >> 32)) & 0x1FFFFFull;
    return v;
}
__host__ __device__ inline uint64_t morton3(uint64_t x, uint64_t y, uint64_t z) {
    return expand_bits(x) | (expand_bits(y) << 1) | (expand_bits(z) << 2);
}
__host__ __device__ inline void demorton3(uint64_t m, int64_t& x, int64_t& y, int64_t& z) {
    x = (int64_t)compact_bits(m);
    y = (int64_t)compact_bits(m >> 1);
    z = (int64_t)compact_bits(m >> 2);
}

// The 26 neighbour offsets, dx outer / dz inner, centre removed (cubic.py:48-51).
__host__ __device__ inline void neigh_offset(int d, int& dx, int& dy, int& dz) {
    int f = d < 13 ? d : d + 1;
    dx = f / 9 - 1;
    dy = (f / 3) % 3 - 1;
    dz = f % 3 - 1;
}

// Throws unless p is memory a kernel on the current device may dereference.
inline void require_device_ptr(const void* p, const char* what) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        throw Error{HFMM_ERR_ARG, std::string(what) + ": not a CUDA pointer"};
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged &&
        !(a.type == cudaMemoryTypeHost && a.devicePointer != nullptr))
        throw Error{HFMM_ERR_ARG, std::string(what) + ": not device-accessible memory"};
}

inline int round_up(int v, int m) { return (v + m - 1) / m * m; }
inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace hfmm
