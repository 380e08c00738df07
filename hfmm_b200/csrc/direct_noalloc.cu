// Allocation-free direct-sum referee: hfmm_direct_noalloc.
//
// Some callers cannot allocate device memory while they run: a JAX/XLA program
// (the reference's own runtime) preallocates most of the GPU for its allocator
// and calls foreign code inside that budget, where a cudaMalloc can fail or
// fragment memory the host framework owns. hfmm_direct allocates its partial-sum
// scratch per call, so this variant keeps the scratch in a fixed file-scope
// device array instead.
//
// The array is NOALLOC_SCRATCH_DOUBLES doubles (8 MiB). It is part of this
// library's device image, so every GPU that loads the library holds it until the
// process exits. Every call shares it and it keeps the last call's contents:
// calls that overlap on the GPU (two streams, two threads) race on it. The
// partial sums are fully written before they are read, so only the error word is
// cleared per call. The call waits for its stream to finish (it reads the error
// word back), like hfmm_direct.
#include "hfmm_internal.cuh"

#include <algorithm>
#include <mutex>

namespace {

constexpr size_t NOALLOC_SCRATCH_DOUBLES = (size_t)1 << 20;   // 8 MiB
constexpr int MAX_DEVICES = 64;

__device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];
__device__ __align__(256) int g_noalloc_err;

// Device addresses of the two arrays, looked up once per device with that device
// current. In host code the symbols are host-side stand-ins, never valid device
// addresses, so kernels always get the looked-up pointers.
struct NoallocSymbols {
    std::mutex mu;
    double* scratch[MAX_DEVICES] = {};
    int* err[MAX_DEVICES] = {};
};

NoallocSymbols& symbols() {
    static NoallocSymbols s;
    return s;
}

void device_symbols(double** scratch, int** err) {
    int dev = -1;
    HFMM_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES)
        throw hfmm::Error{HFMM_ERR_CAPACITY, "hfmm_direct_noalloc: device ordinal above 63"};
    NoallocSymbols& s = symbols();
    std::lock_guard<std::mutex> g(s.mu);
    if (!s.scratch[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw hfmm::Error{HFMM_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") +
                                                 cudaGetErrorString(e)};
        void* q = nullptr;
        e = cudaGetSymbolAddress(&q, g_noalloc_err);
        if (e != cudaSuccess || !q)
            throw hfmm::Error{HFMM_ERR_CUDA, std::string("cudaGetSymbolAddress(err): ") +
                                                 cudaGetErrorString(e)};
        s.scratch[dev] = static_cast<double*>(p);
        s.err[dev] = static_cast<int*>(q);
    }
    *scratch = s.scratch[dev];
    *err = s.err[dev];
}

}  // namespace

extern "C" int hfmm_direct_noalloc(const double* pos, const double* q_re, const double* q_im,
                                   int64_t n, const int32_t* targets, int64_t n_t, double k,
                                   double* phi, double* fld, void* stream) {
    using namespace hfmm;
    if (!pos || !q_re || !targets || !phi || n <= 0 || n_t < 0)
        return fail(HFMM_ERR_ARG, "invalid direct-sum arguments");
    if (!std::isfinite(k)) return fail(HFMM_ERR_ARG, "k must be finite");
    // 8 partial sums per target and source split must fit the fixed scratch
    const int64_t per_split = std::max<int64_t>(n_t, 1) * 8;
    const int64_t max_split = (int64_t)NOALLOC_SCRATCH_DOUBLES / per_split;
    if (max_split < 1)
        return fail(HFMM_ERR_CAPACITY,
                    "hfmm_direct_noalloc: at most " +
                        std::to_string(NOALLOC_SCRATCH_DOUBLES / 8) + " targets per call, got " +
                        std::to_string(n_t));
    try {
        require_device_ptr(pos, "positions");
        require_device_ptr(q_re, "q_re");
        if (q_im) require_device_ptr(q_im, "q_im");
        require_device_ptr(targets, "targets");
        require_device_ptr(phi, "phi_out");
        if (fld) require_device_ptr(fld, "field_out");
        const int splits = (int)std::min<int64_t>(direct_splits(n, n_t), max_split);
        double* scratch = nullptr;
        int* err = nullptr;
        device_symbols(&scratch, &err);
        cudaStream_t s = (cudaStream_t)stream;
        HFMM_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
        direct_sum(pos, q_re, q_im, n, targets, n_t, k, phi, fld, scratch, splits, s, err);
        int h = 0;
        HFMM_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s));
        HFMM_CUDA(cudaStreamSynchronize(s));
        if (h) return fail(HFMM_ERR_ARG, "target index out of range");
        return HFMM_OK;
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    } catch (...) {
        return fail(HFMM_ERR_STATE, "hfmm_direct_noalloc failed");
    }
}
