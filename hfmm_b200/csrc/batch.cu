// Batched evaluate: many independent problems (plans of uneven size and
// wavenumber) in one CUDA-graph launch. No counterpart in the reference, which
// evaluates one problem per call (HFMM.py:83-91).
//
// The plans are spread over S streams by longest-processing-time-first on an
// estimate of each plan's work (M2L GEMM FLOPs + near-field pairs); each stream
// evaluates its plans in turn, so small problems overlap the tails of large ones.
// Plans that stream their M2L tables share one workspace per stream (sized for
// the largest of them), which bounds the table memory of the whole batch by S
// workspaces. The whole batch -- fork, every evaluate, join -- is captured once
// into a graph; a launch replays it with the charge and output pointers given
// before capture.
// Queued M2L: when every problem runs the low-rank mixed evaluate with the same
// number of charge columns, the graph runs every plan's upward half, then one
// persistent M2L kernel (m2l_queue.cu) over a device queue of every plan's M2L work
// (tile x row block of each level and family), largest first, then every plan's
// downward half: the small problems' few tiles no longer run as separate launches.
#include "hfmm_internal.cuh"
#include "mixed.cuh"

#include <algorithm>
#include <memory>
#include <numeric>
#include <vector>

struct hfmm_batch {
    int device = 0;
    std::vector<hfmm_plan*> plans;
    std::vector<int> stream_of;                 // plan -> stream
    std::vector<std::vector<int>> order;        // stream -> plans in launch order
    std::vector<double> cost;
    struct Io {
        const double *q_re = nullptr, *q_im = nullptr;
        double *phi = nullptr, *E = nullptr;
        int precision = 0;
        bool set = false;
        // optional in-graph check against the FP64 direct sum at sampled targets
        const double* pos = nullptr;          // n x 3, input order
        const int32_t* tg = nullptr;
        int n_t = 0, n_split = 1;
        double* sums = nullptr;               // 4 doubles, written by every launch
        hfmm::DevBuf<double> ref, scratch;    // direct-sum values and partial sums
    };
    std::vector<std::unique_ptr<Io>> io_;   // one per plan (Io owns device buffers)
    Io& io(int i) { return *io_[i]; }
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;            // [0] fork, [1 + s] join of stream s
    std::vector<hfmm::DevBuf<double>> ws;       // per stream (streamed plans only)
    // queued M2L (see above): calls, tensor maps and items in device memory
    bool queue_on = true;                       // use the queue when the problems allow it
    bool queued = false;                        // the captured graph uses it
    std::string queue_note;                     // why the last capture did not use it
    int queue_R = 0, n_items = 0;
    hfmm::DevBuf<hfmm::MixedCall> q_calls;
    hfmm::DevBuf<hfmm::MixedMaps> q_maps;
    hfmm::DevBuf<hfmm::M2LItem> q_items;
    hfmm::DevBuf<int> q_next;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    ~hfmm_batch() {
        if (!streams.empty()) cudaStreamSynchronize(streams[0]);
        drop_graph();
        // release the plans: a streaming plan falls back to its own workspace,
        // allocated at its next evaluate
        for (auto* P : plans) {
            if (!P) continue;
            if (P->streamed) {
                P->ws = nullptr;
                P->ws_bytes = 0;
            }
            P->batch_owner = nullptr;
        }
        for (auto e : events) cudaEventDestroy(e);
        for (auto s : streams) cudaStreamDestroy(s);
    }
};

namespace hfmm {

namespace {

// Squared-norm sums of the check: sums = (sum |phi - phi_ref|^2, sum |phi_ref|^2,
// sum |E - E_ref|^2, sum |E_ref|^2) over the sampled targets (E terms 0 without a
// field). One CTA, fixed-order tree reduction: the sums are deterministic.
__global__ void __launch_bounds__(256) k_check_sums(const double* __restrict__ phi,
                                                    const double* __restrict__ E,
                                                    const int32_t* __restrict__ tg, int n_t,
                                                    int64_t n, const double* __restrict__ rphi,
                                                    const double* __restrict__ rE, double* sums,
                                                    int* err) {
    __shared__ double red[4][256];
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (int t = threadIdx.x; t < n_t; t += blockDim.x) {
        const int64_t i = tg[t];
        if (i < 0 || i >= n) {
            atomicOr(err, ERRF_BOUNDS);
            continue;
        }
        for (int c = 0; c < 2; ++c) {
            const double r = rphi[2 * t + c], d = phi[2 * i + c] - r;
            a[0] += d * d;
            a[1] += r * r;
        }
        if (E)
            for (int c = 0; c < 6; ++c) {
                const double r = rE[6 * t + c], d = E[6 * i + c] - r;
                a[2] += d * d;
                a[3] += r * r;
            }
    }
    for (int v = 0; v < 4; ++v) red[v][threadIdx.x] = a[v];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int v = 0; v < 4; ++v) red[v][threadIdx.x] += red[v][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 4) sums[threadIdx.x] = red[threadIdx.x][0];
}

// Work estimate of one evaluate (complex charges): far field M2L+L2L FLOPs and
// near-field pairs weighted by ~40 flops each; only the relative size matters.
// The queued M2L's work list (before capture, queue_items): every plan's low-rank M2L
// calls and their tensor maps, one item per tile and 128-row block, largest first.
// Off when a problem is not a low-rank mixed evaluate or the column counts differ.
void build_queue(hfmm_batch* B) {
    B->queued = false;
    B->queue_note.clear();
    if (!B->queue_on) {
        B->queue_note = "the queue is switched off";
        return;
    }
    int R = 0;
    for (size_t i = 0; i < B->plans.size(); ++i) {
        hfmm_plan* P = B->plans[i];
        const auto& io = B->io((int)i);
        const int r = io.q_im ? 2 : 1;
        // (a plan streaming its dense M2L tables is fine: only its FP64 evaluate reads them)
        const std::string who = "problem " + std::to_string(i);
        if (io.precision != HFMM_PREC_MIXED) B->queue_note = who + " runs the FP64 evaluate";
        else if (!P->compressed) B->queue_note = who + " has no low-rank M2L tables";
        else if (!P->mixed_ready) B->queue_note = who + " has no mixed-precision buffers";
        else if (R && r != R) B->queue_note = who + " has other charge columns than problem 0";
        if (!B->queue_note.empty()) return;
        R = r;
    }
    std::vector<MixedCall> calls;
    std::vector<MixedMaps> maps;
    std::vector<M2LItem> items;
    B->queue_note = queue_items(B->plans.data(), (int)B->plans.size(), R, calls, maps, items);
    if (!B->queue_note.empty()) return;
    B->q_calls.alloc(calls.size());
    B->q_maps.alloc(maps.size());
    B->q_items.alloc(items.size());
    B->q_next.alloc(1);
    HFMM_CUDA(cudaMemcpy(B->q_calls.p, calls.data(), calls.size() * sizeof(MixedCall), cudaMemcpyHostToDevice));
    HFMM_CUDA(cudaMemcpy(B->q_maps.p, maps.data(), maps.size() * sizeof(MixedMaps), cudaMemcpyHostToDevice));
    HFMM_CUDA(cudaMemcpy(B->q_items.p, items.data(), items.size() * sizeof(M2LItem), cudaMemcpyHostToDevice));
    B->n_items = (int)items.size();
    B->queue_R = R;
    B->queued = true;
}

double plan_cost(const hfmm_plan* P) {
    const double ns = P->n_s;
    const double far = 2.0 * ns * ns * 2.0 * P->n_fam * ((double)P->nV + 8.0 * P->nb);
    const double occ = P->n_leaves ? (double)P->n / P->n_leaves : 0.0;
    const double near = 40.0 * (double)P->nNear * occ * occ;
    return far + near + 1e6;   // + a launch-overhead floor
}

}  // namespace

}  // namespace hfmm

using namespace hfmm;

extern "C" {

int hfmm_batch_create(hfmm_plan* const* plans, int32_t n_plans, int32_t n_streams,
                      hfmm_batch** out) {
    if (!out) return fail(HFMM_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!plans || n_plans <= 0) return fail(HFMM_ERR_ARG, "no plans");
    if (n_streams < 1 || n_streams > 64) return fail(HFMM_ERR_ARG, "n_streams must be in [1, 64]");
    int dev = -1;
    for (int i = 0; i < n_plans; ++i) {
        if (!plans[i]) return fail(HFMM_ERR_ARG, "plan is NULL");
        if (!plans[i]->finalized) return fail(HFMM_ERR_STATE, "every plan must be finalized");
        if (dev >= 0 && plans[i]->device != dev)
            return fail(HFMM_ERR_ARG, "plans of one batch must live on one device");
        dev = plans[i]->device;
        for (int j = 0; j < i; ++j)
            if (plans[j] == plans[i]) return fail(HFMM_ERR_ARG, "a plan appears twice");
        if (plans[i]->batch_owner) return fail(HFMM_ERR_STATE, "a plan already belongs to a batch");
    }
    hfmm_batch* B = new hfmm_batch();
    try {
        B->device = dev;
        HFMM_CUDA(cudaSetDevice(dev));
        B->plans.assign(plans, plans + n_plans);
        for (auto* P : B->plans) P->batch_owner = B;
        const int S = std::min<int>(n_streams, n_plans);
        B->cost.resize(n_plans);
        for (int i = 0; i < n_plans; ++i) B->cost[i] = plan_cost(plans[i]);
        std::vector<int> idx(n_plans);
        std::iota(idx.begin(), idx.end(), 0);
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return B->cost[a] > B->cost[b]; });
        std::vector<double> load(S, 0.0);
        B->order.assign(S, {});
        B->stream_of.assign(n_plans, 0);
        for (int i : idx) {   // LPT: the next largest plan goes to the least loaded stream
            const int s = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            load[s] += B->cost[i];
            B->order[s].push_back(i);
            B->stream_of[i] = s;
        }
        for (int i = 0; i < n_plans; ++i) B->io_.push_back(std::make_unique<hfmm_batch::Io>());
        B->streams.resize(S);
        for (auto& s : B->streams) HFMM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        B->events.resize(S + 1);
        for (auto& e : B->events) HFMM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        // one M2L-table workspace per stream, shared by the streamed plans on it
        B->ws = std::vector<DevBuf<double>>(S);
        for (int s = 0; s < S; ++s) {
            size_t need = 0;
            for (int i : B->order[s])
                if (plans[i]->streamed) need = std::max(need, stream_ws_bytes(plans[i]));
            if (!need) continue;
            B->ws[s].alloc(need / sizeof(double));
            for (int i : B->order[s]) {
                if (!plans[i]->streamed) continue;
                int rc = hfmm_plan_bind_workspace(plans[i], B->ws[s].p, (int64_t)need);
                if (rc != HFMM_OK) throw Error{rc, hfmm_last_error()};
            }
        }
        *out = B;
        return HFMM_OK;
    } catch (const Error& e) {
        delete B;
        return fail(e.code, e.msg);
    }
}

int hfmm_batch_stream_of(const hfmm_batch* B, int32_t i) {
    if (!B || i < 0 || i >= (int)B->plans.size()) return fail(HFMM_ERR_ARG, "bad batch or index");
    return B->stream_of[i];
}

int hfmm_batch_set_problem(hfmm_batch* B, int32_t i, const double* q_re_dev, const double* q_im_dev,
                           double* phi_out_dev, double* field_out_dev, int32_t precision) {
    if (!B || i < 0 || i >= (int)B->plans.size()) return fail(HFMM_ERR_ARG, "bad batch or index");
    if (!B->plans[i]) return fail(HFMM_ERR_STATE, "the plan was destroyed");
    if (!q_re_dev || !phi_out_dev) return fail(HFMM_ERR_ARG, "charges and output are required");
    if (precision != HFMM_PREC_FP64 && precision != HFMM_PREC_MIXED)
        return fail(HFMM_ERR_ARG, "precision must be HFMM_PREC_FP64 or HFMM_PREC_MIXED");
    try {
        require_device_ptr(q_re_dev, "q_re");
        if (q_im_dev) require_device_ptr(q_im_dev, "q_im");
        require_device_ptr(phi_out_dev, "phi_out");
        if (field_out_dev) require_device_ptr(field_out_dev, "field_out");
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    }
    auto& io = B->io(i);
    io.q_re = q_re_dev;
    io.q_im = q_im_dev;
    io.phi = phi_out_dev;
    io.E = field_out_dev;
    io.precision = precision;
    io.set = true;
    B->drop_graph();   // pointers changed: the graph must be captured again
    return HFMM_OK;
}

int hfmm_batch_set_check(hfmm_batch* B, int32_t i, const double* pos_dev,
                         const int32_t* targets_dev, int32_t n_t, double* sums_dev) {
    if (!B || i < 0 || i >= (int)B->plans.size()) return fail(HFMM_ERR_ARG, "bad batch or index");
    if (!B->plans[i]) return fail(HFMM_ERR_STATE, "the plan was destroyed");
    if (!pos_dev || !targets_dev || !sums_dev || n_t <= 0)
        return fail(HFMM_ERR_ARG, "positions, targets and sums are required");
    try {
        require_device_ptr(pos_dev, "positions");
        require_device_ptr(targets_dev, "targets");
        require_device_ptr(sums_dev, "sums");
        HFMM_CUDA(cudaSetDevice(B->device));
        auto& io = B->io(i);
        io.pos = pos_dev;
        io.tg = targets_dev;
        io.n_t = n_t;
        io.sums = sums_dev;
        io.n_split = direct_splits(B->plans[i]->n, n_t);
        io.ref.alloc((size_t)8 * n_t);
        io.ref.zero();
        io.scratch.alloc((size_t)io.n_split * n_t * 8);
        B->drop_graph();
        return HFMM_OK;
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    }
}

int hfmm_batch_capture(hfmm_batch* B) {
    if (!B) return fail(HFMM_ERR_ARG, "batch is NULL");
    for (auto& io : B->io_)
        if (!io->set) return fail(HFMM_ERR_STATE, "every problem needs its charges and outputs");
    for (auto* P : B->plans) {
        if (!P) return fail(HFMM_ERR_STATE, "a plan of the batch was destroyed");
        if (plan_profiling(P)) return fail(HFMM_ERR_STATE, "turn profiling off before capture");
        if (P->streamed && !P->ws) return fail(HFMM_ERR_STATE, "a streaming plan has no workspace");
    }
    try {
        HFMM_CUDA(cudaSetDevice(B->device));
        B->drop_graph();
        const int S = (int)B->streams.size();
        cudaStream_t s0 = B->streams[0];
        build_queue(B);
        HFMM_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeRelaxed));
        try {
            HFMM_CUDA(cudaEventRecord(B->events[0], s0));
            for (int s = 1; s < S; ++s) HFMM_CUDA(cudaStreamWaitEvent(B->streams[s], B->events[0], 0));
            if (B->queued) {   // every plan's upward half, then the queued M2L of all of them
                for (int s = 0; s < S; ++s)
                    for (int i : B->order[s]) {
                        auto& io = B->io(i);
                        evaluate_fp64(B->plans[i], io.q_re, io.q_im, io.phi, io.E, B->streams[s], true,
                                      EVAL_UP);
                    }
                for (int s = 1; s < S; ++s) {
                    HFMM_CUDA(cudaEventRecord(B->events[1 + s], B->streams[s]));
                    HFMM_CUDA(cudaStreamWaitEvent(s0, B->events[1 + s], 0));
                }
                int sms = 148;
                HFMM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, B->device));
                m2l_queue(B->q_calls.p, B->q_maps.p, B->q_items.p, B->n_items, B->q_next.p, B->queue_R,
                          sms, s0, g_m2l_starve.load());
                HFMM_CUDA(cudaEventRecord(B->events[0], s0));
                for (int s = 1; s < S; ++s) HFMM_CUDA(cudaStreamWaitEvent(B->streams[s], B->events[0], 0));
            }
            for (int s = 0; s < S; ++s)
                for (int i : B->order[s]) {
                    auto& io = B->io(i);
                    hfmm_plan* P = B->plans[i];
                    evaluate_fp64(P, io.q_re, io.q_im, io.phi, io.E, B->streams[s],
                                  io.precision == HFMM_PREC_MIXED, B->queued ? EVAL_DOWN : EVAL_ALL);
                    if (io.sums) {   // check the result against the direct sum, in the graph
                        double* rphi = io.ref.p;
                        double* rE = io.ref.p + 2 * io.n_t;
                        direct_sum(io.pos, io.q_re, io.q_im, P->n, io.tg, io.n_t, P->k, rphi,
                                   io.E ? rE : nullptr, io.scratch.p, io.n_split, B->streams[s],
                                   P->d_err.p, P->yukawa ? 1 : 0);
                        HFMM_LAUNCH(k_check_sums, 1, 256, 0, B->streams[s], io.phi, io.E, io.tg,
                                    io.n_t, P->n, rphi, rE, io.sums, P->d_err.p);
                    }
                }
            for (int s = 1; s < S; ++s) {
                HFMM_CUDA(cudaEventRecord(B->events[1 + s], B->streams[s]));
                HFMM_CUDA(cudaStreamWaitEvent(s0, B->events[1 + s], 0));
            }
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s0, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        HFMM_CUDA(cudaStreamEndCapture(s0, &B->graph));
        HFMM_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
        return HFMM_OK;
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    }
}

int hfmm_batch_launch(hfmm_batch* B, void* stream) {
    if (!B) return fail(HFMM_ERR_ARG, "batch is NULL");
    for (auto* P : B->plans)
        if (!P) return fail(HFMM_ERR_STATE, "a plan of the batch was destroyed");
    if (!B->exec) return fail(HFMM_ERR_STATE, "capture the batch first");
    try {
        HFMM_CUDA(cudaGraphLaunch(B->exec, (cudaStream_t)stream));
        return HFMM_OK;
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    }
}

void hfmm_batch_destroy(hfmm_batch* B) { delete B; }

int hfmm_batch_set_queue(hfmm_batch* B, int32_t on) {
    if (!B) return fail(HFMM_ERR_ARG, "batch is NULL");
    B->queue_on = on != 0;
    B->drop_graph();
    return HFMM_OK;
}

int hfmm_batch_queued(const hfmm_batch* B) {
    if (!B) return fail(HFMM_ERR_ARG, "batch is NULL");
    return B->queued ? 1 : 0;
}

const char* hfmm_batch_queue_note(const hfmm_batch* B) {
    return B ? B->queue_note.c_str() : "batch is NULL";
}

}  // extern "C"

namespace hfmm {
// A plan destroyed while its batch lives: the batch drops the plan and its graph.
void batch_forget_plan(hfmm_batch* B, hfmm_plan* P) {
    B->drop_graph();
    for (auto& q : B->plans)
        if (q == P) q = nullptr;
}
}  // namespace hfmm

extern "C" {

}  // extern "C"
