// Mixed batches: the blocks of many captures (NTSC and PAL, each with its
// own context, outputs and length) in one persistent demodulator launch fed
// from a device work queue, optionally replayed from a CUDA graph.  No
// counterpart in the reference, which demodulates one capture's blocks at a
// time (DemodCache.worker, lddecode/core.py:1165-1200); each block's
// arithmetic is that of ldg_demod_blocks, so every output is bit-identical
// to demodulating the captures one by one.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ldg_demod.cuh"
#include "ldg_noalloc.h"
#include "ldgpu.h"

struct ldg_queue {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;   // graph capture and NULL-stream runs
    ldg::DemodParams* d_items = nullptr;
    long long* d_first = nullptr;
    int items_cap = 0;
    unsigned long long* d_head = nullptr;
    float2* d_scratch = nullptr;
    int scratch_ctas = 0;
    const float2* tw16 = nullptr;
    const float2* tw32 = nullptr;
    int nitems = 0;
    long long total = 0;
    int grab = 1;
    int ctas = 0;                    // 0: one per SM
    int variant = -1;                // FFT decomposition; -1: the first item's context's
    int item_variant = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_grid = 0;
    cudaEvent_t done = nullptr;
    bool ran = false;
    std::mutex mu;
};

namespace {

int qfail(int code, const std::string& msg) { return ldg::api_fail(code, msg); }  // ldg_last_error()

#define QCK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return qfail(LDG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct Dev {
    int prev = -1;
    explicit Dev(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~Dev() {
        int cur;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

void drop_graph(ldg_queue* q) {
    if (q->exec) cudaGraphExecDestroy(q->exec);
    if (q->graph) cudaGraphDestroy(q->graph);
    q->exec = nullptr;
    q->graph = nullptr;
}

int wait_idle(ldg_queue* q) {
    if (q->ran) QCK(cudaEventSynchronize(q->done));
    return LDG_OK;
}

int grid_of(const ldg_queue* q) {
    const long long want = q->ctas ? q->ctas : q->sms;
    const long long pops = (q->total + q->grab - 1) / q->grab;
    return (int)(want < pops ? want : pops);
}

}  // namespace

extern "C" {

int ldg_queue_create(ldg_queue** out, int32_t device) {
    if (!out) return qfail(LDG_ERR_ARG, "ldg_queue_create: out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return qfail(LDG_ERR_CUDA, "ldg_queue_create: no CUDA device");
    }
    if (device < 0 || device >= ndev) return qfail(LDG_ERR_ARG, "ldg_queue_create: bad device index");
    Dev g(device);
    ldg_queue* q = new ldg_queue();
    q->device = device;
    cudaDeviceGetAttribute(&q->sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&q->done, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&q->d_head, sizeof(unsigned long long)) != cudaSuccess) {
        const std::string msg = cudaGetErrorString(cudaGetLastError());
        ldg_queue_destroy(q);
        return qfail(LDG_ERR_CUDA, "ldg_queue_create: " + msg);
    }
    *out = q;
    return LDG_OK;
}

void ldg_queue_destroy(ldg_queue* q) {
    if (!q) return;
    Dev g(q->device);
    if (q->ran) cudaEventSynchronize(q->done);
    drop_graph(q);
    cudaFree(q->d_items);
    cudaFree(q->d_first);
    cudaFree(q->d_head);
    cudaFree(q->d_scratch);
    if (q->done) cudaEventDestroy(q->done);
    if (q->stream) cudaStreamDestroy(q->stream);
    delete q;
}

int ldg_queue_submit(ldg_queue* q, const ldg_work_item* items, int32_t n) {
    if (!q || (!items && n)) return qfail(LDG_ERR_ARG, "ldg_queue_submit: NULL argument");
    if (n < 0) return qfail(LDG_ERR_ARG, "ldg_queue_submit: negative item count");
    std::lock_guard<std::mutex> lk(q->mu);
    std::vector<ldg::DemodParams> h(n);
    std::vector<long long> first(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        if (!items[i].ctx) return qfail(LDG_ERR_ARG, "ldg_queue_submit: item " + std::to_string(i) + " has no context");
        if (ldg::ctx_device(items[i].ctx) != q->device)
            return qfail(LDG_ERR_ARG, "ldg_queue_submit: item " + std::to_string(i) + "'s context is on another device");
        const int rc = ldg::device_params(items[i].ctx, &items[i].args,
                                          "ldg_queue_submit (item " + std::to_string(i) + ")", &h[i]);
        if (rc) return rc;
        first[i + 1] = first[i] + items[i].args.nblocks;
    }
    Dev g(q->device);
    int rc = wait_idle(q);
    if (rc) return rc;
    drop_graph(q);
    if (n > q->items_cap) {
        cudaFree(q->d_items);
        cudaFree(q->d_first);
        q->d_items = nullptr;
        q->d_first = nullptr;
        q->items_cap = 0;
        QCK(cudaMalloc(&q->d_items, (size_t)n * sizeof(ldg::DemodParams)));
        QCK(cudaMalloc(&q->d_first, (size_t)(n + 1) * sizeof(long long)));
        q->items_cap = n;
    }
    if (n) {
        QCK(cudaMemcpy(q->d_items, h.data(), (size_t)n * sizeof(ldg::DemodParams), cudaMemcpyHostToDevice));
        QCK(cudaMemcpy(q->d_first, first.data(), (size_t)(n + 1) * sizeof(long long), cudaMemcpyHostToDevice));
        q->tw16 = h[0].tw16;
        q->tw32 = h[0].tw32;
        q->item_variant = h[0].variant;
    }
    q->nitems = n;
    q->total = first[n];
    return LDG_OK;
}

int ldg_queue_set_schedule(ldg_queue* q, int32_t grab, int32_t ctas) {
    if (!q) return qfail(LDG_ERR_ARG, "ldg_queue_set_schedule: NULL queue");
    if (grab < 1 || grab > 64) return qfail(LDG_ERR_ARG, "ldg_queue_set_schedule: grab must be in [1, 64]");
    std::lock_guard<std::mutex> lk(q->mu);
    if (ctas < 0 || ctas > 4 * q->sms)
        return qfail(LDG_ERR_ARG, "ldg_queue_set_schedule: ctas must be in [0, 4 x SMs]");
    if (grab != q->grab || ctas != q->ctas) {
        Dev g(q->device);
        int rc = wait_idle(q);
        if (rc) return rc;
        drop_graph(q);
    }
    q->grab = grab;
    q->ctas = ctas;
    return LDG_OK;
}

int ldg_queue_set_variant(ldg_queue* q, int32_t variant) {
    if (!q) return qfail(LDG_ERR_ARG, "ldg_queue_set_variant: NULL queue");
    if (variant < -1 || variant >= ldg::kNumVariants)
        return qfail(LDG_ERR_ARG, "ldg_queue_set_variant: variant must be -1, LDG_VARIANT_STOCKHAM or LDG_VARIANT_IN_PLACE");
    std::lock_guard<std::mutex> lk(q->mu);
    if (variant != q->variant) {
        Dev g(q->device);
        int rc = wait_idle(q);
        if (rc) return rc;
        drop_graph(q);
    }
    q->variant = variant;
    return LDG_OK;
}

int ldg_queue_info(ldg_queue* q, int64_t* total_blocks, int32_t* grid) {
    if (!q) return qfail(LDG_ERR_ARG, "ldg_queue_info: NULL queue");
    std::lock_guard<std::mutex> lk(q->mu);
    if (total_blocks) *total_blocks = q->total;
    if (grid) *grid = q->total ? grid_of(q) : 0;
    return LDG_OK;
}

int ldg_queue_run(ldg_queue* q, void* stream, int32_t use_graph) {
    if (!q) return qfail(LDG_ERR_ARG, "ldg_queue_run: NULL queue");
    std::lock_guard<std::mutex> lk(q->mu);
    if (q->total == 0) return LDG_OK;
    Dev g(q->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : q->stream;
    const int grid = grid_of(q);
    if (grid > q->scratch_ctas) {
        int rc = wait_idle(q);
        if (rc) return rc;
        drop_graph(q);
        cudaFree(q->d_scratch);
        q->d_scratch = nullptr;
        q->scratch_ctas = 0;
        QCK(cudaMalloc(&q->d_scratch, (size_t)grid * ldg::kScratchPerCta));
        q->scratch_ctas = grid;
    }
    ldg::QueueParams p;
    memset(&p, 0, sizeof(p));
    p.items = q->d_items;
    p.first_block = q->d_first;
    p.nitems = q->nitems;
    p.grab = q->grab;
    p.total = q->total;
    p.head = q->d_head;
    p.scratch = q->d_scratch;
    p.tw16 = q->tw16;
    p.tw32 = q->tw32;
    p.variant = q->variant >= 0 ? q->variant : q->item_variant;
    QCK(ldg::prepare_demod_queue());
    if (use_graph) {
        if (!q->exec || q->graph_grid != grid) {
            drop_graph(q);
            // captured on the queue's own stream: memset of the head, the launch
            QCK(cudaStreamBeginCapture(q->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e1 = cudaMemsetAsync(q->d_head, 0, sizeof(unsigned long long), q->stream);
            cudaError_t e2 = e1 == cudaSuccess ? ldg::launch_demod_queue(p, grid, q->stream) : e1;
            cudaGraph_t gr = nullptr;
            cudaError_t e3 = cudaStreamEndCapture(q->stream, &gr);
            if (e2 != cudaSuccess || e3 != cudaSuccess) {
                if (gr) cudaGraphDestroy(gr);
                return qfail(LDG_ERR_CUDA, std::string("ldg_queue_run: graph capture: ") +
                                               cudaGetErrorString(e2 != cudaSuccess ? e2 : e3));
            }
            q->graph = gr;
            QCK(cudaGraphInstantiate(&q->exec, q->graph, 0));
            q->graph_grid = grid;
        }
        QCK(cudaGraphLaunch(q->exec, st));
    } else {
        QCK(cudaMemsetAsync(q->d_head, 0, sizeof(unsigned long long), st));
        QCK(ldg::launch_demod_queue(p, grid, st));
    }
    QCK(cudaEventRecord(q->done, st));
    q->ran = true;
    return LDG_OK;
}

}  // extern "C"
