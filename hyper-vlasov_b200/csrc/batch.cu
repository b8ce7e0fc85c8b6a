// Batched runs: many independent nuclei advanced together on one GPU.
//
// The reference runs one nucleus per process.  A batch holds several float
// contexts (each its own nucleus, test-particle count, grid and parameters,
// created with hv_ctx_create) and advances them step by step together: per
// step, every instance's particle step, smoothing and Skyrme potential run as
// parallel branches on per-instance streams, then the Coulomb solves run as a
// few cooperative launches ("waves") that each solve several instances at once
// (k_sor_fast in its batched form: every block looks up its instance, and
// barriers, residual sums and the boundary exchange stay within the
// instance), then every instance's forces.  Chunks of steps are captured into
// one CUDA graph and replayed.  The results of every instance are those of
// its own hv_run on the fused path, up to float rounding.
//
// How many blocks each instance's solve uses is a plan choice: fewer blocks
// pack more instances into a wave, more blocks make each solve faster.
// hv_batch_plan takes a cap; hv_batch_autotune times candidate caps on trial
// steps and keeps the fastest, then the particle step's block size.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "hv_internal.h"

using namespace hv;

struct hv_batch {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    std::vector<hv_ctx *> ctx;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> ev_a, ev_c;  // per instance: end of its phase A / C
    cudaEvent_t ev_fork_a = nullptr, ev_fork_c = nullptr;
    std::vector<SorWave> waves;
    int cap = -1;                         // SOR block cap of the current plan (0: own plans)
    cudaGraphExec_t graph = nullptr;
    int graph_len = 0;
    int chunk = 8;
};

namespace {

void drop_graph(hv_batch *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_len = 0;
}

// One step of every instance, on the batch stream with per-instance branches.
hv_status enqueue_batch_step(hv_batch *b) {
    const int n = (int)b->ctx.size();
    HV_CUDA(cudaEventRecord(b->ev_fork_a, b->stream));
    for (int i = 0; i < n; i++) {
        HV_CUDA(cudaStreamWaitEvent(b->streams[i], b->ev_fork_a, 0));
        HV_TRY(fused_batch_phase_a(b->ctx[i], b->streams[i]));
        HV_CUDA(cudaEventRecord(b->ev_a[i], b->streams[i]));
        HV_CUDA(cudaStreamWaitEvent(b->stream, b->ev_a[i], 0));
    }
    for (const SorWave &w : b->waves) HV_TRY(sor_wave_launch(w, b->stream));
    HV_CUDA(cudaEventRecord(b->ev_fork_c, b->stream));
    for (int i = 0; i < n; i++) {
        HV_CUDA(cudaStreamWaitEvent(b->streams[i], b->ev_fork_c, 0));
        HV_TRY(fused_batch_phase_c(b->ctx[i], b->streams[i]));
        HV_CUDA(cudaEventRecord(b->ev_c[i], b->streams[i]));
        HV_CUDA(cudaStreamWaitEvent(b->stream, b->ev_c[i], 0));
    }
    return HV_OK;
}

hv_status enqueue_batch_steps(hv_batch *b, int k) {
    for (int s = 0; s < k; s++) HV_TRY(enqueue_batch_step(b));
    return HV_OK;
}

void release_waves(hv_batch *b) {
    for (SorWave &w : b->waves) sor_wave_release(w);
    b->waves.clear();
}

}  // namespace

extern "C" {

hv_status hv_batch_create(int n, hv_ctx *const *ctxs, hv_batch **out) {
    if (!out || n < 1 || !ctxs) return HV_ERR_BAD_ARG;
    *out = nullptr;
    for (int i = 0; i < n; i++) {
        if (!ctxs[i]) return HV_ERR_BAD_ARG;
        if (ctxs[i]->prec != HV_F32 || ctxs[i]->device != ctxs[0]->device) return HV_ERR_UNSUPPORTED;
        for (int j = 0; j < i; j++)
            if (ctxs[j] == ctxs[i]) return HV_ERR_BAD_ARG;
    }
    hv_batch *b = new hv_batch();
    b->device = ctxs[0]->device;
    b->sm_count = ctxs[0]->sm_count;
    b->ctx.assign(ctxs, ctxs + n);
    auto fail = [&](hv_status s) {
        hv_batch_destroy(b);
        return s;
    };
    if (cudaSetDevice(b->device) != cudaSuccess) return fail(HV_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(HV_ERR_CUDA);
    if (cudaEventCreateWithFlags(&b->ev_fork_a, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_fork_c, cudaEventDisableTiming) != cudaSuccess)
        return fail(HV_ERR_CUDA);
    b->streams.resize(n);
    b->ev_a.resize(n);
    b->ev_c.resize(n);
    for (int i = 0; i < n; i++) {
        if (cudaStreamCreateWithFlags(&b->streams[i], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->ev_a[i], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->ev_c[i], cudaEventDisableTiming) != cudaSuccess)
            return fail(HV_ERR_CUDA);
    }
    for (hv_ctx *c : b->ctx) {
        hv_status st = fused_batch_ready(c);
        if (st != HV_OK) return fail(st);
    }
    hv_status st = hv_batch_plan(b, 0);
    if (st != HV_OK) return fail(st);
    *out = b;
    return HV_OK;
}

hv_status hv_batch_destroy(hv_batch *b) {
    if (!b) return HV_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    release_waves(b);
    for (cudaStream_t s : b->streams)
        if (s) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->ev_a)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : b->ev_c)
        if (e) cudaEventDestroy(e);
    if (b->ev_fork_a) cudaEventDestroy(b->ev_fork_a);
    if (b->ev_fork_c) cudaEventDestroy(b->ev_fork_c);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return HV_OK;
}

hv_status hv_batch_plan(hv_batch *b, int sor_max_blocks) {
    if (!b || sor_max_blocks < 0) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(b->device));
    HV_CUDA(cudaStreamSynchronize(b->stream));
    drop_graph(b);
    release_waves(b);
    const int n = (int)b->ctx.size();
    for (hv_ctx *c : b->ctx) {
        HV_CUDA(cudaStreamSynchronize(c->stream));
        if (c->fused.graph) {  // a context's own graph holds the old SOR buffers
            cudaGraphExecDestroy(c->fused.graph);
            c->fused.graph = nullptr;
            c->fused.graph_len = 0;
        }
        // the cap, doubled for an instance whose grid needs more blocks' shared
        // memory (the batched solve is a tagged sweep: it needs the source and
        // the row tables in shared memory too)
        auto usable = [&] { return c->fused.sor.ok && c->fused.sor.tables; };
        int m = sor_max_blocks;
        HV_TRY(sor_fast_replan(c, m));
        while (!usable() && m > 0 && m < b->sm_count) {
            m = std::min(2 * m, b->sm_count);
            HV_TRY(sor_fast_replan(c, m));
        }
        if (!usable()) {
            set_last_error("batch: an instance's SOR does not fit on chip");
            return HV_ERR_UNSUPPORTED;
        }
    }
    // first fit by decreasing block count into waves of at most one block per SM
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return b->ctx[x]->fused.sor.nblocks > b->ctx[y]->fused.sor.nblocks; });
    std::vector<std::vector<int>> groups;
    std::vector<int> used;
    for (int i : order) {
        const int nb = b->ctx[i]->fused.sor.nblocks;
        size_t g = 0;
        while (g < groups.size() && used[g] + nb > b->sm_count) g++;
        if (g == groups.size()) {
            groups.emplace_back();
            used.push_back(0);
        }
        groups[g].push_back(i);
        used[g] += nb;
    }
    for (auto &grp : groups) {
        std::vector<hv_ctx *> cs;
        std::vector<const float *> rho;
        std::vector<int *> ctl, its;
        int ring = 0;
        for (int i : grp) {
            const float *r;
            int *cl, *it;
            fused_batch_sor_inputs(b->ctx[i], &r, &cl, &it, &ring);
            cs.push_back(b->ctx[i]);
            rho.push_back(r);
            ctl.push_back(cl);
            its.push_back(it);
        }
        b->waves.emplace_back();
        hv_status st = sor_wave_build(b->waves.back(), cs, rho, ctl, its, ring);
        if (st != HV_OK) {
            set_last_error("batch: a wave of solves cannot be launched together");
            return st;
        }
    }
    b->cap = sor_max_blocks;
    return HV_OK;
}

int hv_batch_waves(const hv_batch *b) { return b ? (int)b->waves.size() : -1; }

hv_status hv_batch_run(hv_batch *b, int n_steps, hv_observables *obs) {
    if (!b || n_steps < 0) return HV_ERR_BAD_ARG;
    if (n_steps == 0) return HV_OK;
    HV_CUDA(cudaSetDevice(b->device));
    const int n = (int)b->ctx.size();
    std::vector<int> exc(n, -1);
    for (int i = 0; i < n; i++) HV_TRY(fused_batch_begin(b->ctx[i], n_steps, &exc[i]));
    int done = 0;
    while (done < n_steps) {
        const int k = std::min(b->chunk, n_steps - done);
        bool launched = false;
        if (k == b->chunk) {
            if (!b->graph || b->graph_len != k) {
                drop_graph(b);
                cudaGraph_t gr = nullptr;
                if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                    hv_status es = enqueue_batch_steps(b, k);
                    cudaError_t ce = cudaStreamEndCapture(b->stream, &gr);
                    if (es == HV_OK && ce == cudaSuccess && gr &&
                        cudaGraphInstantiate(&b->graph, gr, 0) == cudaSuccess)
                        b->graph_len = k;
                    else
                        b->graph = nullptr;
                    if (gr) cudaGraphDestroy(gr);
                    cudaGetLastError();
                }
            }
            if (b->graph) {
                HV_CUDA(cudaGraphLaunch(b->graph, b->stream));
                launched = true;
            }
        }
        if (!launched) HV_TRY(enqueue_batch_steps(b, k));
        for (int i = 0; i < n; i++) {
            hv_ctx *c = b->ctx[i];
            HV_TRY(fused_batch_rows(c, b->stream, c->step_index + done, k,
                                    obs ? obs + (size_t)i * n_steps + done : nullptr));
        }
        done += k;
    }
    for (int i = 0; i < n; i++) HV_TRY(fused_batch_end(b->ctx[i], n_steps, exc[i]));
    return HV_OK;
}

hv_status hv_batch_autotune(hv_batch *b, int trial_steps, int *chosen_cap) {
    if (!b || trial_steps < 1) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(b->device));
    const int caps[] = {0, 64, 32, 16, 8, 4};
    cudaEvent_t e0, e1;
    HV_CUDA(cudaEventCreate(&e0));
    HV_CUDA(cudaEventCreate(&e1));
    int best = -1;
    float best_ms = 0.0f;
    for (int cap : caps) {
        if (hv_batch_plan(b, cap) != HV_OK) continue;
        HV_TRY(hv_batch_run(b, 1, nullptr));  // first use: graphs, caches
        HV_CUDA(cudaEventRecord(e0, b->stream));
        HV_TRY(hv_batch_run(b, trial_steps, nullptr));
        HV_CUDA(cudaEventRecord(e1, b->stream));
        HV_CUDA(cudaEventSynchronize(e1));
        float ms = 0.0f;
        HV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (best < 0 || ms < best_ms) {
            best = cap;
            best_ms = ms;
        }
    }
    if (best < 0) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return HV_ERR_UNSUPPORTED;
    }
    HV_TRY(hv_batch_plan(b, best));
    // then the particle step's block size, the same for every instance
    int best_pb = 0;
    best_ms = 0.0f;
    for (int pb : {128, 256, 512}) {
        for (hv_ctx *c : b->ctx) c->fused.pblock = pb;
        drop_graph(b);
        HV_TRY(hv_batch_run(b, 1, nullptr));
        HV_CUDA(cudaEventRecord(e0, b->stream));
        HV_TRY(hv_batch_run(b, trial_steps, nullptr));
        HV_CUDA(cudaEventRecord(e1, b->stream));
        HV_CUDA(cudaEventSynchronize(e1));
        float ms = 0.0f;
        HV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (best_pb == 0 || ms < best_ms) {
            best_pb = pb;
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (hv_ctx *c : b->ctx) c->fused.pblock = best_pb;
    drop_graph(b);
    if (chosen_cap) *chosen_cap = best;
    return HV_OK;
}

hv_status hv_batch_tiles(const hv_batch *b, int *sor_planes, int *sor_rows, int *sor_blocks, int *particle_block,
                         int n) {
    if (!b || n < 0 || n > (int)b->ctx.size()) return HV_ERR_BAD_ARG;
    for (int i = 0; i < n; i++) {
        const hv_ctx *c = b->ctx[i];
        if (sor_planes) sor_planes[i] = c->fused.sor.P;
        if (sor_rows) sor_rows[i] = c->fused.sor.R;
        if (sor_blocks) sor_blocks[i] = c->fused.sor.nblocks;
        if (particle_block) particle_block[i] = c->fused.pblock;
    }
    return HV_OK;
}

}  // extern "C"
