// Batched ensemble: many independent realizations (grid size, seed, forcing per realization)
// advanced together on one GPU.
//
// Every realization is a full solver handle (its own buffers, records and stream).  A batch of
// n steps of all realizations is captured once as one CUDA graph: a fork from the ensemble's
// stream into every realization's stream, the n steps of that realization's kernels there
// (programmatic dependent launch between consecutive kernels), the copy of its n per-step
// records into pinned host memory, and a join.  Replaying the graph advances the whole
// ensemble by n steps with one launch; the branches run concurrently on the GPU.  The graph is
// rebuilt only when n or the plan changes.
//
// Plan: a realization's persistent grids may use 1/2^share of the blocks that fit on the
// device (bastr_set_plan), so that concurrent realizations do not each spread over all SMs.
// bastr_ensemble_tune times the graph for each share per grid-size class (greedy, class by
// class) and keeps the fastest; the state is restored after every trial.
//
// Included by capi.cu (it uses the handle internals).

#include <cstdint>

struct bastr_ensemble {
    std::vector<bastr_handle*> hs;
    int device = 0;
    cudaStream_t main = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    double* host_rec = nullptr;   // pinned [n_real][kChunk][R_COUNT]
    unsigned int* host_halt = nullptr;   // pinned [n_real]: each realization's stop word after the batch
    cudaGraphExec_t exec = nullptr;
    int exec_steps = 0;
    std::string err;
};

namespace {

int efail(bastr_ensemble* e, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (e) e->err = buf;
    return code;
}

#define ECK(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return efail(e, BASTR_E_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                         __FILE__, __LINE__);                                              \
    } while (0)

void drop_graph(bastr_ensemble* e) {
    if (e->exec) cudaGraphExecDestroy(e->exec);
    e->exec = nullptr;
    e->exec_steps = 0;
}

// Captures the graph of nsteps steps of every realization.  The host counters of the handles
// are left as they were: the capture advances them, so they are saved and restored.
int capture(bastr_ensemble* e, int nsteps) {
    drop_graph(e);
    const size_t nr = e->hs.size();
    std::vector<int64_t> n0(nr);
    std::vector<double> t0(nr);
    for (size_t i = 0; i < nr; ++i) { n0[i] = e->hs[i]->nstep; t0[i] = e->hs[i]->time; }
    ECK(cudaStreamBeginCapture(e->main, cudaStreamCaptureModeRelaxed));
    cudaError_t st = cudaEventRecord(e->fork, e->main);
    for (size_t i = 0; i < nr && st == cudaSuccess; ++i) {
        bastr_handle* h = e->hs[i];
        st = cudaStreamWaitEvent(h->stream, e->fork, 0);
        if (st == cudaSuccess) st = launch_batch(h, nsteps);
        if (st == cudaSuccess)
            st = cudaMemcpyAsync(e->host_rec + i * (size_t)kChunk * R_COUNT, h->rec,
                                 (size_t)nsteps * R_COUNT * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        if (st == cudaSuccess)
            st = cudaMemcpyAsync(e->host_halt + i, h->done + T_HALT, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                 h->stream);
        if (st == cudaSuccess) st = cudaEventRecord(e->join[i], h->stream);
        if (st == cudaSuccess) st = cudaStreamWaitEvent(e->main, e->join[i], 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t st2 = cudaStreamEndCapture(e->main, &graph);
    for (size_t i = 0; i < nr; ++i) { e->hs[i]->nstep = n0[i]; e->hs[i]->time = t0[i]; }
    if (st != cudaSuccess || st2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return efail(e, BASTR_E_CUDA, "ensemble graph capture: %s",
                     cudaGetErrorString(st != cudaSuccess ? st : st2));
    }
    st = cudaGraphInstantiate(&e->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (st != cudaSuccess) return efail(e, BASTR_E_CUDA, "ensemble graph instantiate: %s", cudaGetErrorString(st));
    e->exec_steps = nsteps;
    return BASTR_OK;
}

// Replays the graph of nsteps (capturing it first if needed) and waits for it.
int run_graph(bastr_ensemble* e, int nsteps) {
    if (e->exec_steps != nsteps || !e->exec) {
        const int r = capture(e, nsteps);
        if (r) return r;
    }
    ECK(cudaGraphLaunch(e->exec, e->main));
    ECK(cudaStreamSynchronize(e->main));
    return BASTR_OK;
}

// Host bookkeeping of a replayed batch: counters, records, pending forcing scale.  A realization
// whose stop word is set (a NaN energy) keeps the counters of that step (apply_halt).
void after_batch(bastr_ensemble* e, int nsteps) {
    for (size_t r = 0; r < e->hs.size(); ++r) {
        bastr_handle* h = e->hs[r];
        h->batch_n0 = h->nstep;
        h->batch_t0 = h->time;
        for (int i = 0; i < nsteps; ++i) {
            h->nstep += 1;
            h->time = h->time + h->p.deltat;
        }
        h->chunk_used = nsteps;
        if (h->p.forcemethod == 1 && nsteps > 0) h->scale_pending = true;
        apply_halt(h, e->host_halt[r], nsteps);
    }
}

}  // namespace

extern "C" {

int bastr_ensemble_create(const bastr_params* params, int32_t n, bastr_ensemble** out) {
    if (!params || !out || n < 1) return BASTR_E_INVALID;
    bastr_ensemble* e = new bastr_ensemble();
    *out = e;   // also on failure, so that the caller can read the message; destroy it either way
    e->device = params[0].device;
    for (int i = 0; i < n; ++i) {
        if (params[i].device != e->device)
            return efail(e, BASTR_E_INVALID, "realization %d: all realizations must share one device", i);
        if (params[i].velgrad_every < 0 || params[i].velgrad_every > 1)
            return efail(e, BASTR_E_UNSUPPORTED, "realization %d: velgrad_every must be 0 or 1 in an ensemble", i);
        bastr_handle* h = nullptr;
        const int r = bastr_create(&params[i], &h);
        if (r) {
            e->err = "realization " + std::to_string(i) + ": " + (h ? h->err : std::string("create failed"));
            if (h) bastr_destroy(h);
            return r;
        }
        e->hs.push_back(h);
    }
    ECK(cudaSetDevice(e->device));
    ECK(cudaStreamCreateWithFlags(&e->main, cudaStreamNonBlocking));
    ECK(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
    e->join.resize(n);
    for (int i = 0; i < n; ++i) ECK(cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming));
    ECK(cudaMallocHost(&e->host_rec, (size_t)n * kChunk * R_COUNT * sizeof(double)));
    ECK(cudaMallocHost(&e->host_halt, (size_t)n * sizeof(unsigned int)));
    memset(e->host_halt, 0, (size_t)n * sizeof(unsigned int));
    return BASTR_OK;
}

int bastr_ensemble_destroy(bastr_ensemble* e) {
    if (!e) return BASTR_OK;
    cudaSetDevice(e->device);
    if (e->main) cudaStreamSynchronize(e->main);
    drop_graph(e);
    for (bastr_handle* h : e->hs) bastr_destroy(h);
    for (cudaEvent_t ev : e->join) if (ev) cudaEventDestroy(ev);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->main) cudaStreamDestroy(e->main);
    if (e->host_rec) cudaFreeHost(e->host_rec);
    if (e->host_halt) cudaFreeHost(e->host_halt);
    delete e;
    return BASTR_OK;
}

int bastr_ensemble_size(bastr_ensemble* e, int32_t* n) {
    if (!e || !n) return BASTR_E_INVALID;
    *n = (int32_t)e->hs.size();
    return BASTR_OK;
}

int bastr_ensemble_set_state(bastr_ensemble* e, int32_t i, const double* u1, const double* u2, const double* u3) {
    if (!e || i < 0 || i >= (int)e->hs.size()) return efail(e, BASTR_E_INVALID, "realization index");
    const int r = bastr_set_state(e->hs[i], u1, u2, u3);
    if (r) e->err = "realization " + std::to_string(i) + ": " + e->hs[i]->err;
    return r;
}

int bastr_ensemble_get_state(bastr_ensemble* e, int32_t i, double* u1, double* u2, double* u3) {
    if (!e || i < 0 || i >= (int)e->hs.size()) return efail(e, BASTR_E_INVALID, "realization index");
    const int r = bastr_get_state(e->hs[i], u1, u2, u3);
    if (r) e->err = "realization " + std::to_string(i) + ": " + e->hs[i]->err;
    return r;
}

// out: [n_real][nsteps] records (realization-major).  Returns BASTR_E_NAN if some realization's
// Es+Ed became NaN (all records are filled; the message names the first one).
int bastr_ensemble_step(bastr_ensemble* e, int32_t nsteps, bastr_step_out* out) {
    NvtxRange range("bastr_ensemble_step");
    if (!e || nsteps < 0 || nsteps > kChunk) return efail(e, BASTR_E_INVALID, "nsteps must be in [0, %d]", kChunk);
    for (size_t i = 0; i < e->hs.size(); ++i)
        if (!e->hs[i]->have_state) return efail(e, BASTR_E_STATE, "realization %zu: no state set", i);
    if (nsteps == 0) return BASTR_OK;
    ECK(cudaSetDevice(e->device));
    int r = run_graph(e, nsteps);
    if (r) return r;
    after_batch(e, nsteps);
    int status = BASTR_OK;
    for (size_t i = 0; i < e->hs.size(); ++i) {
        bastr_step_out* o = out ? out + i * (size_t)nsteps : nullptr;
        const int valid = e->hs[i]->chunk_used;   // steps up to a NaN stop
        decode_records(e->hs[i], e->host_rec + i * (size_t)kChunk * R_COUNT, valid, o);
        blank_records(o, valid, nsteps);
        if (valid < nsteps || e->host_halt[i] != 0) {
            if (status == BASTR_OK)
                status = efail(e, BASTR_E_NAN, "realization %zu: \"E\" is a NaN at nstep %lld", i,
                               (long long)e->hs[i]->nstep);
        }
    }
    return status;
}

// Advances the ensemble by nsteps = k * batch steps as k replays of the batch graph, timed on the
// device with events on the ensemble's stream around all of them; only the last batch's records
// stay (bastr_ensemble_step reads them for a batch).  device_ms: total device time.
int bastr_ensemble_run(bastr_ensemble* e, int32_t nsteps, int32_t batch, double* device_ms) {
    NvtxRange range("bastr_ensemble_run");
    if (!e || batch < 1 || batch > kChunk || nsteps < 0 || nsteps % batch)
        return efail(e, BASTR_E_INVALID, "nsteps must be a multiple of batch, batch in [1, %d]", kChunk);
    for (size_t i = 0; i < e->hs.size(); ++i)
        if (!e->hs[i]->have_state) return efail(e, BASTR_E_STATE, "realization %zu: no state set", i);
    ECK(cudaSetDevice(e->device));
    if (e->exec_steps != batch || !e->exec) {
        const int r = capture(e, batch);
        if (r) return r;
    }
    cudaEvent_t a = nullptr, b = nullptr;
    ECK(cudaEventCreate(&a));
    ECK(cudaEventCreate(&b));
    const int k = nsteps / batch;
    cudaError_t st = cudaEventRecord(a, e->main);
    for (int i = 0; i < k && st == cudaSuccess; ++i) st = cudaGraphLaunch(e->exec, e->main);
    if (st == cudaSuccess) st = cudaEventRecord(b, e->main);
    if (st == cudaSuccess) st = cudaEventSynchronize(b);
    float ms = 0.f;
    if (st == cudaSuccess) st = cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (st != cudaSuccess) return efail(e, BASTR_E_CUDA, "ensemble run: %s", cudaGetErrorString(st));
    if (device_ms) *device_ms = ms;
    // host bookkeeping: the first k-1 batches advance the counters, the last one also reads the
    // stop words (a realization that stopped keeps stopping at once in every later batch)
    for (int i = 0; i + 1 < k; ++i)
        for (bastr_handle* h : e->hs)
            for (int j = 0; j < batch; ++j) {
                h->nstep += 1;
                h->time = h->time + h->p.deltat;
            }
    if (k > 0) after_batch(e, batch);
    for (size_t i = 0; i < e->hs.size(); ++i)
        if (k > 0 && e->host_halt[i] != 0)
            return efail(e, BASTR_E_NAN, "realization %zu: \"E\" is a NaN at nstep %lld", i,
                         (long long)e->hs[i]->nstep);
    return BASTR_OK;
}

// Filtered fields and subgrid term of realization i's current state (bastr_subgrid): the
// ensemble's output as closure training data.
int bastr_ensemble_subgrid(bastr_ensemble* e, int32_t i, int32_t r, float* d_ubar, float* d_tau) {
    if (!e || i < 0 || i >= (int)e->hs.size()) return efail(e, BASTR_E_INVALID, "realization index");
    const int rc = bastr_subgrid(e->hs[i], r, d_ubar, d_tau);
    if (rc) e->err = "realization " + std::to_string(i) + ": " + e->hs[i]->err;
    return rc;
}

// Sets the plan of realization i (-1: all) and drops the captured graph.
int bastr_ensemble_set_plan(bastr_ensemble* e, int32_t i, int32_t share_log2) {
    if (!e) return BASTR_E_INVALID;
    if (share_log2 < 0 || share_log2 > 7) return efail(e, BASTR_E_INVALID, "share_log2 must be in [0, 7]");
    if (i < -1 || i >= (int)e->hs.size()) return efail(e, BASTR_E_INVALID, "realization index");
    for (size_t k = 0; k < e->hs.size(); ++k)
        if (i < 0 || (int)k == i) e->hs[k]->share_log2 = share_log2;
    drop_graph(e);
    return BASTR_OK;
}

int bastr_ensemble_get_plan(bastr_ensemble* e, int32_t* share_log2 /* [n_real] */) {
    if (!e || !share_log2) return BASTR_E_INVALID;
    for (size_t k = 0; k < e->hs.size(); ++k) share_log2[k] = e->hs[k]->share_log2;
    return BASTR_OK;
}

// Autotuner: for each grid-size class (realizations with the same ia, ja, ka and precision), in
// order of decreasing size, tries shares 0..max_share_log2 with the other classes at their
// current choice, timing `nsteps` steps of the whole ensemble graph (best of `reps` replays),
// and keeps the fastest.  The state and counters of every realization are restored after each
// trial.  best_ms (optional) receives the time per step of the final plan.
int bastr_ensemble_tune(bastr_ensemble* e, int32_t nsteps, int32_t reps, int32_t max_share_log2, double* best_ms) {
    if (!e || nsteps < 1 || nsteps > kChunk || reps < 1 || max_share_log2 < 0 || max_share_log2 > 7)
        return efail(e, BASTR_E_INVALID, "bastr_ensemble_tune arguments");
    for (size_t i = 0; i < e->hs.size(); ++i)
        if (!e->hs[i]->have_state) return efail(e, BASTR_E_STATE, "realization %zu: no state set", i);
    ECK(cudaSetDevice(e->device));
    const size_t nr = e->hs.size();
    // snapshot: state, pending forcing scale, counters
    std::vector<void*> snap(nr, nullptr);
    std::vector<double2> pend(nr);
    std::vector<bool> spend(nr);
    std::vector<int64_t> n0(nr);
    std::vector<double> t0(nr);
    for (size_t i = 0; i < nr; ++i) {
        bastr_handle* h = e->hs[i];
        ECK(cudaMalloc(&snap[i], h->n_state * sizeof(double2)));
        ECK(cudaMemcpyAsync(snap[i], h->u0, h->n_state * sizeof(double2), cudaMemcpyDeviceToDevice, e->main));
        ECK(cudaMemcpyAsync(&pend[i], h->pend, sizeof(double2), cudaMemcpyDeviceToHost, e->main));
        spend[i] = h->scale_pending;
        n0[i] = h->nstep;
        t0[i] = h->time;
    }
    ECK(cudaStreamSynchronize(e->main));
    auto restore = [&]() -> cudaError_t {
        for (size_t i = 0; i < nr; ++i) {
            bastr_handle* h = e->hs[i];
            cudaError_t st = cudaMemcpyAsync(h->u0, snap[i], h->n_state * sizeof(double2), cudaMemcpyDeviceToDevice, e->main);
            if (st == cudaSuccess) st = cudaMemcpyAsync(h->pend, &pend[i], sizeof(double2), cudaMemcpyHostToDevice, e->main);
            if (st != cudaSuccess) return st;
            h->scale_pending = spend[i];
            h->nstep = n0[i];
            h->time = t0[i];
        }
        return cudaStreamSynchronize(e->main);
    };
    cudaEvent_t a = nullptr, b = nullptr;
    ECK(cudaEventCreate(&a));
    ECK(cudaEventCreate(&b));
    auto trial = [&](float* ms) -> int {
        int r = capture(e, nsteps);
        if (r) return r;
        float best = 1e30f;
        for (int k = 0; k < reps + 1; ++k) {   // the first replay warms up
            ECK(cudaEventRecord(a, e->main));
            ECK(cudaGraphLaunch(e->exec, e->main));
            ECK(cudaEventRecord(b, e->main));
            ECK(cudaEventSynchronize(b));
            float t = 0;
            ECK(cudaEventElapsedTime(&t, a, b));
            if (k > 0) best = std::min(best, t);
            ECK(restore());
        }
        *ms = best / nsteps;
        return BASTR_OK;
    };
    // classes in order of decreasing grid size
    std::vector<std::tuple<long long, int, int, int, int>> keys;
    for (bastr_handle* h : e->hs) {
        auto k = std::make_tuple(-(long long)h->p.ia * h->p.ja * std::max(h->p.ka, 1), h->p.ia, h->p.ja, h->p.ka,
                                 h->p.precision);
        if (std::find(keys.begin(), keys.end(), k) == keys.end()) keys.push_back(k);
    }
    std::sort(keys.begin(), keys.end());
    float cur = 0;
    int r = trial(&cur);
    for (size_t c = 0; c < keys.size() && r == BASTR_OK; ++c) {
        const auto& k = keys[c];
        auto in_class = [&](const bastr_handle* h) {
            return h->p.ia == std::get<1>(k) && h->p.ja == std::get<2>(k) && h->p.ka == std::get<3>(k) &&
                   h->p.precision == std::get<4>(k);
        };
        int keep = 0;
        for (bastr_handle* h : e->hs) if (in_class(h)) keep = h->share_log2;
        for (int s = 0; s <= max_share_log2 && r == BASTR_OK; ++s) {
            if (s == keep) continue;
            for (bastr_handle* h : e->hs) if (in_class(h)) h->share_log2 = s;
            float ms = 0;
            r = trial(&ms);
            if (r == BASTR_OK && ms < cur) { cur = ms; keep = s; }
        }
        for (bastr_handle* h : e->hs) if (in_class(h)) h->share_log2 = keep;
    }
    drop_graph(e);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    for (void* q : snap) if (q) cudaFree(q);
    if (r) return r;
    if (best_ms) *best_ms = cur;
    return BASTR_OK;
}

int bastr_ensemble_last_error(bastr_ensemble* e, char* buf, int32_t n) {
    if (!e) return 0;
    const int len = (int)e->err.size();
    if (buf && n > 0) {
        const int m = std::min(len, n - 1);
        memcpy(buf, e->err.data(), m);
        buf[m] = 0;
    }
    return len;
}

}  // extern "C"
