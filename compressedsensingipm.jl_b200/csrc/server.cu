// C ABI (include/csipm.h), part 4: the serving loop.
//
// Recoveries of uneven sizes arrive as requests; a fixed number of slots
// (worker threads, each with its own non-blocking CUDA stream) take them in
// arrival order as soon as a slot is free and the request's device footprint
// fits in what the admitted requests leave of the HBM budget.  A request that
// does not fit yet lets smaller ones behind it go first (up to
// ADMIT_LOOKAHEAD places), so the device stays busy while memory frees up.
// Each admitted request keeps its whole interior-point state resident in a
// handle on its slot's stream; the slots' kernels overlap on the device.
// Handles take their memory from the stream-ordered pool, so creating and
// destroying them does not stall the other slots.
//
// With batching on (csipm_server_options.batch > 1) a slot that admits a
// request also admits up to batch - 1 more of the same batch class (the
// dimension count, the long-row 1D passes, missing samples or not), the
// closest in size first, as far as the budget allows, and solves them
// together with csipm_solve_batch: one launch per step for all of them.
// Requests above batch_max_n samples (when set) are solved alone: they fill
// the GPU by themselves, and alone they keep their precision (a batch runs
// FP64).
//
// The reference has no serving layer; it solves one recovery per call
// (src/CompressedSensingIPM.jl:31-36).
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>

#include "internal.h"

namespace {

using Clock = std::chrono::steady_clock;

constexpr int ADMIT_LOOKAHEAD = 16;
// queued requests a batch looks through for members of its class
constexpr int BATCH_SCAN = 512;

struct Pending {
    csipm_request req;
    size_t footprint;
    long long n;          // samples
    int bclass;           // batch class: requests of one class can share a csipm_solve_batch
    Clock::time_point t_submit;
};

// dimension count, long-row 1D passes (half-length above the one-CTA row
// pass's limit), missing samples or not
int batch_class(const csipm_problem& p) {
    const bool long1d = p.dim == 1 && p.size[0] / 2 > csipm::L1D_MIN_M;
    return p.dim * 4 + (long1d ? 2 : 0) + (p.n_missing > 0 ? 1 : 0);
}

}  // namespace

struct csipm_server_s {
    int device = 0;
    int slots = 0;
    int cuda_graphs = 0;
    int batch = 1;
    long long batch_max_n = 0;
    size_t budget = 0;
    size_t in_use = 0;
    bool stopping = false;
    long long submitted = 0, finished = 0;
    std::mutex mu;
    std::condition_variable cv_work;    // workers: a request or a stop arrived, or memory freed
    std::condition_variable cv_done;    // pollers / destroy: a result arrived
    std::deque<Pending> queue;
    std::deque<csipm_result> results;
    std::vector<std::thread> workers;

    void work(int slot);
    bool take(std::vector<Pending>* out);    // with mu held
};

namespace csipm_internal {

// Device bytes csipm_create allocates for a problem (the handle's vectors,
// spectra, mask, plane map and reduction workspace), plus the two N-vectors
// the server stages z0 and beta in.
size_t footprint_bytes(int dim, const int* size, int precision, int64_t n_missing) {
    const long long n1 = size[0], n2 = dim >= 2 ? size[1] : 1, n3 = dim >= 3 ? size[2] : 1;
    const size_t N = (size_t)(n1 * n2 * n3);
    const size_t Nh = (size_t)((n1 / 2 + 1) * n2 * n3);
    size_t b = 0;
    b += 24 * 8 * N;                              // FP64 beta-space vectors (IPM state, CG, solver-order A^T z0)
    b += 16 * Nh;                                 // FP64 spectrum
    if (precision == CSIPM_MIXED) b += 8 * 4 * N + 8 * Nh;   // FP32 CG vectors and directions + FP32 spectrum
    if (n_missing > 0) b += (size_t)((n1 + 31) / 32) * 4 * (size_t)(n2 * n3) * (precision == CSIPM_MIXED ? 2 : 1);
    b += 2 * 16 * (size_t)(n2 * n3);              // plane map
    b += 8 * 8 * 65536 + (1 << 20);               // reduction partials, slots, twiddles (upper bound)
    b += 2 * 8 * N;                               // the server's z0 / beta staging
    return b;
}

}  // namespace csipm_internal

bool csipm_server_s::take(std::vector<Pending>* out) {
    out->clear();
    const size_t avail = budget > in_use ? budget - in_use : 0;
    int look = 0;
    auto head = queue.end();
    for (auto it = queue.begin(); it != queue.end() && look < ADMIT_LOOKAHEAD; ++it, ++look)
        if (it->footprint <= avail) {
            head = it;
            break;
        }
    // nothing admitted runs and the head still does not fit: admit it alone
    // rather than wait forever (it then fails in csipm_create with OOM if the
    // device really cannot hold it)
    if (head == queue.end() && in_use == 0 && !queue.empty()) head = queue.begin();
    if (head == queue.end()) return false;
    out->push_back(*head);
    in_use += head->footprint;
    queue.erase(head);
    if (batch <= 1) return true;
    // members of the head's class, closest in size first, while they fit;
    // requests above batch_max_n samples are solved alone
    const Pending& h = out->front();
    if (batch_max_n > 0 && h.n > batch_max_n) return true;
    std::vector<std::pair<double, int>> cand;
    int k = 0;
    for (auto it = queue.begin(); it != queue.end() && k < BATCH_SCAN; ++it, ++k)
        if (it->bclass == h.bclass && (batch_max_n <= 0 || it->n <= batch_max_n))
            cand.push_back({std::fabs(std::log((double)it->n / (double)h.n)), k});
    std::stable_sort(cand.begin(), cand.end());
    std::vector<int> pick;
    for (const auto& c : cand) {
        if ((int)(out->size() + pick.size()) >= batch) break;
        const Pending& q = queue[c.second];
        if (in_use + q.footprint > budget) continue;
        in_use += q.footprint;
        pick.push_back(c.second);
    }
    std::sort(pick.begin(), pick.end());
    for (int j : pick) out->push_back(queue[j]);
    for (auto it = pick.rbegin(); it != pick.rend(); ++it) queue.erase(queue.begin() + *it);
    return true;
}

// A slot's pinned host staging buffer for z0 and beta: copies from and to
// pinned memory run asynchronously on the slot's stream (a pageable copy
// would hold the slot's thread until the driver has staged it).  It grows in
// powers of two and is handed back to the process-wide pinned free list.
struct PinnedStage {
    double* p = nullptr;
    size_t bytes = 0;
    bool ensure(size_t need) {
        if (need <= bytes) return true;
        size_t b = 1 << 16;
        while (b < need) b <<= 1;
        if (p) pinned_put(p, bytes);
        p = static_cast<double*>(pinned_get(b));
        bytes = p ? b : 0;
        return p != nullptr;
    }
    ~PinnedStage() {
        if (p) pinned_put(p, bytes);
    }
};

static void set_message(csipm_result* r, const char* msg) {
    std::strncpy(r->message, msg ? msg : "", sizeof(r->message) - 1);
    r->message[sizeof(r->message) - 1] = 0;
}

// Solves an admitted group on the slot's stream — one request through
// csipm_solve, several through csipm_solve_batch — and fills one result per
// member (status, stats, message).  Members stage z0 and beta through one
// pinned buffer, each at its own offset.
static void run_group(const std::vector<Pending>& g, int cuda_graphs, cudaStream_t st, cudaMemPool_t pool,
                      PinnedStage& stage, std::vector<csipm_result>& res) {
    const int K = (int)g.size();
    const bool batched = K > 1;
    const auto t_start = Clock::now();
    res.assign(K, csipm_result{});
    std::vector<size_t> off(K + 1, 0);
    for (int k = 0; k < K; ++k) off[k + 1] = off[k] + (size_t)g[k].n;
    std::vector<double*> z0(K, nullptr), beta(K, nullptr);
    std::vector<csipm_handle> h(K, nullptr);
    std::vector<int> status(K, CSIPM_OK);
    std::vector<std::string> msg(K);
    std::vector<char> copied(K, 0);
    auto failk = [&](int k, int code, const std::string& m) {
        if (status[k] != CSIPM_OK && status[k] != CSIPM_ERR_IPM_MAXITER && status[k] != CSIPM_ERR_CG_MAXITER) return;
        status[k] = code;
        msg[k] = m;
    };
    const bool staged = stage.ensure(sizeof(double) * off[K]);
    for (int k = 0; k < K; ++k) {
        res[k].tag = g[k].req.tag;
        res[k].footprint = g[k].footprint;
        res[k].group = K;
        res[k].queue_ms = std::chrono::duration<double, std::milli>(t_start - g[k].t_submit).count();
        const csipm_problem& pr = g[k].req.problem;
        const size_t bytes = sizeof(double) * (size_t)g[k].n;
        if (!pool || cudaMallocFromPoolAsync((void**)&z0[k], bytes, pool, st) != cudaSuccess ||
            cudaMallocFromPoolAsync((void**)&beta[k], bytes, pool, st) != cudaSuccess) {
            failk(k, CSIPM_ERR_OOM, "out of device memory (staging z0 / beta)");
            continue;
        }
        if (!staged) {
            failk(k, CSIPM_ERR_OOM, "pinned host allocation failed");
            continue;
        }
        std::memcpy(stage.p + off[k], pr.z0, bytes);
        if (cudaMemcpyAsync(z0[k], stage.p + off[k], bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            failk(k, CSIPM_ERR_CUDA, "z0 upload failed");
            continue;
        }
        csipm_problem dp = pr;
        dp.z0 = z0[k];
        csipm_options o = g[k].req.options;
        o.stream = st;
        // a served handle lives for one solve: its graphs are captured for
        // that one solve, which pays off on the server's say-so only
        o.cuda_graphs = cuda_graphs;
        // a batch solves in FP64 (a mixed-precision request gets FP64 iterates,
        // to its own tolerance)
        if (batched) o.precision = CSIPM_FP64;
        const int r = csipm_create(&dp, &o, &h[k]);
        if (r != CSIPM_OK) {
            h[k] = nullptr;
            failk(k, r, csipm_last_error(nullptr));
        }
    }
    if (!batched) {
        if (h[0] && status[0] == CSIPM_OK) {
            const int r = csipm_solve(h[0], beta[0], nullptr, &res[0].stats);
            if (r != CSIPM_OK) failk(0, r, h[0]->err);
        }
    } else {
        std::vector<int> live;
        std::vector<csipm_handle> hl;
        std::vector<double*> bl;
        for (int k = 0; k < K; ++k)
            if (h[k] && status[k] == CSIPM_OK) {
                live.push_back(k);
                hl.push_back(h[k]);
                bl.push_back(beta[k]);
            }
        if (!hl.empty()) {
            std::vector<csipm_stats> S(hl.size());
            const int r = csipm_solve_batch(hl.data(), (int)hl.size(), bl.data(), S.data());
            const std::string batch_err = r != CSIPM_OK ? csipm_last_error(nullptr) : "";
            for (size_t j = 0; j < live.size(); ++j) {
                const int k = live[j];
                res[k].stats = S[j];
                if (S[j].status != CSIPM_OK) failk(k, S[j].status, h[k]->err.empty() ? batch_err : h[k]->err);
            }
        }
    }
    for (int k = 0; k < K; ++k) {
        const int sk = status[k];
        if (!h[k] || !g[k].req.beta_out) continue;
        if (sk != CSIPM_OK && sk != CSIPM_ERR_IPM_MAXITER && sk != CSIPM_ERR_CG_MAXITER) continue;
        if (cudaMemcpyAsync(stage.p + off[k], beta[k], sizeof(double) * (size_t)g[k].n, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess)
            failk(k, CSIPM_ERR_CUDA, "beta download failed");
        else
            copied[k] = 1;
    }
    const bool synced = cudaStreamSynchronize(st) == cudaSuccess;
    for (int k = 0; k < K; ++k) {
        if (!synced && h[k]) failk(k, CSIPM_ERR_CUDA, "stream synchronisation failed");
        else if (copied[k]) std::memcpy(g[k].req.beta_out, stage.p + off[k], sizeof(double) * (size_t)g[k].n);
    }
    for (int k = 0; k < K; ++k) {
        if (h[k]) csipm_destroy(h[k]);
        if (z0[k]) cudaFreeAsync(z0[k], st);
        if (beta[k]) cudaFreeAsync(beta[k], st);
        res[k].status = status[k];
        if (status[k] != CSIPM_OK) set_message(&res[k], msg[k].c_str());
    }
    cudaStreamSynchronize(st);
}

void csipm_server_s::work(int slot) {
    (void)slot;
    cudaSetDevice(device);
    cudaStream_t st = nullptr;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    cudaMemPool_t pool = device_pool(device);
    PinnedStage stage;
    std::vector<Pending> got;
    std::vector<csipm_result> res;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu);
            bool ok = false;
            cv_work.wait(lk, [&] {
                ok = take(&got);
                return ok || (stopping && queue.empty());
            });
            if (!ok) break;   // shutting down and nothing left to run
        }
        run_group(got, cuda_graphs, st, pool, stage, res);
        const auto t_end = Clock::now();
        {
            std::lock_guard<std::mutex> lk(mu);
            for (size_t k = 0; k < got.size(); ++k) {
                res[k].latency_ms = std::chrono::duration<double, std::milli>(t_end - got[k].t_submit).count();
                in_use -= got[k].footprint;
                results.push_back(res[k]);
                ++finished;
            }
        }
        cv_done.notify_all();
        cv_work.notify_all();   // memory freed: a waiting request may fit now
    }
    cudaStreamDestroy(st);
}

extern "C" {

int csipm_footprint(int dim, const int* size, int precision, int64_t n_missing, size_t* bytes) {
    std::string err;
    int status = 0;
    if (!bytes) return fail(nullptr, CSIPM_ERR_INVALID, "null argument");
    if (!valid_dims(dim, size, &err, &status)) return fail(nullptr, status, err);
    *bytes = footprint_bytes(dim, size, precision, n_missing);
    return CSIPM_OK;
}

int csipm_server_create(const csipm_server_options* opt, csipm_server* out) {
    if (!out) return fail(nullptr, CSIPM_ERR_INVALID, "null argument");
    *out = nullptr;
    int dev = opt && opt->device >= 0 ? opt->device : -1;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return fail(nullptr, CSIPM_ERR_NO_DEVICE, "no CUDA device");
    if (cudaSetDevice(dev) != cudaSuccess) return fail(nullptr, CSIPM_ERR_NO_DEVICE, "cannot select the device");
    auto* s = new csipm_server_s();
    s->device = dev;
    s->slots = opt && opt->slots > 0 ? opt->slots : 8;
    s->cuda_graphs = opt && opt->cuda_graphs ? 1 : 0;
    s->batch = opt && opt->batch > 1 ? opt->batch : 1;
    s->batch_max_n = opt && opt->batch_max_n > 0 ? opt->batch_max_n : 0;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    s->budget = opt && opt->hbm_budget > 0 ? opt->hbm_budget : (size_t)(0.8 * (double)free_b);
    if (!device_pool(dev)) {
        delete s;
        return fail(nullptr, CSIPM_ERR_CUDA, "device memory pool creation failed");
    }
    for (int k = 0; k < s->slots; ++k) s->workers.emplace_back([s, k] { s->work(k); });
    *out = s;
    return CSIPM_OK;
}

int csipm_server_submit(csipm_server s, const csipm_request* r) {
    if (!s || !r || !r->problem.z0) return fail(nullptr, CSIPM_ERR_INVALID, "null argument");
    std::string err;
    int status = 0;
    if (!valid_dims(r->problem.dim, r->problem.size, &err, &status)) return fail(nullptr, status, err);
    Pending p;
    p.req = *r;
    p.footprint = footprint_bytes(r->problem.dim, r->problem.size, r->options.precision, r->problem.n_missing);
    p.n = (long long)r->problem.size[0] * (r->problem.dim >= 2 ? r->problem.size[1] : 1) *
          (r->problem.dim >= 3 ? r->problem.size[2] : 1);
    p.bclass = batch_class(r->problem);
    p.t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping) return fail(nullptr, CSIPM_ERR_INVALID, "server is shutting down");
        s->queue.push_back(p);
        ++s->submitted;
    }
    s->cv_work.notify_one();
    return CSIPM_OK;
}

int csipm_server_poll(csipm_server s, csipm_result* out, int max, int* n, int timeout_ms) {
    if (!s || !out || !n || max < 1) return fail(nullptr, CSIPM_ERR_INVALID, "bad argument");
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->results.empty() && timeout_ms != 0) {
        auto ready = [&] { return !s->results.empty() || s->finished == s->submitted; };
        if (timeout_ms < 0) s->cv_done.wait(lk, ready);
        else s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
    }
    int k = 0;
    while (k < max && !s->results.empty()) {
        out[k++] = s->results.front();
        s->results.pop_front();
    }
    *n = k;
    return CSIPM_OK;
}

int csipm_server_destroy(csipm_server s) {
    if (!s) return CSIPM_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    delete s;
    return CSIPM_OK;
}

}  // extern "C"
