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

struct Pending {
    csipm_request req;
    size_t footprint;
    Clock::time_point t_submit;
};

}  // namespace

struct csipm_server_s {
    int device = 0;
    int slots = 0;
    int cuda_graphs = 0;
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
    bool take(Pending* out);             // with mu held
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

bool csipm_server_s::take(Pending* out) {
    const size_t avail = budget > in_use ? budget - in_use : 0;
    int look = 0;
    for (auto it = queue.begin(); it != queue.end() && look < ADMIT_LOOKAHEAD; ++it, ++look) {
        if (it->footprint <= avail) {
            *out = *it;
            in_use += it->footprint;
            queue.erase(it);
            return true;
        }
    }
    // nothing admitted runs and the head still does not fit: admit it alone
    // rather than wait forever (it then fails in csipm_create with OOM if the
    // device really cannot hold it)
    if (in_use == 0 && !queue.empty()) {
        *out = queue.front();
        in_use += out->footprint;
        queue.pop_front();
        return true;
    }
    return false;
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

void csipm_server_s::work(int slot) {
    (void)slot;
    cudaSetDevice(device);
    cudaStream_t st = nullptr;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    cudaMemPool_t pool = device_pool(device);
    PinnedStage stage;
    for (;;) {
        Pending p{};
        bool got = false;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] {
                got = take(&p);
                return got || (stopping && queue.empty());
            });
            if (!got) break;   // shutting down and nothing left to run
        }
        const auto t_start = Clock::now();
        csipm_result res{};
        res.tag = p.req.tag;
        res.footprint = p.footprint;
        res.queue_ms = std::chrono::duration<double, std::milli>(t_start - p.t_submit).count();
        const csipm_problem& pr = p.req.problem;
        const long long n = (long long)pr.size[0] * (pr.dim >= 2 ? pr.size[1] : 1) * (pr.dim >= 3 ? pr.size[2] : 1);
        double* z0 = nullptr;
        double* beta = nullptr;
        int status = CSIPM_OK;
        const char* msg = nullptr;
        std::string err;
        if (!pool || cudaMallocFromPoolAsync((void**)&z0, sizeof(double) * n, pool, st) != cudaSuccess ||
            cudaMallocFromPoolAsync((void**)&beta, sizeof(double) * n, pool, st) != cudaSuccess) {
            status = CSIPM_ERR_OOM;
            msg = "out of device memory (staging z0 / beta)";
        }
        if (status == CSIPM_OK && !stage.ensure(sizeof(double) * (size_t)n)) {
            status = CSIPM_ERR_OOM;
            msg = "pinned host allocation failed";
        }
        csipm_handle h = nullptr;
        if (status == CSIPM_OK) {
            std::memcpy(stage.p, pr.z0, sizeof(double) * (size_t)n);
            if (cudaMemcpyAsync(z0, stage.p, sizeof(double) * n, cudaMemcpyHostToDevice, st) != cudaSuccess) {
                status = CSIPM_ERR_CUDA;
                msg = "z0 upload failed";
            }
        }
        if (status == CSIPM_OK) {
            csipm_problem dp = pr;
            dp.z0 = z0;
            csipm_options o = p.req.options;
            o.stream = st;
            // a served handle lives for one solve: its graphs are captured
            // for that one solve, which pays off on the server's say-so only
            o.cuda_graphs = cuda_graphs;
            status = csipm_create(&dp, &o, &h);
            if (status != CSIPM_OK) err = csipm_last_error(nullptr);
        }
        if (status == CSIPM_OK) {
            status = csipm_solve(h, beta, nullptr, &res.stats);
            if (status != CSIPM_OK) err = h->err;
            if (status == CSIPM_OK || status == CSIPM_ERR_IPM_MAXITER || status == CSIPM_ERR_CG_MAXITER) {
                if (p.req.beta_out &&
                    cudaMemcpyAsync(stage.p, beta, sizeof(double) * n, cudaMemcpyDeviceToHost, st) != cudaSuccess) {
                    status = CSIPM_ERR_CUDA;
                    msg = "beta download failed";
                }
                if (cudaStreamSynchronize(st) != cudaSuccess) {
                    status = CSIPM_ERR_CUDA;
                    msg = "stream synchronisation failed";
                }
                if (status != CSIPM_ERR_CUDA && p.req.beta_out)
                    std::memcpy(p.req.beta_out, stage.p, sizeof(double) * (size_t)n);
            }
        }
        if (status != CSIPM_OK) set_message(&res, msg ? msg : err.c_str());
        if (h) csipm_destroy(h);
        if (z0) cudaFreeAsync(z0, st);
        if (beta) cudaFreeAsync(beta, st);
        cudaStreamSynchronize(st);
        res.status = status;
        res.latency_ms = std::chrono::duration<double, std::milli>(Clock::now() - p.t_submit).count();
        {
            std::lock_guard<std::mutex> lk(mu);
            in_use -= p.footprint;
            results.push_back(res);
            ++finished;
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
