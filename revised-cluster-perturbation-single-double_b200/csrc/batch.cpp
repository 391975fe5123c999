// Independent molecules in one call: each molecule's whole SF-CIS +
// SF-CPS(D-3) pipeline (cpsd_pipeline) runs on one of a pool of host worker
// threads, each with its own CUDA stream, library context (plan caches,
// scratch arena, mailboxes) and device-driven solver loops, so the launches
// of different molecules overlap on the GPU: the small molecules' latency-
// bound steps fill the gaps of the large ones.  Molecules are taken largest
// first.  The reference runs one molecule per program invocation; there is
// no counterpart of this entry in it.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "drivers.hpp"

namespace cpsd {

namespace {

// persistent workers: their thread-local plan caches and arenas are reused
// by the next batch
struct Workers {
    std::mutex m;
    std::condition_variable cv;
    std::deque<std::function<void()>> jobs;
    int nthreads = 0;

    void ensure(int n, int device) {
        std::lock_guard<std::mutex> lock(m);
        for (; nthreads < n; nthreads++) std::thread([this, device] { run(device); }).detach();
    }
    void run(int device) {
        in_pool_worker() = true;
        cudaSetDevice(device);
        cudaStream_t s = nullptr;
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        ctx().stream = s;
        for (;;) {
            std::function<void()> job;
            {
                std::unique_lock<std::mutex> lock(m);
                cv.wait(lock, [this] { return !jobs.empty(); });
                job = std::move(jobs.front());
                jobs.pop_front();
            }
            job();
        }
    }
    void submit(std::function<void()> f) {
        {
            std::lock_guard<std::mutex> lock(m);
            jobs.push_back(std::move(f));
        }
        cv.notify_one();
    }
};
Workers &workers() {
    static Workers *w = new Workers;  // never destroyed: the threads outlive static destruction
    return *w;
}

// work estimate of a molecule: the particle-particle ladder, v^4 o^2 / nirrep
double weight(const cpsd_system *s) {
    double o = 0, v = 0;
    for (int r = 0; r < 8; r++) {
        o += (double)(s->popa[r] + s->popb[r]);
        v += (double)(s->vrta[r] + s->vrtb[r]);
    }
    return v * v * v * v * o * o / (double)std::max<int64_t>(s->nirrep, 1);
}

}  // namespace

bool &in_pool_worker() {
    thread_local bool w = false;
    return w;
}

void pool_submit(int nthreads, std::function<void()> job) {
    int device = 0;
    cudaGetDevice(&device);
    Workers &W = workers();
    W.ensure(nthreads, device);
    W.submit(std::move(job));
}

}  // namespace cpsd

using namespace cpsd;

extern "C" {

int cpsd_pipeline_batch(int64_t nmol, const cpsd_system *s, const cpsd_integrals *I, const cpsd_params *p,
                        int64_t nworkers, double *omega_cis, double *w2, double *w3, int64_t *nroots) {
    if (nmol < 0 || (nmol > 0 && (!s || !I || !p || !omega_cis || !w2 || !w3)))
        return set_error(CPSD_EARG, "pipeline_batch: null argument");
    if (nworkers < 1 || nworkers > 64) return set_error(CPSD_EARG, "pipeline_batch: 1..64 workers");
    std::vector<int64_t> off((size_t)nmol + 1, 0);
    for (int64_t m = 0; m < nmol; m++) {
        int64_t n = 0;
        for (int h = 0; h < 8; h++) n += p[m].estate_sym[h];
        off[(size_t)m + 1] = off[(size_t)m] + n;
    }
    if (nroots) *nroots = off[(size_t)nmol];
    if (nmol == 0) return CPSD_OK;
    std::vector<int64_t> order((size_t)nmol);
    for (int64_t m = 0; m < nmol; m++) order[(size_t)m] = m;
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t a, int64_t b) { return weight(s + a) > weight(s + b); });
    int device = 0;
    CPSD_TRY(cuda_check(cudaGetDevice(&device), "cudaGetDevice"));
    // the batch starts after the caller's stream work (its integrals)
    cudaEvent_t ready;
    CPSD_TRY(cuda_check(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming), "event"));
    CPSD_TRY(cuda_check(cudaEventRecord(ready, stream()), "event record"));
    const int digits = ctx().oz_digits;
    const double min_flops = ctx().oz_min_flops;
    Workers &W = workers();
    W.ensure((int)nworkers, device);
    std::mutex dm;
    std::condition_variable dcv;
    int64_t done = 0, launches = 0;
    double flops = 0;
    int first_rc = CPSD_OK;
    std::string first_msg;
    std::atomic<int64_t> next{0};
    const int64_t njobs = std::min<int64_t>(nworkers, nmol);
    for (int64_t j = 0; j < njobs; j++) {
        W.submit([&] {
            Context &c = ctx();
            c.oz_digits = digits;
            c.oz_min_flops = min_flops;
            c.mem_share = 1.0 / (double)njobs;
            const int64_t l0 = c.launches;
            const double f0 = c.flops;
            int rc = cuda_check(cudaStreamWaitEvent(c.stream, ready, 0), "stream wait");
            for (int64_t k; rc == CPSD_OK && (k = next.fetch_add(1)) < nmol;) {
                const int64_t m = order[(size_t)k];
                int64_t nr = 0;
                rc = cpsd_pipeline(s + m, I + m, p + m, omega_cis + off[(size_t)m], w2 + off[(size_t)m],
                                   w3 + off[(size_t)m], &nr);
                if (rc != CPSD_OK) next.store(nmol);  // stop handing out molecules
            }
            // an idle worker keeps no scratch: the next batch may run its
            // largest molecules on other workers
            if (!arena().external) arena().free_all();
            std::lock_guard<std::mutex> lock(dm);
            if (rc != CPSD_OK && first_rc == CPSD_OK) {
                first_rc = rc;
                first_msg = last_error();
            }
            launches += c.launches - l0;
            flops += c.flops - f0;
            done++;
            dcv.notify_one();
        });
    }
    {
        std::unique_lock<std::mutex> lock(dm);
        dcv.wait(lock, [&] { return done == njobs; });
    }
    cudaEventDestroy(ready);
    ctx().launches += launches;
    ctx().flops += flops;
    if (first_rc != CPSD_OK) return set_error(first_rc, "pipeline_batch: " + first_msg);
    return CPSD_OK;
}

int cpsd_release_device_cache(void) {
    CPSD_TRY(cuda_check(cudaStreamSynchronize(stream()), "sync"));
    pool_release_idle();
    if (!arena().external) arena().free_all();
    return CPSD_OK;
}

}  // extern "C"
