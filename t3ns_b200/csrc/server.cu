// Request loop for independent ground-state solves on one GPU.
//
// A request is one Davidson solve of an effective Hamiltonian (a
// t3ns_heff_desc with its guess and diagonal).  Requests queue in arrival
// order and are admitted against a fixed device-memory budget: a worker
// thread takes the first queued request whose estimated footprint fits in
// what the running ones leave free (so a large request does not hold back
// smaller ones behind it), builds its plan, runs the solve on the plan's own
// stream -- concurrently with the other admitted requests, each matvec
// launch taking 1/k of the persistent grid while k solves run -- writes the
// result into the caller's buffer and releases its share of the budget.  A
// request larger than the whole budget is rejected at submission.
//
// The descriptor, guess/result and diagonal passed to submit must stay valid
// until the request has been waited for.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.h"
#include "heff_internal.h"

namespace t3ns {
namespace {

double now_s()
{
        return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
                .count();
}

struct Request {
        int64_t id = 0;
        const t3ns_heff_desc *desc = nullptr;
        int precision = T3NS_PREC_FP64;
        double *result = nullptr;
        const double *diag = nullptr;
        double tol = 1e-5;
        int max_its = 100, max_vecs = 30, keep = 2;
        int64_t bytes = 0;
        double t_submit = 0, t_start = 0, t_done = 0;
        int rc = T3NS_OK;
        double energy = 0;
        t3ns_davidson_info info{};
        bool done = false;
        std::string error;
};

}  // namespace

// Device bytes a solve of `desc` needs: operators (and their {hi, lo} copy
// in split precision), the plan's term table (upper bound: every instruction of
// every combination present) and tilings, the plan's staging vectors, and
// the Davidson basis V, VA plus its work vectors.
int64_t estimate_solve_bytes(const t3ns_heff_desc *d, int precision, int max_vecs)
{
        const int nops = d->isdmrg ? 2 : 3;
        int64_t op_elems = 0;
        for (int i = 0; i < nops; ++i)
                for (int k = 0; k < d->ops[i].nrops; ++k)
                        op_elems += d->ops[i].op_beginblock[k][d->ops[i].op_nblocks[k]];
        const int64_t n = d->block_off[d->nblocks];
        const int64_t npairs = d->pair_ptr[d->nblocks];
        int64_t tasks = 0;
        for (int64_t c = 0; c < d->combo_ptr[npairs]; ++c)
                tasks += d->MPOc_beg[d->combo_mpo[c] + 1] - d->MPOc_beg[d->combo_mpo[c]];
        const bool split = precision == T3NS_PREC_3XTF32;
        const bool bf = precision == T3NS_PREC_BF16X3;
        int64_t b = op_elems * (split ? 16 : bf ? 12 : 8);     // FP64 (+ {hi, lo} pairs)
        // the transposed operators of the contraction-ordered configurations
        // (rows padded to 4: bounded here by twice the operators; their {hi, lo}
        // pairs too in split precision) and their offsets per term
        b += op_elems * (split ? 32 : 16) + tasks * 3 * (int64_t) sizeof(int64_t);
        b += tasks * (int64_t) sizeof(HeffTask);
        b += kNumCfgs * npairs * (int64_t) (sizeof(HeffPair) + 4 * sizeof(HeffUnit));
        b += n * (16 + (split ? 8 : bf ? 4 : 0));             // plan staging (+ split input)
        b += n * 8 * (2 * (int64_t) std::max(max_vecs, 3) + 6); // basis + work vectors
        return b + b / 20 + (16 << 20);                      // 5% + 16 MiB slack
}

}  // namespace t3ns

using namespace t3ns;

struct t3ns_server {
        int64_t budget = 0, in_use = 0, peak = 0;
        int device = 0;
        int64_t next_id = 1;
        std::deque<Request *> queue;
        std::map<int64_t, Request *> reqs;
        std::mutex mu;
        std::condition_variable cv_work, cv_done;
        std::vector<std::thread> workers;
        bool stop = false;
        std::atomic<int> running{0};   // solves on the GPU (their matvecs share the SMs)

        void run(Request *r)
        {
                cudaSetDevice(device);
                t3ns_heff *h = nullptr;
                double *d_res = nullptr, *d_diag = nullptr;
                int rc = t3ns_heff_create(r->desc, r->precision, &h);
                // tune only while this solve has the GPU to itself: timings taken
                // beside other solves are skewed and would be cached for the size
                // bucket (later plans, here and elsewhere, start on the cached
                // choice); otherwise the plan keeps the bucket's cached or default
                // configuration
                if (rc == T3NS_OK && running.load() <= 1) rc = t3ns_heff_autotune(h, 1, 0, nullptr);
                if (rc == T3NS_OK) h->dp.share = &running;
                const int64_t n = r->desc->block_off[r->desc->nblocks];
                const size_t bytes = sizeof(double) * (size_t) std::max<int64_t>(n, 1);
                if (rc == T3NS_OK && (cudaMalloc(&d_res, bytes) != cudaSuccess ||
                                      cudaMalloc(&d_diag, bytes) != cudaSuccess)) {
                        cudaGetLastError();
                        rc = set_error(T3NS_E_NOMEM, "server: solve vectors");
                }
                if (rc == T3NS_OK &&
                    (cudaMemcpyAsync(d_res, r->result, bytes, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
                     cudaMemcpyAsync(d_diag, r->diag, bytes, cudaMemcpyHostToDevice, h->stream) != cudaSuccess))
                        rc = set_error(T3NS_E_CUDA, "server: upload");
                if (rc == T3NS_OK)
                        rc = t3ns_davidson_device(h, d_res, &r->energy, r->max_vecs, r->keep, r->tol,
                                                  r->max_its, d_diag, &r->info, h->stream);
                if (rc >= 0 && (cudaMemcpyAsync(r->result, d_res, bytes, cudaMemcpyDeviceToHost,
                                                h->stream) != cudaSuccess ||
                                cudaStreamSynchronize(h->stream) != cudaSuccess))
                        rc = set_error(T3NS_E_CUDA, "server: download");
                if (rc < 0) r->error = t3ns_last_error();
                cudaFree(d_res);
                cudaFree(d_diag);
                t3ns_heff_destroy(h);
                r->rc = rc;
        }

        void worker()
        {
                for (;;) {
                        Request *r = nullptr;
                        {
                                std::unique_lock<std::mutex> lk(mu);
                                auto fits = [&] {
                                        for (Request *q : queue)
                                                if (q->bytes <= budget - in_use) return true;
                                        return false;
                                };
                                // at shutdown the queue is drained first
                                cv_work.wait(lk, [&] { return fits() || (stop && queue.empty()); });
                                if (stop && queue.empty()) return;
                                for (auto it = queue.begin(); it != queue.end(); ++it)
                                        if ((*it)->bytes <= budget - in_use) {
                                                r = *it;
                                                queue.erase(it);
                                                break;
                                        }
                                if (!r) continue;
                                in_use += r->bytes;
                                peak = std::max(peak, in_use);
                                r->t_start = now_s();
                                running.fetch_add(1);
                        }
                        run(r);
                        {
                                std::lock_guard<std::mutex> lk(mu);
                                running.fetch_sub(1);
                                in_use -= r->bytes;
                                r->t_done = now_s();
                                r->done = true;
                        }
                        cv_work.notify_all();
                        cv_done.notify_all();
                }
        }
};

extern "C" {

int64_t t3ns_server_estimate_bytes(const t3ns_heff_desc *desc, int precision, int max_vecs)
{
        if (!desc || desc->nblocks < 0) return set_error(T3NS_E_ARG, "null descriptor");
        return estimate_solve_bytes(desc, precision, max_vecs);
}

int t3ns_server_create(int64_t budget_bytes, int max_inflight, t3ns_server **out)
{
        if (!out || budget_bytes <= 0 || max_inflight < 1)
                return set_error(T3NS_E_ARG, "server: need a positive budget and max_inflight >= 1");
        t3ns_server *s = new (std::nothrow) t3ns_server();
        if (!s) return set_error(T3NS_E_NOMEM, "server: host allocation");
        s->budget = budget_bytes;
        T3NS_CUDA_TRY(cudaGetDevice(&s->device));
        for (int i = 0; i < max_inflight; ++i) s->workers.emplace_back([s] { s->worker(); });
        *out = s;
        return T3NS_OK;
}

int t3ns_server_submit(t3ns_server *s, const t3ns_heff_desc *desc, int precision,
                       double *guess_and_result, const double *diagonal, double tol, int max_its,
                       int max_vecs, int keep, int64_t *id_out)
{
        if (!s || !desc || !guess_and_result || !diagonal || !id_out)
                return set_error(T3NS_E_ARG, "server: null argument");
        auto *r = new (std::nothrow) Request();
        if (!r) return set_error(T3NS_E_NOMEM, "server: host allocation");
        r->desc = desc;
        r->precision = precision;
        r->result = guess_and_result;
        r->diag = diagonal;
        r->tol = tol;
        r->max_its = max_its;
        r->max_vecs = max_vecs;
        r->keep = keep;
        r->bytes = estimate_solve_bytes(desc, precision, max_vecs);
        r->t_submit = now_s();
        std::lock_guard<std::mutex> lk(s->mu);
        if (r->bytes > s->budget) {
                const std::string msg = "server: request needs " + std::to_string(r->bytes) +
                                        " bytes, more than the whole budget of " +
                                        std::to_string(s->budget);
                delete r;
                return set_error(T3NS_E_LIMIT, msg);
        }
        r->id = s->next_id++;
        s->reqs[r->id] = r;
        s->queue.push_back(r);
        *id_out = r->id;
        s->cv_work.notify_all();
        return T3NS_OK;
}

int t3ns_server_wait(t3ns_server *s, int64_t id, t3ns_request_result *out)
{
        if (!s || !out) return set_error(T3NS_E_ARG, "server: null argument");
        Request *r = nullptr;
        {
                std::unique_lock<std::mutex> lk(s->mu);
                auto it = s->reqs.find(id);
                if (it == s->reqs.end()) return set_error(T3NS_E_ARG, "server: unknown request");
                r = it->second;
                s->cv_done.wait(lk, [&] { return r->done; });
                s->reqs.erase(it);
        }
        out->id = r->id;
        out->status = r->rc;
        out->energy = r->energy;
        out->info = r->info;
        out->bytes = r->bytes;
        out->queue_seconds = r->t_start - r->t_submit;
        out->run_seconds = r->t_done - r->t_start;
        out->latency_seconds = r->t_done - r->t_submit;
        const int rc = r->rc;
        const std::string err = r->error;
        delete r;
        if (rc < 0) return set_error(rc, err);
        return T3NS_OK;
}

int t3ns_server_stats(t3ns_server *s, int64_t *in_use, int64_t *peak, int *queued)
{
        if (!s) return set_error(T3NS_E_ARG, "server: null argument");
        std::lock_guard<std::mutex> lk(s->mu);
        if (in_use) *in_use = s->in_use;
        if (peak) *peak = s->peak;
        if (queued) *queued = (int) s->queue.size();
        return T3NS_OK;
}

void t3ns_server_destroy(t3ns_server *s)
{
        if (!s) return;
        {
                std::lock_guard<std::mutex> lk(s->mu);
                s->stop = true;
        }
        s->cv_work.notify_all();
        for (auto &t : s->workers) t.join();
        for (auto &kv : s->reqs) delete kv.second;
        delete s;
}

}  // extern "C"
