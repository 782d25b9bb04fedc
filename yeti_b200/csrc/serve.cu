// Serving: a persistent request loop for WQ elasticity solves.
//
// No counterpart in the reference (YETI solves one model per Python call).
// Requests (a patch of any degree 2..5 and element counts, material, clamps,
// 1..8 right-hand sides) are queued by yeti_serve_submit.  One engine thread
// and a pool of worker threads serve them:
//   admission  (engine) in arrival order, while the number of active
//              requests is below the slot count and the estimated device
//              bytes of the request fit in the HBM budget next to the active
//              ones;
//   setup      (worker) the WQ operator on the device (yeti_wq_setup, FP64
//              data) and the start of one resumable FP64 Krylov solve per
//              right-hand side (CgSolve) in the request's mode: CG or
//              BiCGSTAB, Jacobi or fast-diagonalisation preconditioned (the
//              bench serves with fast-diagonalisation BiCGSTAB);
//   solve      (engine) the solves advance in chunks of iterations captured
//              in a CUDA graph, so that the solves of all active requests
//              overlap on the device; the engine polls chunk events and
//              relaunches until converged;
//   retire     (worker) solutions and true residuals copied out, operator
//              and workspaces freed (stream-ordered, no device-wide
//              synchronisation), budget released, waiters notified.
// Setups and retirements wait for host copies; on the engine thread they
// stalled the relaunch of every other request's chunks (measured: 30 ms per
// setup under load against 2 ms alone), so they run on the workers, each with
// its own context and a high-priority stream; the solve streams have the low
// priority.  Operators, Krylov vectors and scalars stay on the device for the
// life of a request; the host only sees one small scalar copy per chunk.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "wq.cuh"

namespace yeti {
namespace {

constexpr int kMaxRhs = 8;
constexpr int kStreams = 64;

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    int64_t ticket = 0;
    int p[3] = {0, 0, 0}, nel[3] = {0, 0, 0};
    std::vector<double> cps, weights, rhs;
    double E = 0, nu = 0, rtol = 0;
    int maxit = 0, nrhs = 0, mode = 0;
    uint8_t dir[18] = {};
    int64_t ndof = 0;
    size_t est = 0;
    yeti_wq_op *op = nullptr;
    std::vector<std::unique_ptr<CgSolve>> solves;
    std::vector<int> finished;   // per right-hand side: 0 running, 2 done, 3 breakdown
    int fail = YETI_OK;          // an error of the engine's polls
    std::vector<double> x;
    int iters[kMaxRhs] = {};
    double rel[kMaxRhs] = {};
    int status = 1;   // 1 pending, 0 done, < 0 error code
    std::string err;
    double t_submit = 0, t_admit = 0, t_done = 0;
};

// Device bytes a request may hold at its peak: the FP64 coefficients twice
// (element-block and streaming layouts during the re-layout), |det J|, the
// diagonal and its inverse, six vectors per right-hand side (CG; BiCGSTAB
// eleven), and tables; with fast diagonalisation two more vectors per
// right-hand side and the plan's two intermediate vectors and 1-D matrices.
size_t estimate_bytes(const Request &r) {
    int64_t nqp = 1, ncp = 1, mat = 0;
    for (int d = 0; d < 3; d++) {
        nqp *= 2 * (r.p[d] + r.nel[d]) - 1;
        ncp *= r.p[d] + r.nel[d];
        mat += 2 * (int64_t)(r.p[d] + r.nel[d]) * (r.p[d] + r.nel[d]);
    }
    const int64_t ndof = 3 * ncp;
    const int64_t fd = (r.mode & YETI_PCG_FD) ? 1 : 0;
    const int64_t vec = (r.mode & YETI_PCG_BICGSTAB) ? 11 : 6;
    return (size_t)(nqp * 45 * 8 * 2 + nqp * 8 + ndof * 8 * 2 +
                    (int64_t)r.nrhs * ((vec + 2 * fd) * ndof * 8 + 65536) +
                    fd * (2 * ndof * 8 + 3 * mat * 8)) + ((size_t)4 << 20);
}

}  // namespace
}  // namespace yeti

using namespace yeti;

struct yeti_server {
    yeti_ctx *ctx = nullptr;           // the engine's context
    size_t budget = 0;
    int max_active = 0;
    std::mutex mu;                     // everything below except `active`
    std::condition_variable cv_work;   // engine: new requests, ready solves, stop
    std::condition_variable cv_task;   // workers: new tasks, stop
    std::condition_variable cv_done;   // callers: finished requests
    std::deque<Request *> queue;       // submitted, not admitted
    std::deque<std::pair<int, Request *>> tasks;   // (0 setup | 1 retire, request)
    std::vector<Request *> ready;      // set up, first chunks launched
    std::map<int64_t, std::unique_ptr<Request>> reqs;
    std::vector<Request *> active;     // engine thread only
    std::vector<cudaStream_t> streams; // solve streams (low priority)
    void *pinned = nullptr;            // scalar slots of the CG solves
    std::vector<void *> free_slots;
    std::vector<yeti_ctx *> wctx;      // one context per worker (high-priority stream)
    // one stream per worker that only its worker uses, and only to capture
    // chunk graphs: no other thread enqueues into it (work enqueued into a
    // capturing stream would join the capture)
    std::vector<cudaStream_t> wcap;
    std::vector<std::thread> workers;
    int64_t next_ticket = 1;
    size_t committed = 0;
    int64_t n_done = 0;
    int n_active = 0, peak_active = 0;
    int rr = 0;
    // worker time in setups and retirements, engine time in polls (ms)
    double t_setup_ms = 0, t_retire_ms = 0, t_poll_ms = 0;
    bool stop = false, stop_workers = false;
    std::thread engine;

    // Release everything a request holds and publish its result (workers).
    void finish(Request *r, int status, const std::string &err) {
        for (auto &cs : r->solves) {
            // a failed request may still have chunks in flight: let them end
            // before the operator they read is freed
            if (cs->in_flight) cudaEventSynchronize(cs->ev);
            cs->release();
        }
        if (r->op) {
            yeti_wq_destroy(r->op);
            r->op = nullptr;
        }
        std::lock_guard<std::mutex> lk(mu);
        for (auto &cs : r->solves)
            if (cs->host_scal) free_slots.push_back(cs->host_scal);
        r->solves.clear();
        r->status = status;
        r->err = err;
        r->t_done = now_ms();
        committed -= r->est;
        n_active--;
        n_done++;
        cv_done.notify_all();
        cv_work.notify_one();   // a slot and budget are free again
    }

    // Worker: operator setup and start of the solves; the request then goes
    // to the engine through `ready`.
    void setup(Request *r, yeti_ctx *wc, cudaStream_t cap) {
        r->t_admit = now_ms();
        yeti_wq_op *op = nullptr;
        int rc = yeti_wq_setup(wc, r->p, r->nel, r->cps.data(), r->weights.data(), r->E, r->nu,
                               r->dir, YETI_WQ_F64, &op);
        if (rc != YETI_OK) {
            finish(r, rc, yeti_last_error());
            return;
        }
        r->op = op;
        r->ndof = op->ndof;
        r->x.assign((size_t)r->nrhs * r->ndof, 0.0);
        r->finished.assign(r->nrhs, 0);
        for (int k = 0; k < r->nrhs; k++) {
            std::unique_ptr<CgSolve> cs(new CgSolve());
            void *slot;
            cudaStream_t st;
            {
                std::lock_guard<std::mutex> lk(mu);
                slot = free_slots.back();
                free_slots.pop_back();
                st = streams[rr++ % (int)streams.size()];
            }
            // FD-preconditioned solves take tens of iterations: short chunks
            // (cheaper graphs, fewer iterations launched past convergence)
            const int chunk = (r->mode & YETI_PCG_FD) ? 4 : 0;
            rc = cgsolve_begin(*cs, op, st, slot, r->rhs.data() + (size_t)k * r->ndof, r->rtol,
                               r->maxit, cap, r->mode, chunk);
            cs->host_scal = slot;   // returned by finish whatever happened
            if (rc == YETI_OK) rc = cgsolve_launch(*cs);
            r->solves.push_back(std::move(cs));
            if (rc != YETI_OK) {
                // the failed solve may have start work queued on st that reads
                // the operator: let it end before finish frees the operator
                const std::string err = yeti_last_error();
                cudaStreamSynchronize(st);
                (void)cudaGetLastError();
                finish(r, rc, err);
                return;
            }
        }
        std::lock_guard<std::mutex> lk(mu);
        ready.push_back(r);
        cv_work.notify_one();
    }

    // Worker: copy the solutions out and retire the request.
    void retire(Request *r, yeti_ctx *wc) {
        int rc = r->fail;
        bool broke = false;
        for (int k = 0; k < r->nrhs && rc == YETI_OK; k++) {
            CgSolve &cs = *r->solves[k];
            r->iters[k] = cs.iterations;
            rc = cgsolve_finish(cs, r->x.data() + (size_t)k * r->ndof, wc->stream);
            r->rel[k] = cs.rel_residual;
            broke = broke || r->finished[k] == 3;
        }
        if (rc == YETI_OK && broke) {
            rc = YETI_EBREAKDOWN;
            set_error("serving: Krylov breakdown");
        }
        finish(r, rc, rc == YETI_OK ? std::string() : std::string(yeti_last_error()));
    }

    void work(int w) {
        cudaSetDevice(ctx->device);
        for (;;) {
            std::pair<int, Request *> t;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_task.wait(lk, [&] { return stop_workers || !tasks.empty(); });
                if (tasks.empty()) return;
                t = tasks.front();
                tasks.pop_front();
            }
            const double t0 = now_ms();
            if (t.first == 0) setup(t.second, wctx[w], wcap[w]);
            else retire(t.second, wctx[w]);
            std::lock_guard<std::mutex> lk(mu);
            (t.first == 0 ? t_setup_ms : t_retire_ms) += now_ms() - t0;
        }
    }

    // Engine: poll the solves of a request, relaunch chunks; true when every
    // right-hand side is finished (or an error occurred).
    bool progress(Request *r, bool &moved) {
        int left = 0;
        for (int k = 0; k < r->nrhs; k++) {
            if (r->finished[k]) continue;
            CgSolve &cs = *r->solves[k];
            int state = 0;
            int rc = cgsolve_poll(cs, &state);
            if (rc == YETI_OK && state == 1) {
                rc = cgsolve_launch(cs);
                moved = true;
            } else if (rc == YETI_OK && state >= 2) {
                r->finished[k] = state;
                moved = true;
            }
            if (rc != YETI_OK) {
                r->fail = rc;
                return true;
            }
            left += !r->finished[k];
        }
        return left == 0;
    }

    // Engine: admission, chunk relaunches, hand-over of finished requests.
    void run() {
        cudaSetDevice(ctx->device);
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                if (active.empty() && ready.empty())
                    cv_work.wait_for(lk, std::chrono::milliseconds(2), [&] {
                        return stop || !ready.empty() ||
                               (!queue.empty() && n_active < max_active &&
                                (!budget || committed + queue.front()->est <= budget));
                    });
                if (stop && active.empty() && ready.empty() && n_active == 0) {
                    for (Request *q : queue) {
                        q->status = YETI_EINVAL;
                        q->err = "serving: server closed before the request was admitted";
                        q->t_done = now_ms();
                    }
                    queue.clear();
                    stop_workers = true;
                    cv_task.notify_all();
                    cv_done.notify_all();
                    return;
                }
                while (!stop && !queue.empty() && n_active < max_active) {
                    Request *q = queue.front();
                    if (budget && committed + q->est > budget) break;   // in order
                    queue.pop_front();
                    committed += q->est;
                    n_active++;
                    peak_active = std::max(peak_active, n_active);
                    tasks.emplace_back(0, q);
                    cv_task.notify_one();
                }
                for (Request *q : ready) active.push_back(q);
                ready.clear();
            }
            const double t1 = now_ms();
            bool moved = false;
            for (size_t i = 0; i < active.size();) {
                Request *r = active[i];
                if (!progress(r, moved)) {
                    i++;
                    continue;
                }
                moved = true;
                active.erase(active.begin() + i);
                std::lock_guard<std::mutex> lk(mu);
                tasks.emplace_back(1, r);
                cv_task.notify_one();
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                t_poll_ms += now_ms() - t1;
            }
            if (!moved && !active.empty()) std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
};

// ---------------------------------------------------------------- C ABI
YETI_API int yeti_serve_open(int device, size_t hbm_budget_bytes, int max_active,
                             yeti_server **out) {
    YETI_CHECK(out, YETI_EINVAL, "yeti_serve_open: out is NULL");
    *out = nullptr;
    YETI_CHECK(max_active >= 1 && max_active <= 1024, YETI_EINVAL,
               "yeti_serve_open: max_active %d", max_active);
    std::unique_ptr<yeti_server> s(new yeti_server());
    YETI_TRY(yeti_ctx_create(device, hbm_budget_bytes, &s->ctx));
    s->ctx->stream_ordered = true;
    s->budget = hbm_budget_bytes;
    s->max_active = max_active;
    DeviceGuard g(device);
    int prio_low = 0, prio_high = 0;
    YETI_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    for (int i = 0; i < kStreams; i++) {
        cudaStream_t st;
        YETI_CUDA(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio_low));
        s->streams.push_back(st);
    }
    // keep the memory that retired requests free in the device's
    // stream-ordered pool instead of returning it to the driver at every
    // synchronisation
    {
        cudaMemPool_t pool;
        YETI_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t keep = hbm_budget_bytes ? (uint64_t)hbm_budget_bytes : UINT64_MAX, cur = 0;
        YETI_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur));
        if (cur < keep) YETI_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    constexpr int kWorkers = 4;
    for (int w = 0; w < kWorkers; w++) {
        yeti_ctx *wc = nullptr;
        YETI_TRY(yeti_ctx_create(device, 0, &wc));
        wc->stream_ordered = true;
        cudaStream_t hs;
        YETI_CUDA(cudaStreamCreateWithPriority(&hs, cudaStreamNonBlocking, prio_high));
        cudaStreamDestroy(wc->own_stream);
        wc->own_stream = hs;
        wc->stream = hs;
        s->wctx.push_back(wc);
        cudaStream_t cs;
        YETI_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        s->wcap.push_back(cs);
    }
    const size_t slot = (cgsolve_scal_bytes() + 127) / 128 * 128;
    const int nslots = max_active * kMaxRhs;
    YETI_CUDA(cudaMallocHost(&s->pinned, slot * nslots));
    for (int i = nslots - 1; i >= 0; i--)
        s->free_slots.push_back(static_cast<char *>(s->pinned) + slot * i);
    yeti_server *raw = s.get();
    for (int w = 0; w < kWorkers; w++) s->workers.emplace_back([raw, w] { raw->work(w); });
    s->engine = std::thread([raw] { raw->run(); });
    *out = s.release();
    return YETI_OK;
}

YETI_API int yeti_serve_submit(yeti_server *srv, const yeti_serve_request *q, int64_t *ticket) {
    YETI_CHECK(srv && q && ticket, YETI_EINVAL, "yeti_serve_submit: NULL argument");
    YETI_CHECK(q->cps && q->weights && q->rhs, YETI_EINVAL, "yeti_serve_submit: NULL array");
    YETI_CHECK(q->nrhs >= 1 && q->nrhs <= kMaxRhs, YETI_EINVAL,
               "yeti_serve_submit: nrhs %d not in 1..%d", q->nrhs, kMaxRhs);
    YETI_CHECK(q->rtol > 0 && q->maxit > 0, YETI_EINVAL, "yeti_serve_submit: rtol %g maxit %d",
               q->rtol, q->maxit);
    {
        const int fd_bits = YETI_PCG_FD | YETI_PCG_FD_SCALED | YETI_PCG_FD_UNIT | YETI_PCG_FD_TD;
        YETI_CHECK((q->mode & ~(fd_bits | YETI_PCG_BICGSTAB)) == 0 &&
                       ((q->mode & fd_bits) == 0 || (q->mode & YETI_PCG_FD)),
                   YETI_EINVAL, "yeti_serve_submit: mode %d (FP64 CG/BiCGSTAB, Jacobi/FD)",
                   q->mode);
    }
    std::unique_ptr<Request> r(new Request());
    int64_t ncp = 1;
    for (int d = 0; d < 3; d++) {
        YETI_CHECK(q->p[d] >= 2 && q->p[d] <= 8 && q->nel[d] >= 2 && q->nel[d] <= 4096,
                   YETI_EINVAL, "yeti_serve_submit: p[%d]=%d nel[%d]=%d", d, q->p[d], d,
                   q->nel[d]);
        r->p[d] = q->p[d];
        r->nel[d] = q->nel[d];
        ncp *= q->p[d] + q->nel[d];
    }
    r->ndof = 3 * ncp;
    r->cps.assign(q->cps, q->cps + 3 * ncp);
    r->weights.assign(q->weights, q->weights + ncp);
    r->rhs.assign(q->rhs, q->rhs + (size_t)q->nrhs * r->ndof);
    r->E = q->E;
    r->nu = q->nu;
    r->rtol = q->rtol;
    r->maxit = q->maxit;
    r->mode = q->mode;
    r->nrhs = q->nrhs;
    std::memcpy(r->dir, q->dirichlet, 18);
    r->est = estimate_bytes(*r);
    YETI_CHECK(!srv->budget || r->est <= srv->budget, YETI_ENOMEM,
               "yeti_serve_submit: request needs about %zu device bytes, budget %zu", r->est,
               srv->budget);
    std::lock_guard<std::mutex> lk(srv->mu);
    YETI_CHECK(!srv->stop, YETI_EINVAL, "yeti_serve_submit: server is closing");
    r->ticket = srv->next_ticket++;
    r->t_submit = now_ms();
    *ticket = r->ticket;
    srv->queue.push_back(r.get());
    srv->reqs[r->ticket] = std::move(r);
    srv->cv_work.notify_one();
    return YETI_OK;
}

static int take_result(yeti_server *srv, std::map<int64_t, std::unique_ptr<Request>>::iterator it,
                       double *x, yeti_serve_result *res) {
    Request *r = it->second.get();
    if (res) {
        std::memset(res, 0, sizeof(*res));
        res->status = r->status;
        res->ndof = r->ndof;
        res->nrhs = r->nrhs;
        for (int k = 0; k < r->nrhs; k++) {
            res->iterations[k] = r->iters[k];
            res->rel_residual[k] = r->rel[k];
        }
        res->queue_ms = r->t_admit > 0 ? r->t_admit - r->t_submit : r->t_done - r->t_submit;
        res->solve_ms = r->t_admit > 0 ? r->t_done - r->t_admit : 0.0;
        res->total_ms = r->t_done - r->t_submit;
    }
    const int status = r->status;
    if (status == YETI_OK && x) std::memcpy(x, r->x.data(), r->x.size() * sizeof(double));
    if (status != YETI_OK) set_error("%s", r->err.c_str());
    srv->reqs.erase(it);
    return status == YETI_OK ? 1 : status;
}

YETI_API int yeti_serve_poll(yeti_server *srv, int64_t ticket, double *x, yeti_serve_result *res) {
    YETI_CHECK(srv, YETI_EINVAL, "yeti_serve_poll: NULL server");
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->reqs.find(ticket);
    YETI_CHECK(it != srv->reqs.end(), YETI_EINVAL, "yeti_serve_poll: unknown ticket %lld",
               (long long)ticket);
    if (it->second->status == 1) return 0;
    return take_result(srv, it, x, res);
}

YETI_API int yeti_serve_wait(yeti_server *srv, int64_t ticket, double timeout_ms, double *x,
                             yeti_serve_result *res) {
    YETI_CHECK(srv, YETI_EINVAL, "yeti_serve_wait: NULL server");
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->reqs.find(ticket);
    YETI_CHECK(it != srv->reqs.end(), YETI_EINVAL, "yeti_serve_wait: unknown ticket %lld",
               (long long)ticket);
    Request *r = it->second.get();
    auto ready = [&] { return r->status != 1; };
    if (timeout_ms < 0) srv->cv_done.wait(lk, ready);
    else if (!srv->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready)) {
        set_error("yeti_serve_wait: ticket %lld not done after %g ms", (long long)ticket, timeout_ms);
        return YETI_ETIMEDOUT;
    }
    return take_result(srv, it, x, res);
}

YETI_API int yeti_serve_times(yeti_server *srv, double *setup_ms, double *retire_ms,
                              double *poll_ms) {
    YETI_CHECK(srv, YETI_EINVAL, "yeti_serve_times: NULL server");
    std::lock_guard<std::mutex> lk(srv->mu);
    if (setup_ms) *setup_ms = srv->t_setup_ms;
    if (retire_ms) *retire_ms = srv->t_retire_ms;
    if (poll_ms) *poll_ms = srv->t_poll_ms;
    return YETI_OK;
}

YETI_API int yeti_serve_stats(yeti_server *srv, int64_t *done, int64_t *queued, int32_t *active,
                              int32_t *peak_active, size_t *committed_bytes) {
    YETI_CHECK(srv, YETI_EINVAL, "yeti_serve_stats: NULL server");
    std::lock_guard<std::mutex> lk(srv->mu);
    if (done) *done = srv->n_done;
    if (queued) *queued = (int64_t)srv->queue.size();
    if (active) *active = srv->n_active;
    if (peak_active) *peak_active = srv->peak_active;
    if (committed_bytes) *committed_bytes = srv->committed;
    return YETI_OK;
}

YETI_API int yeti_serve_close(yeti_server *srv) {
    if (!srv) return YETI_OK;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stop = true;
        srv->cv_work.notify_all();
    }
    if (srv->engine.joinable()) srv->engine.join();
    for (auto &w : srv->workers)
        if (w.joinable()) w.join();
    for (yeti_ctx *wc : srv->wctx) yeti_ctx_destroy(wc);
    for (cudaStream_t cs : srv->wcap) cudaStreamDestroy(cs);
    {
        DeviceGuard g(srv->ctx->device);
        for (cudaStream_t st : srv->streams) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        if (srv->pinned) cudaFreeHost(srv->pinned);
    }
    yeti_ctx_destroy(srv->ctx);
    delete srv;
    return YETI_OK;
}
