// serve.cu -- request loop for streams of SPD solves (continuous batching).
//
// No reference counterpart: the reference solves one system per call.  This
// server takes requests of mixed order N and right-hand-side count from host
// threads (CHAM_B200_Serve_Submit) and returns FP64-accurate solutions:
//
//   * small systems (N <= small_n, no factor kept) are coalesced: every such
//     request that arrived while the previous batch was on the GPU joins the
//     next launch of the uneven-size batched dposv (one persistent kernel, one
//     CTA per system, FP64 tile Cholesky), on the batch stream;
//   * larger systems run the mixed-precision solver (BF16x3 factorization +
//     FP64 iterative refinement, FP64 fallback) on one of `slots` worker
//     streams, each with its own executor and solver workspaces, so several
//     requests are on the GPU at once;
//   * a request with factor_key >= 0 and a matrix keeps its factor on the
//     device under that key (FP64 matrix + FP32 factor); a later request with
//     the same key and A == NULL only runs the solve and the refinement.
//
// Admission: a request starts only when its device memory fits in the HBM
// budget next to the running requests and the kept factors (unused kept
// factors are released least recently used first); among the queued large
// requests the shortest goes first unless the oldest has waited 50 ms.  A
// request larger than the whole budget starts when nothing else runs.  Each
// slot's factorization launch holds at most its share of the SMs, and a new
// matrix streams in (its referenced triangle) while it is being factored.  Times are CHAM_B200_Serve_Now() (CLOCK_MONOTONIC seconds).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/chameleon_b200.h"
#include "internal.h"

namespace chb {
namespace {

double now_s() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

// Grow-only device buffer.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    int reserve(size_t bytes) {
        if (bytes <= cap) return 0;
        dev_free(p);
        cap = 0;
        if (!(p = dev_alloc(bytes))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        cap = bytes;
        return 0;
    }
    ~DevBuf() { dev_free(p); }
};

// A factor kept on the device for later right-hand sides.
struct Kept {
    int64_t key = -1;
    int N = 0, uplo = ChamLower;
    double *A = nullptr;   // FP64 matrix (ld N); after an FP64 fallback it holds the FP64 factor
    bool fp64 = false;     // true: A holds the FP64 Cholesky factor, mws unused
    MixedWs mws;           // mws.A32 holds the FP32 factor
    ExecWs ews;
    size_t bytes = 0;
    int users = 0;         // requests running on it (guarded by the server mutex)
    std::mutex mu;         // one solve at a time per kept factor
    ~Kept() {
        dev_free(A);
        free_mixed_ws(mws);
        free_exec_ws(ews);
    }
};

struct Slot {
    cudaStream_t s = nullptr;
    ExecWs ews;
    MixedWs mws;
    DevBuf A, B, X;
    TriStreamState tri;   // copy stream of the request matrices (streamed triangle)
};

struct Server {
    int small_n = 512;
    double age_s = 0.05;   // a queued request older than this is served next (CHAMELEON_B200_SERVE_AGE_MS)
    size_t budget = 0;
    size_t used = 0;   // bytes of running requests + kept factors (guarded by mu)
    bool stop = false;
    std::mutex mu;
    std::condition_variable cv;        // wakes the workers
    std::condition_variable done_cv;   // wakes Drain
    std::deque<CHAM_b200_request_t *> large_q, small_q;
    int64_t inflight = 0;
    std::map<int64_t, std::shared_ptr<Kept>> kept;
    std::list<int64_t> lru;            // least recently used first
    std::vector<std::thread> threads;
    std::vector<std::unique_ptr<Slot>> slots;
    // batch stream
    cudaStream_t bs = nullptr;
    BatchWs bws;
    DevBuf bA, bB, binfo;
    // counters
    int64_t completed = 0, batches = 0, batched = 0, reused = 0, max_batch = 0;
};

int choose_nb(int N) { return N >= 4096 ? 512 : 256; }

constexpr int kReserveSMs = 16;        // SMs left to short kernels next to the slots' launches

size_t kept_bytes(int N) {
    const size_t n = N, nb = choose_nb(N), nt = (n + nb - 1) / nb;
    return n * n * 8 + nt * nt * nb * nb * 4 + nt * nb * nb * 4;   // FP64 A, FP32 tiles, inverse blocks
}

// Device bytes a request holds while it runs.
size_t need_bytes(const CHAM_b200_request_t *r, int small_n) {
    const size_t N = r->N, k = r->nrhs;
    if (!r->A) return 6 * N * k * 8;
    if (r->N <= small_n && r->factor_key < 0) return (N * N + N * k) * 8;
    const size_t nb = choose_nb(r->N), nt = (N + nb - 1) / nb;
    return N * N * 8 + nt * nt * nb * nb * (4 + 2) + 6 * N * k * 8 + ((size_t)16 << 20);
}

void finish(Server *sv, CHAM_b200_request_t *r, int status, int iters) {
    r->iterations = iters;
    r->t_done = now_s();
    std::lock_guard<std::mutex> lk(sv->mu);
    __atomic_store_n(&r->status, status, __ATOMIC_RELEASE);
    sv->completed++;
    if (--sv->inflight == 0) sv->done_cv.notify_all();
}

// Release unused kept factors, least recently used first, until `bytes`
// fits.  Caller holds sv->mu.
bool make_room(Server *sv, size_t bytes) {
    auto it = sv->lru.begin();
    while (sv->used + bytes > sv->budget && it != sv->lru.end()) {
        auto k = sv->kept.find(*it);
        if (k != sv->kept.end() && k->second->users == 0) {
            sv->used -= k->second->bytes;
            sv->kept.erase(k);   // freed here or when the last running user drops it
            it = sv->lru.erase(it);
        } else {
            ++it;
        }
    }
    return sv->used + bytes <= sv->budget;
}

int upload(void *dst, const double *src, int ld, int rows, int cols, cudaStream_t s) {
    CHB_CUDA(cudaMemcpy2DAsync(dst, (size_t)rows * 8, src, (size_t)ld * 8, (size_t)rows * 8, cols,
                               cudaMemcpyHostToDevice, s));
    return 0;
}

int download(double *dst, int ld, const void *src, int rows, int cols, cudaStream_t s) {
    CHB_CUDA(cudaMemcpy2DAsync(dst, (size_t)ld * 8, src, (size_t)rows * 8, (size_t)rows * 8, cols,
                               cudaMemcpyDeviceToHost, s));
    return 0;
}

struct Descs {
    CHAM_desc_t *A = nullptr, *B = nullptr, *X = nullptr;
    ~Descs() {
        if (A) CHAMELEON_Desc_Destroy(&A);
        if (B) CHAMELEON_Desc_Destroy(&B);
        if (X) CHAMELEON_Desc_Destroy(&X);
    }
};

// Diagnostics (CHAMELEON_B200_SERVE_TRACE=1): the host-side phases of every
// request whose service takes longer than 100 ms go to stderr.
bool serve_trace() {
    static const bool on = [] {
        const char *e = getenv("CHAMELEON_B200_SERVE_TRACE");
        return e && *e && *e != '0';
    }();
    return on;
}
struct PhaseLog {
    double t[8] = {0};
    const char *name[8] = {nullptr};
    int n = 0;
    void mark(const char *what) {
        if (n < 8) {
            t[n] = now_s();
            name[n++] = what;
        }
    }
    void report(const CHAM_b200_request_t *r, double t_start) const {
        if (!serve_trace() || n == 0 || t[n - 1] - t_start < 0.1) return;
        fprintf(stderr, "serve: N=%d nrhs=%d reuse=%d service %.1f ms:", r->N, r->nrhs, r->A ? 0 : 1,
                (t[n - 1] - t_start) * 1e3);
        double prev = t_start;
        for (int i = 0; i < n; ++i) {
            fprintf(stderr, " %s %.1f", name[i], (t[i] - prev) * 1e3);
            prev = t[i];
        }
        fprintf(stderr, "\n");
    }
};

// Mixed-precision solve of one request on slot `sl` (or on its kept factor).
int solve_large(Server *sv, Slot &sl, CHAM_b200_request_t *r, int *iters) {
    PhaseLog pl;
    const double t_in = now_s();
    const int N = r->N, nrhs = r->nrhs, NB = choose_nb(N);
    const int NT = (N + NB - 1) / NB;
    const cham_uplo_t uplo = (r->uplo == ChamUpper) ? ChamUpper : ChamLower;
    // Each slot's persistent launch holds at most its share of the SMs minus a
    // reserve: a CTA of it fills an SM's register file, so kernels of other
    // slots and of the batch stream could otherwise start only when it ends
    const int share = std::max(8, (ctx().num_sms - kReserveSMs) / (int)sv->slots.size());
    const int grid = std::min(share, std::max(8, NT * (NT + 1) * 4));
    cudaStream_t s = sl.s;
    const size_t bb = (size_t)N * nrhs * 8;
    if (int rc = sl.B.reserve(bb)) return rc;
    if (int rc = sl.X.reserve(bb)) return rc;
    if (int rc = upload(sl.B.p, r->B, r->ldb, N, nrhs, s)) return rc;
    pl.mark("B");

    std::shared_ptr<Kept> kp;
    if (!r->A) {   // solve with a kept factor
        std::lock_guard<std::mutex> lk(sv->mu);
        auto it = sv->kept.find(r->factor_key);
        if (it == sv->kept.end() || it->second->N != N || it->second->uplo != uplo) return CHAMELEON_ERR_NOT_FOUND;
        kp = it->second;
        kp->users++;
        sv->lru.remove(r->factor_key);
        sv->lru.push_back(r->factor_key);
        sv->reused++;
    } else if (r->factor_key >= 0) {
        kp = std::make_shared<Kept>();
        kp->key = r->factor_key;
        kp->N = N;
        kp->uplo = uplo;
        kp->bytes = kept_bytes(N);
        if (!(kp->A = (double *)dev_alloc((size_t)N * N * 8))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
    }
    const bool reuse = kp && !r->A;
    int iter = 0, rc = 0;
    {
        std::unique_lock<std::mutex> flock;
        if (kp) flock = std::unique_lock<std::mutex>(kp->mu);
        double *dA = nullptr;
        if (kp) {
            dA = kp->A;
        } else {
            rc = sl.A.reserve((size_t)N * N * 8);
            dA = (double *)sl.A.p;
        }
        // the referenced triangle of a new matrix streams in while the
        // factorization casts the columns that have landed
        const int nbf = factor_tile(NB);
        const bool stream_a = r->A && nbf % 64 == 0 && N > nbf && ctx().use_tcgen05;
        TriStream tri{};
        pl.mark("lock+alloc");
        if (!rc && r->A) {
            if (stream_a) rc = tri_stream_start(sl.tri, uplo, r->A, r->lda, dA, N, nbf, &tri);
            else rc = upload(dA, r->A, r->lda, N, N, s);
        }
        pl.mark("A");
        Descs d;
        if (!rc) rc = desc_create_cm(&d.A, dA, N, N, N, NB);
        if (!rc) rc = desc_create_cm(&d.B, (double *)sl.B.p, N, N, nrhs, NB);
        if (!rc) rc = desc_create_cm(&d.X, (double *)sl.X.p, N, N, nrhs, NB);
        if (!rc && reuse && kp->fp64) {
            // the kept matrix holds the FP64 factor: FP64 solve only
            if (cudaMemcpyAsync(sl.X.p, sl.B.p, bb, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
                rc = CHAMELEON_ERR_UNEXPECTED;
            ExecResult res;
            if (!rc) rc = run_cholesky_dag(MODE_SOLVE, uplo, d.A, d.X, s, &res, 0, &kp->ews, grid);
            if (!rc) rc = res.error ? res.error : res.info;
        } else if (!rc) {
            MixedWs &m = kp ? kp->mws : sl.mws;
            ExecWs &e = kp ? kp->ews : sl.ews;
            rc = mixed_posv_ws(uplo, CHAM_B200_PREC_BF16X3, d.A, d.B, d.X, &iter, nullptr, s, m, &e, grid, reuse,
                               stream_a ? &tri : nullptr);
            if (kp && iter < 0) kp->fp64 = true;   // the FP64 fallback factored the kept matrix in place
        }
        pl.mark("solve");
        if (!rc) rc = download(r->X, r->ldx, sl.X.p, N, nrhs, s);
        if (cudaStreamSynchronize(s) != cudaSuccess && !rc) rc = CHAMELEON_ERR_UNEXPECTED;
        // the request's host matrix is not read after it completes
        if (stream_a && cudaStreamSynchronize(sl.tri.cs) != cudaSuccess && !rc) rc = CHAMELEON_ERR_UNEXPECTED;
        pl.mark("X");
    }
    pl.report(r, t_in);
    *iters = iter;
    std::shared_ptr<Kept> replaced;   // released after the lock
    std::lock_guard<std::mutex> lk(sv->mu);
    if (reuse) {
        kp->users--;
    } else if (kp && rc == 0) {
        auto old = sv->kept.find(r->factor_key);
        if (old != sv->kept.end()) {   // replaced; freed when its last user drops it
            sv->used -= old->second->bytes;
            sv->lru.remove(r->factor_key);
            replaced = old->second;
        }
        sv->kept[r->factor_key] = kp;
        sv->lru.push_back(r->factor_key);
        sv->used += kp->bytes;
    }
    return rc;
}

void slot_worker(Server *sv, int idx) {
    Slot &sl = *sv->slots[idx];
    cudaSetDevice(ctx().device);
    while (true) {
        CHAM_b200_request_t *r = nullptr;
        size_t need = 0;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            // Shortest first (a solve with a kept factor counts as a quarter of
            // its order), so that small requests do not wait behind large
            // ones; a request that has waited age_s goes next whatever
            // its size, so that large ones are not starved.
            size_t pick = 0;
            auto choose = [&]() {
                pick = 0;
                if (now_s() - sv->large_q.front()->t_submit > sv->age_s) return;
                auto cost = [](const CHAM_b200_request_t *q) { return q->A ? (double)q->N : 0.25 * q->N; };
                for (size_t i = 1; i < sv->large_q.size(); ++i)
                    if (cost(sv->large_q[i]) < cost(sv->large_q[pick])) pick = i;
            };
            sv->cv.wait(lk, [&] {
                if (sv->large_q.empty()) return sv->stop;
                choose();
                const size_t nb = need_bytes(sv->large_q[pick], sv->small_n);
                return make_room(sv, nb) || sv->used == 0 || sv->stop;
            });
            if (sv->large_q.empty()) return;   // stop requested and nothing queued
            r = sv->large_q[pick];
            sv->large_q.erase(sv->large_q.begin() + (std::ptrdiff_t)pick);
            need = need_bytes(r, sv->small_n);
            sv->used += need;
        }
        r->t_start = now_s();
        int iters = 0;
        const int rc = solve_large(sv, sl, r, &iters);
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            sv->used -= need;
        }
        sv->cv.notify_all();
        finish(sv, r, rc, iters);
    }
}

void batch_worker(Server *sv) {
    cudaSetDevice(ctx().device);
    while (true) {
        std::vector<CHAM_b200_request_t *> batch;
        size_t need = 0;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            sv->cv.wait(lk, [&] { return sv->stop || !sv->small_q.empty(); });
            if (sv->small_q.empty()) return;
            // everything that arrived while the previous batch ran joins now,
            // up to the memory that fits next to the running requests
            while (!sv->small_q.empty()) {
                const size_t nb = need_bytes(sv->small_q.front(), sv->small_n);
                if (!batch.empty() && !make_room(sv, need + nb)) break;
                need += nb;
                batch.push_back(sv->small_q.front());
                sv->small_q.pop_front();
            }
            sv->used += need;
        }
        const double t0 = now_s();
        size_t na = 0, nx = 0;
        for (auto *r : batch) {
            na += (size_t)r->N * r->N;
            nx += (size_t)r->N * r->nrhs;
        }
        int rc = sv->bA.reserve(na * 8);
        if (!rc) rc = sv->bB.reserve(nx * 8);
        if (!rc) rc = sv->binfo.reserve(batch.size() * sizeof(int));
        std::vector<BatchItem> items(batch.size());
        std::vector<int> info(batch.size(), 0);
        size_t oa = 0, ob = 0;
        for (size_t i = 0; i < batch.size() && !rc; ++i) {
            auto *r = batch[i];
            r->t_start = t0;
            items[i] = BatchItem{(int64_t)oa, (int64_t)ob, r->N, r->nrhs, r->N, r->N, (int)i, 0};
            rc = upload((double *)sv->bA.p + oa, r->A, r->lda, r->N, r->N, sv->bs);
            if (!rc) rc = upload((double *)sv->bB.p + ob, r->B, r->ldb, r->N, r->nrhs, sv->bs);
            oa += (size_t)r->N * r->N;
            ob += (size_t)r->N * r->nrhs;
        }
        if (!rc && cudaMemsetAsync(sv->binfo.p, 0, batch.size() * sizeof(int), sv->bs) != cudaSuccess)
            rc = CHAMELEON_ERR_UNEXPECTED;
        // one launch per triangle: requests reading the upper triangle go
        // in a second launch on the same stream
        for (int upper = 0; upper < 2 && !rc; ++upper) {
            std::vector<BatchItem> launch;
            for (size_t i = 0; i < batch.size(); ++i)
                if ((batch[i]->uplo == ChamUpper) == (upper == 1)) launch.push_back(items[i]);
            if (!launch.empty())
                rc = launch_posv_batch(launch, (double *)sv->bA.p, (double *)sv->bB.p, upper, (int *)sv->binfo.p,
                                       sv->bs, sv->bws);
        }
        for (size_t i = 0; i < batch.size() && !rc; ++i)
            rc = download(batch[i]->X, batch[i]->ldx, (double *)sv->bB.p + items[i].b_off, batch[i]->N,
                          batch[i]->nrhs, sv->bs);
        if (!rc && cudaMemcpyAsync(info.data(), sv->binfo.p, batch.size() * sizeof(int), cudaMemcpyDeviceToHost,
                                   sv->bs) != cudaSuccess)
            rc = CHAMELEON_ERR_UNEXPECTED;
        if (cudaStreamSynchronize(sv->bs) != cudaSuccess && !rc) rc = CHAMELEON_ERR_UNEXPECTED;
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            sv->used -= need;
            sv->batches++;
            sv->batched += (int64_t)batch.size();
            sv->max_batch = std::max<int64_t>(sv->max_batch, (int64_t)batch.size());
        }
        sv->cv.notify_all();
        for (size_t i = 0; i < batch.size(); ++i) finish(sv, batch[i], rc ? rc : info[i], 0);
    }
}

}  // namespace
}  // namespace chb

using namespace chb;

extern "C" {

double CHAM_B200_Serve_Now(void) { return now_s(); }

int CHAM_B200_Serve_Create(CHAM_b200_server_t *out, int slots, double hbm_budget_bytes, int small_n) {
    int rc = ensure_init();
    if (rc) return rc;
    if (!out || slots < 1 || slots > 16 || small_n < 0 || small_n > 4096) return CHAMELEON_ERR_ILLEGAL_VALUE;
    Server *sv = new Server();
    sv->small_n = small_n;
    if (const char *e = getenv("CHAMELEON_B200_SERVE_AGE_MS")) {
        const double ms = atof(e);
        if (ms > 0) sv->age_s = ms * 1e-3;
    }
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    sv->budget = hbm_budget_bytes > 0 ? (size_t)hbm_budget_bytes : (size_t)(0.8 * (double)fr);
    // the requests' buffers and workspaces come from memory mapped now, not
    // on the request path (half the budget, at most 48 GB)
    pool_reserve(std::min(sv->budget / 2, (size_t)48 << 30));
    if (cudaStreamCreateWithFlags(&sv->bs, cudaStreamNonBlocking) != cudaSuccess) {
        delete sv;
        return CHAMELEON_ERR_UNEXPECTED;
    }
    for (int i = 0; i < slots; ++i) {
        sv->slots.emplace_back(new Slot());
        if (cudaStreamCreateWithFlags(&sv->slots.back()->s, cudaStreamNonBlocking) != cudaSuccess) {
            for (auto &sl : sv->slots)
                if (sl->s) cudaStreamDestroy(sl->s);
            cudaStreamDestroy(sv->bs);
            delete sv;
            return CHAMELEON_ERR_UNEXPECTED;
        }
    }
    sv->threads.emplace_back(batch_worker, sv);
    for (int i = 0; i < slots; ++i) sv->threads.emplace_back(slot_worker, sv, i);
    *out = reinterpret_cast<CHAM_b200_server_t>(sv);
    return 0;
}

int CHAM_B200_Serve_Submit(CHAM_b200_server_t srv, CHAM_b200_request_t *r) {
    Server *sv = reinterpret_cast<Server *>(srv);
    if (!sv || !r) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (r->N <= 0 || r->nrhs <= 0 || !r->B || !r->X || r->ldb < r->N || r->ldx < r->N)
        return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (r->uplo != ChamUpper && r->uplo != ChamLower) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (r->A ? (r->lda < r->N) : (r->factor_key < 0)) return CHAMELEON_ERR_ILLEGAL_VALUE;
    r->iterations = 0;
    r->t_submit = now_s();
    r->t_start = r->t_done = 0;
    __atomic_store_n(&r->status, CHAM_B200_REQ_PENDING, __ATOMIC_RELAXED);
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        if (sv->stop) return CHAMELEON_ERR_NOT_INITIALIZED;
        sv->inflight++;
        if (r->A && r->N <= sv->small_n && r->factor_key < 0) sv->small_q.push_back(r);
        else sv->large_q.push_back(r);
    }
    sv->cv.notify_all();
    return 0;
}

int CHAM_B200_Serve_Drain(CHAM_b200_server_t srv) {
    Server *sv = reinterpret_cast<Server *>(srv);
    if (!sv) return CHAMELEON_ERR_ILLEGAL_VALUE;
    std::unique_lock<std::mutex> lk(sv->mu);
    sv->done_cv.wait(lk, [&] { return sv->inflight == 0; });
    return 0;
}

int CHAM_B200_Serve_Stats(CHAM_b200_server_t srv, CHAM_b200_serve_stats_t *st) {
    Server *sv = reinterpret_cast<Server *>(srv);
    if (!sv || !st) return CHAMELEON_ERR_ILLEGAL_VALUE;
    std::lock_guard<std::mutex> lk(sv->mu);
    st->completed = sv->completed;
    st->batches = sv->batches;
    st->batched_requests = sv->batched;
    st->max_batch = sv->max_batch;
    st->reused_factors = sv->reused;
    st->kept_factors = (long long)sv->kept.size();
    st->bytes_in_use = (double)sv->used;
    st->budget_bytes = (double)sv->budget;
    return 0;
}

int CHAM_B200_Serve_Destroy(CHAM_b200_server_t srv) {
    Server *sv = reinterpret_cast<Server *>(srv);
    if (!sv) return CHAMELEON_ERR_UNALLOCATED;
    CHAM_B200_Serve_Drain(srv);
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv.notify_all();
    for (auto &t : sv->threads) t.join();
    sv->kept.clear();
    for (auto &sl : sv->slots) {
        cudaStreamSynchronize(sl->s);
        free_mixed_ws(sl->mws);
        free_exec_ws(sl->ews);
        cudaStreamDestroy(sl->s);
        free_tri_stream(sl->tri);
    }
    sv->slots.clear();
    cudaStreamSynchronize(sv->bs);
    dev_free(sv->bws.items);
    dev_free(sv->bws.scratch);
    dev_free(sv->bws.cursor);
    dev_free(sv->bws.info);
    sv->bA = DevBuf();
    sv->bB = DevBuf();
    sv->binfo = DevBuf();
    cudaStreamDestroy(sv->bs);
    delete sv;
    return 0;
}

}  // extern "C"
