// executor.cu -- persistent tile-DAG executor of the Cholesky factor/solve.
//
// Host side (device side: executor_kernel.cuh): record the sub-tile task DAG of chameleon_pdpotrf (compute/
// pzpotrf.c:84-194) and of the two chameleon_pdtrsm solves of dpotrs
// (compute/zpotrs.c:302-304 -> compute/pztrsm.c:58-200), order it by a
// list-scheduling simulation with critical-path priorities (the reference's
// task priorities `2*mt - 2*k - n - m`, compute/pzpotrf.c:90-124, play the same
// role for StarPU), cache it per shape, and launch one persistent kernel.
// Device side: dispatch by atomic cursor, bounded waits on per-tile counters,
// tile operations from core.cuh, release by red.release.
#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <memory>
#include <queue>
#include <unordered_map>
#include <cstring>

#include "core.cuh"
#include "internal.h"
#include "rec.cuh"
#include "tc05.cuh"

namespace chb {

// ---------------------------------------------------------------------------
// Host: DAG recording and list-scheduling order
// ---------------------------------------------------------------------------
namespace {

// Cost profile of the task kinds, per execution path: list-scheduling order
// depends on the relative durations, which differ a lot between the FP64 DMMA
// path and the tcgen05 path (where updates are ~6x cheaper relative to the
// panel tasks).  Multipliers of the flop model, calibrated from per-task
// device traces at NB = 512 (POTRF, TRSM, UPD, FWD/BWD TRSM, FWD/BWD UPD).
enum CostProfile : int { PROF_FP64 = 0, PROF_F32_MMA = 1, PROF_F32_TC05 = 2 };
// upd_fix: the fixed cost of one update task (C read and write, dispatch) in
// units of one panel's product, so that a group of cnt panels costs
// upd * (cnt + upd_fix) / (1 + upd_fix).
struct Calib {
    double potrf, trsm, upd, strsm, supd, upd_fix;
};
static const Calib kCalib[3] = {
    {4.9, 4.7, 5.8, 3.9, 7.1, 0.05},   // FP64 DMMA
    {4.0, 4.7, 2.1, 2.4, 3.3, 0.2},    // FP32, split products on mma.sync
    {4.2, 2.7, 0.92, 1.9, 4.0, 0.6},   // FP32, tcgen05 updates, full-inverse substitutions (row-block sub-tasks)
};

// Single-panel update groups at the end of each tile column, per cost profile
// (CHAMELEON_B200_UPD_TAIL_F64 for the FP64 path).
int upd_tail(int prof) { return prof == PROF_FP64 ? ctx().utail_f64 : UPD_TAIL; }

struct Shape {
    int mode, N, NB, nrhs, NBB, P, prof, G;   // G: update group size (upd_group_of)
    int h2d_gbs;                              // MODE_CAST: host-to-device bandwidth of the model (GB/s)
    int tail = UPD_TAIL;                      // single-panel groups at the end of each column
    bool operator==(const Shape &o) const {
        return mode == o.mode && N == o.N && NB == o.NB && nrhs == o.nrhs && NBB == o.NBB && P == o.P &&
               prof == o.prof && G == o.G && h2d_gbs == o.h2d_gbs && tail == o.tail;
    }
};
struct ShapeHash {
    size_t operator()(const Shape &s) const {
        size_t h = 1469598103934665603ull;
        for (int v : {s.mode, s.N, s.NB, s.nrhs, s.NBB, s.P, s.prof, s.G, s.h2d_gbs, s.tail})
            h = (h ^ (size_t)v) * 1099511628211ull;
        return h;
    }
};

constexpr int TK_COPY = 100;   // model only: the host-to-device copy of one tile column (not emitted)

struct Coarse {
    int16_t kind, m, n, k, bn;   // TK_UPD: k = first panel of the group, bn = panel count
    int grp;                     // TK_UPD: index of the group in tile column n
    bool virt = false;           // model-only task: runs on the copy engine, not on a CTA
    int nsub;
    double dur;               // duration of one sub-task (model units)
    std::vector<int> succ;
    int npred = 0;
    double blevel = 0;
};

struct Schedule {
    std::vector<Task> tasks;
    Task *d_tasks = nullptr;
    int npotrf = 0;              // POTRF tasks (for the dedicated CTA), their indices after the tasks
    const int *d_potrf = nullptr;
};

template <class NBI>
std::vector<Task> list_schedule(std::vector<Coarse> &ct, int P, NBI nbi);

std::vector<Task> build_order(const Shape &s) {
    const int NT = (s.N + s.NB - 1) / s.NB;
    const int NTB = s.nrhs > 0 ? (s.nrhs + s.NBB - 1) / s.NBB : 0;
    auto tm = [&](int m) { return (m == NT - 1) ? s.N - m * s.NB : s.NB; };
    auto nbi = [&](int m) { return (tm(m) + SUBB - 1) / SUBB; };
    auto wB = [&](int bn) { return (bn == NTB - 1) ? s.nrhs - bn * s.NBB : s.NBB; };
    const bool fact = s.mode & MODE_FACT, solve = s.mode & MODE_SOLVE;

    std::vector<Coarse> ct;
    ct.reserve(fact ? (size_t)NT * NT * NT / 6 + 4 * NT * NT : 4 * NT * NT + 8);
    auto add = [&](int kind, int m, int n, int k, int bn, int nsub, double dur) {
        Coarse c;
        c.kind = kind; c.m = m; c.n = n; c.k = k; c.bn = bn; c.grp = 0; c.nsub = nsub; c.dur = dur;
        ct.push_back(c);
        return (int)ct.size() - 1;
    };
    auto edge = [&](int a, int b) {
        if (a < 0 || b < 0) return;
        ct[a].succ.push_back(b);
        ct[b].npred++;
    };
    // ids: potrf[k], trsm[m,k], upd[m,n,k] (last update of tile (m,n) so far)
    std::vector<int> P(NT, -1), XI(NT, -1), Tr((size_t)NT * NT, -1), lastU((size_t)NT * NT, -1);
    std::vector<int> Cst((size_t)NT * NT, -1);   // MODE_CAST: cast task of tile (m, n)
    const bool cast = fact && (s.mode & MODE_CAST);
    const bool xinv = s.mode & MODE_XINV;
    const double nb = s.NB;
    const Calib &cal = kCalib[(s.prof >= 0 && s.prof < 3) ? s.prof : 0];
    // tcgen05 path: task durations in microseconds from per-task device traces
    // at NB = 256 and 512 (N = 32768; the diagonal factorization measured
    // alone, 1.05 t: under the full load it runs ~20% longer, but the lower
    // figure ordered the list best -- 1.25 t and 0.8 t both lengthened the
    // launch by 5-8%).  The diagonal and panel tasks there are
    // latency-bound and grow linearly with the tile order, not with its flops,
    // so a flop model misorders the list (tasks whose inputs are not ready are
    // claimed first and their CTAs wait).
    const bool lat = (s.prof == PROF_F32_TC05);
    auto c_potrf = [&](double t) { return lat ? 1.05 * t : cal.potrf * 6.0 * t * t * t / 3.0; };
    auto c_xinv = [&](double t) { return lat ? 1.5 * t : cal.potrf * 6.0 * t * t * t / 3.0; };
    auto c_trsm = [&]() { return lat ? 0.27 * nb : cal.trsm * 2.0 * SUBB * nb * nb; };
    auto c_upd = [&](int cnt) {
        return lat ? 5.0 + 0.011 * nb * cnt
                   : cal.upd * SUBB * SUBB * nb * 2.0 * (cnt + cal.upd_fix) / (1.0 + cal.upd_fix);
    };
    auto c_strsm = [&](double t, double w, int parts) {
        return lat ? 13.0 + 0.01 * t : cal.strsm * 3.0 * t * t * w / parts;
    };
    auto c_supd = [&](double t, double w) {
        return lat ? 8.0 + 0.04 * t : cal.supd * 2.0 * solve_rows(s.mode) * t * w;
    };
    if (cast) {
        // the copy engine delivers the stored triangle one tile column after
        // the other (model-only tasks, in order); each tile's cast waits for
        // its column
        const double gbs = std::max(1, s.h2d_gbs);
        int prev = -1;
        for (int q = 0; q < NT; ++q) {
            const double rows = (s.mode & MODE_CAST) ? (double)(s.N - q * s.NB) : 0.0;
            const double us = lat ? rows * tm(q) * 8.0 / (gbs * 1e3) : 0.0;
            const int cp = add(TK_COPY, q, q, q, 0, 1, us);
            ct[cp].virt = true;
            edge(prev, cp);
            prev = cp;
            // a column's copy covers tile column q of the lower triangle, or
            // tile row q's stored tiles of the upper one: the same tiles by symmetry
            for (int m = q; m < NT; ++m) {
                Cst[m + (size_t)NT * q] = add(TK_CAST, m, q, q, 0, 1, lat ? 8.0 * tm(m) * tm(q) / 65536.0 : 1.0);
                edge(cp, Cst[m + (size_t)NT * q]);
            }
        }
    }
    if (fact) {
        for (int k = 0; k < NT; ++k) {
            const double tk = tm(k);
            P[k] = add(TK_POTRF, k, k, k, 0, 1, c_potrf(tk));
            edge(lastU[k + (size_t)NT * k], P[k]);
            if (k == 0) edge(Cst[0], P[k]);
            if (xinv && solve) {
                XI[k] = add(TK_XINV, k, k, k, 0, 1, c_xinv(tk));
                edge(P[k], XI[k]);
            }
            for (int m = k + 1; m < NT; ++m) {
                const int id = add(TK_TRSM, m, k, k, 0, nbi(m), c_trsm());
                edge(P[k], id);
                edge(lastU[m + (size_t)NT * k], id);
                if (k == 0) edge(Cst[m], id);
                Tr[m + (size_t)NT * k] = id;
            }
            // the update groups of each later tile column whose last panel is k
            // (upd_group_of): they become ready with this step's panel solves
            for (int n = k + 1; n < NT; ++n) {
                int k0, cnt, gi;
                upd_group_of(n, k, s.G, s.tail, &k0, &cnt, &gi);
                if (k0 + cnt - 1 != k) continue;
                for (int m = n; m < NT; ++m) {
                    const int sub = (m == n) ? nbi(m) * (nbi(m) + 1) / 2 : nbi(m) * nbi(n);
                    const double dur = c_upd(cnt);
                    const int id = add(TK_UPD, m, n, k0, cnt, sub, dur);
                    ct[id].grp = gi;
                    if (gi == 0) edge(Cst[m + (size_t)NT * n], id);
                    edge(Tr[m + (size_t)NT * k], id);
                    if (m != n) edge(Tr[n + (size_t)NT * k], id);
                    edge(lastU[m + (size_t)NT * n], id);
                    lastU[m + (size_t)NT * n] = id;
                }
            }
        }
    } else if (solve && !(s.mode & MODE_NOINV)) {
        for (int k = 0; k < NT; ++k) {
            if (xinv) XI[k] = add(TK_XINV, k, k, k, 0, 1, c_xinv(tm(k)));
            else P[k] = add(TK_INV, k, k, k, 0, 1, 1.0 * tm(k) * IB * IB);
        }
    }
    if (solve) {
        // substitution row blocks (SOLB rows with full tile inverses)
        const int srb = solve_rows(s.mode);
        auto nsb = [&](int m) { return (tm(m) + srb - 1) / srb; };
        std::vector<int> F((size_t)NT * NTB, -1), lastFU((size_t)NT * NTB, -1);
        std::vector<int> Bk((size_t)NT * NTB, -1), lastBU((size_t)NT * NTB, -1);
        for (int bn = 0; bn < NTB; ++bn) {
            const double w = wB(bn);
            for (int k = 0; k < NT; ++k) {
                // MODE_XINV: one sub-task per row block (each applies its rows of the inverse)
                const int f = add(TK_FWD_TRSM, k, k, k, bn, xinv ? nsb(k) : 1,
                                  c_strsm(tm(k), w, xinv ? nsb(k) : 1));
                edge(xinv ? XI[k] : P[k], f);
                edge(lastFU[k + (size_t)NT * bn], f);
                F[k + (size_t)NT * bn] = f;
                for (int m = k + 1; m < NT; ++m) {
                    const int u = add(TK_FWD_UPD, m, k, k, bn, nsb(m), c_supd(tm(k), w));
                    edge(f, u);
                    if (fact) edge(Tr[m + (size_t)NT * k], u);
                    edge(lastFU[m + (size_t)NT * bn], u);
                    lastFU[m + (size_t)NT * bn] = u;
                }
            }
            for (int k = NT - 1; k >= 0; --k) {
                const int b = add(TK_BWD_TRSM, k, k, k, bn, xinv ? nsb(k) : 1,
                                  c_strsm(tm(k), w, xinv ? nsb(k) : 1));
                edge(F[k + (size_t)NT * bn], b);
                edge(lastBU[k + (size_t)NT * bn], b);
                Bk[k + (size_t)NT * bn] = b;
                for (int m = k - 1; m >= 0; --m) {
                    const int u = add(TK_BWD_UPD, m, k, k, bn, nsb(m), c_supd(tm(k), w));
                    edge(b, u);
                    edge(lastBU[m + (size_t)NT * bn], u);
                    lastBU[m + (size_t)NT * bn] = u;
                }
            }
        }
    }
    return list_schedule(ct, s.P, nbi);
}

// List scheduling of a coarse DAG (generation order topological) on P
// workers with critical-path priorities; emits the sub-tasks in start order.
template <class NBI>
std::vector<Task> list_schedule(std::vector<Coarse> &ct, int P, NBI nbi) {
    // bottom levels (generation order is topological)
    for (int i = (int)ct.size() - 1; i >= 0; --i) {
        double b = 0;
        for (int sidx : ct[i].succ) b = std::max(b, ct[sidx].blevel);
        ct[i].blevel = b + ct[i].dur;
    }
    // list scheduling on s.P workers
    struct Ready {
        double prio; int id;
        bool operator<(const Ready &o) const { return prio < o.prio || (prio == o.prio && id > o.id); }
    };
    struct Fin {
        double t; int id;
        bool operator<(const Fin &o) const { return t > o.t; }
    };
    std::priority_queue<Ready> ready;
    std::priority_queue<Fin> running;
    std::vector<int> started(ct.size(), 0), finished(ct.size(), 0);
    double now = 0;
    // model-only tasks start as soon as they are ready, without a worker
    auto make_ready = [&](int i) {
        if (ct[i].virt) running.push({now + ct[i].dur, i});
        else ready.push({ct[i].blevel, i});
    };
    for (int i = 0; i < (int)ct.size(); ++i)
        if (ct[i].npred == 0) make_ready(i);
    std::vector<Task> out;
    size_t total = 0;
    for (auto &c : ct)
        if (!c.virt) total += c.nsub;
    out.reserve(total);
    int free_w = P;
    auto emit = [&](const Coarse &c, int j) {
        Task t{};
        t.kind = c.kind; t.m = c.m; t.n = c.n; t.k = c.k; t.bn = c.bn; t.sub = 0; t.grp = c.grp;
        if (c.kind == TK_UPD) {
            const int a = nbi(c.m);
            int bi = 0, bj = 0;
            if (c.m == c.n) {   // j-th lower sub-block (row-major over bi >= bj)
                int rem = j;
                bi = 0;
                while (rem > bi) { rem -= bi + 1; ++bi; }
                bj = rem;
            } else {
                bi = j / nbi(c.n);
                bj = j % nbi(c.n);
            }
            (void)a;
            t.sub = (int16_t)(bi | (bj << 8));
        } else if (c.kind == TK_TRSM || c.kind == TK_FWD_UPD || c.kind == TK_BWD_UPD || c.kind == TK_FWD_TRSM ||
                   c.kind == TK_BWD_TRSM) {
            t.sub = (int16_t)j;   // row block (the substitutions have one unless MODE_XINV)
        }
        out.push_back(t);
    };
    while (out.size() < total) {
        while (free_w > 0 && !ready.empty()) {
            const int id = ready.top().id;
            Coarse &c = ct[id];
            emit(c, started[id]);
            started[id]++;
            if (started[id] == c.nsub) ready.pop();
            running.push({now + c.dur, id});
            --free_w;
        }
        if (running.empty()) break;   // cannot happen for a well-formed DAG
        const Fin f = running.top();
        running.pop();
        now = f.t;
        if (!ct[f.id].virt) ++free_w;
        if (++finished[f.id] == ct[f.id].nsub) {
            for (int sidx : ct[f.id].succ)
                if (--ct[sidx].npred == 0) make_ready(sidx);
        }
    }
    return out;
}

std::mutex g_sched_mu;
std::unordered_map<Shape, std::unique_ptr<Schedule>, ShapeHash> g_sched;

// Device copy of a task list (and of its POTRF indices).
int upload_schedule(Schedule *sch) {
    if (!sch->tasks.empty()) {
        std::vector<int> pidx;
        for (size_t i = 0; i < sch->tasks.size(); ++i)
            if (sch->tasks[i].kind == TK_POTRF) pidx.push_back((int)i);
        const size_t tbytes = sch->tasks.size() * sizeof(Task);
        const size_t bytes = tbytes + pidx.size() * sizeof(int);
        if (!(sch->d_tasks = (Task *)dev_alloc(bytes))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        sch->npotrf = (int)pidx.size();
        sch->d_potrf = reinterpret_cast<const int *>(reinterpret_cast<const uint8_t *>(sch->d_tasks) + tbytes);
        cudaStream_t ms = meta_stream();
        if (cudaMemcpyAsync(sch->d_tasks, sch->tasks.data(), tbytes, cudaMemcpyHostToDevice, ms) != cudaSuccess ||
            (!pidx.empty() && cudaMemcpyAsync((void *)sch->d_potrf, pidx.data(), pidx.size() * sizeof(int),
                                              cudaMemcpyHostToDevice, ms) != cudaSuccess) ||
            cudaStreamSynchronize(ms) != cudaSuccess)
            return CHAMELEON_ERR_UNEXPECTED;
    }
    return 0;
}

Schedule *get_schedule(const Shape &s) {
    std::lock_guard<std::mutex> lk(g_sched_mu);
    auto it = g_sched.find(s);
    if (it != g_sched.end()) return it->second.get();
    auto sch = std::make_unique<Schedule>();
    sch->tasks = build_order(s);
    if (upload_schedule(sch.get())) return nullptr;
    Schedule *raw = sch.get();
    g_sched[s] = std::move(sch);
    return raw;
}

ExecWs g_ws;   // workspace of the synchronous API entry points

// Grow-only workspace buffers, stream-ordered (no device-wide synchronization).
int ensure_ws(ExecWs &w, size_t ctr_bytes, size_t inv_bytes) {
    if (!w.st) {
        if (!(w.st = (ExecState *)dev_alloc(sizeof(ExecState)))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        CHB_CUDA(cudaEventCreate(&w.e0));
        CHB_CUDA(cudaEventCreate(&w.e1));
    }
    if (ctr_bytes > w.ctr_bytes) {
        dev_free(w.ctr);
        w.ctr_bytes = 0;
        if (!(w.ctr = dev_alloc(ctr_bytes))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        w.ctr_bytes = ctr_bytes;
    }
    if (inv_bytes > w.inv_bytes) {
        dev_free(w.inv);
        w.inv_bytes = 0;
        if (!(w.inv = dev_alloc(inv_bytes))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        w.inv_bytes = inv_bytes;
    }
    return 0;
}

}  // namespace

TraceRec *g_trace_buf = nullptr;   // set by the tracing entry point (host-owned device buffer)
int g_trace_cap = 0;

// Kernel variants, one translation unit each (exec_*.cu).
int launch_dag_f64(const ExecParams &p, int grid, cudaStream_t s);
int launch_dag_f32(const ExecParams &p, int grid, cudaStream_t s);
int launch_dag_f32tc(const ExecParams &p, int grid, cudaStream_t s);
int launch_dag_tf32(const ExecParams &p, int grid, cudaStream_t s);

void free_exec_ws(ExecWs &w) {
    dev_free(w.xinv);
    dev_free(w.y);
    dev_free(w.split);
    dev_free(w.ctr);
    dev_free(w.inv);
    dev_free(w.st);
    if (w.e0) cudaEventDestroy(w.e0);
    if (w.e1) cudaEventDestroy(w.e1);
    w = ExecWs();
}

// A task list recorded by a caller (CHAM_B200_Dag_*), already checked and on
// the device; its update groups are single panels.
static thread_local const Schedule *t_given = nullptr;

int run_cholesky_dag(int mode, cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B, cudaStream_t s,
                     ExecResult *res, int split, ExecWs *wsp, int grid_req, int flags, const CastIn *cin) {
    Context &c = ctx();
    ExecWs &w = wsp ? *wsp : g_ws;
    const int N = A->n;
    const int NB = A->nb;
    const int NT = A->nt;
    const int nrhs = (B && (mode & MODE_SOLVE)) ? B->n : 0;
    const int NBB = B ? B->nb : NB;
    const int NTB = nrhs ? B->nt : 0;
    const bool f32 = (A->dtyp == ChamRealFloat);
    res->info = 0; res->error = 0; res->ms = 0.f;
    if (N == 0) return 0;
    if (nrhs && B->dtyp != A->dtyp) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (cin) {
        if (!f32 || !(mode & MODE_FACT)) return CHAMELEON_ERR_ILLEGAL_VALUE;
        mode |= MODE_CAST;
    }
    // tcgen05 trailing updates: FP32 factorization with BF16x3 products and
    // 64-aligned tiles (the split chunks are 64 wide in k).
    const bool tc = f32 && split == SPLIT_BF16X3 && (mode & MODE_FACT) && (NB % tc05::BK == 0) && NT > 1 &&
                    c.use_tcgen05;
    int rc = 0;
    // grid_req counts SMs; FP64 places two executor CTAs on each
    const int cps = f32 ? 1 : 2;
    const int grid = cps * ((grid_req > 0) ? std::min(grid_req, c.num_sms) : c.num_sms);
    const int prof = !f32 ? PROF_FP64 : (tc ? PROF_F32_TC05 : PROF_F32_MMA);
    const bool full_inv = f32 && c.rec_tile && NB <= (64 << rec::MAX_LVL);
    // FP32 substitutions with full diagonal-tile inverses: computed off the
    // critical path in a factor+solve launch, reused by later solve-only
    // launches on the same factor and workspace (flags & EXEC_REUSE_INV).
    const bool xinv = f32 && !full_inv && c.xinv_solve && (mode & MODE_SOLVE) && nrhs > 0 &&
                      NB <= (64 << rec::MAX_LVL);
    if (xinv) {
        mode |= MODE_XINV;
        if (!(mode & MODE_FACT) && (flags & EXEC_REUSE_INV) && w.xinv_owner == A->mat && w.xinv_nt == NT &&
            w.xinv_nb == NB && w.xinv_n == N)
            mode |= MODE_NOINV;
    }
    // The task list depends on N only through NT and the number of SUBB-row
    // blocks of the last tile row, and on nrhs only through NTB (the kernel
    // takes the exact sizes from the parameters): key the cache on that
    // canonical shape so that callers with many distinct N share schedules.
    // (the finer of the update and substitution row blocks decides)
    const int gran = std::min(SUBB, solve_rows(mode));
    const int last_sub = ((N - (NT - 1) * NB) + gran - 1) / gran;
    const int canonN = (NT - 1) * NB + std::min(NB, last_sub * gran);
    // nrhs enters the cost model (not the task list): keep it, with the last
    // block's width rounded up to 16, so that the costs stay close and the
    // number of distinct schedules stays small
    const int canonR = nrhs ? (NTB - 1) * NBB + std::min(NBB, ((nrhs - (NTB - 1) * NBB + 15) / 16) * 16) : 0;
    // update group size: fused k steps amortize the C round trip and the
    // dispatch of an update over G panels (CHAMELEON_B200_UPD_GROUP per path)
    const int G = t_given ? 1 : std::max(1, prof == PROF_FP64 ? c.kgroup_f64 : (tc ? c.kgroup_tc : c.kgroup_f32));
    Shape sh{mode, canonN, NB, canonR, NBB, grid, prof, G, cin ? std::max(1, cin->h2d_gbs) : 0, upd_tail(prof)};
    const Schedule *sch = t_given ? t_given : get_schedule(sh);
    if (!sch) return CHAMELEON_ERR_OUT_OF_RESOURCES;
    const int NIB = (NB + IB - 1) / IB;
    const size_t nctr = (size_t)(cin ? 3 : 2) * NT * NT + (size_t)4 * NT * std::max(NTB, 1) + NT;
    const size_t esz = f32 ? sizeof(float) : sizeof(double);
    const size_t inv_elems = full_inv ? (size_t)NT * NB * NB : (size_t)NT * NIB * IB * IB;
    rc = ensure_ws(w, nctr * sizeof(int), inv_elems * esz);
    if (rc) return rc;
    int rcA = desc_upload(A);
    if (rcA) return rcA;
    if (nrhs) {
        int rcB = desc_upload(B);
        if (rcB) return rcB;
    }
    ExecParams p{};
    p.tasks = sch->d_tasks;
    p.ntasks = (int)sch->tasks.size();
    // one CTA runs the diagonal-tile factorizations (its instruction cache stays
    // warm for their long unrolled leaves); the others skip them
    const bool dedicate = c.potrf_cta && grid > 1 && sch->npotrf > 1;
    p.npotrf = dedicate ? sch->npotrf : 0;
    p.potrf_idx = sch->d_potrf;
    p.mode = mode;
    p.upper = (uplo == ChamUpper);
    p.NT = NT; p.N = N; p.NB = NB;
    p.A = A->mat;
    p.a_off = priv(A)->dev.off;
    p.a_ld = priv(A)->dev.ld;
    p.NTB = NTB; p.nrhs = nrhs; p.NBB = NBB;
    p.B = nrhs ? B->mat : nullptr;
    p.b_off = nrhs ? priv(B)->dev.off : nullptr;
    p.b_ld = nrhs ? priv(B)->dev.ld : nullptr;
    int *ctr = (int *)w.ctr;
    p.updA = ctr;
    p.panA = ctr + (size_t)NT * NT;
    const size_t nb4 = (size_t)NT * std::max(NTB, 1);
    p.fwdB = ctr + (size_t)2 * NT * NT;
    p.fwdDone = p.fwdB + nb4;
    p.bwdB = p.fwdDone + nb4;
    p.bwdDone = p.bwdB + nb4;
    p.invd = w.inv;
    p.NIB = NIB;
    p.full_inv = full_inv ? 1 : 0;
    p.xinvDone = p.bwdDone + nb4;
    if (cin) {
        p.castDone = p.xinvDone + NT;
        p.csrc = cin->src;
        p.csrc_ld = cin->ld;
        p.carrive = cin->arrive;
        p.cepoch = cin->epoch;
        p.colsum = cin->colsum;
        p.covf = cin->ovf;
    }
    p.xinv = nullptr;
    if (xinv) {
        const size_t xbytes = (size_t)NT * NB * NB * sizeof(float);
        if (xbytes > w.xinv_bytes) {
            dev_free(w.xinv);
            w.xinv_bytes = 0;
            w.xinv_owner = nullptr;
            if (!(w.xinv = dev_alloc(xbytes))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
            w.xinv_bytes = xbytes;
        }
        p.xinv = w.xinv;
        if (!(mode & MODE_NOINV)) w.xinv_owner = nullptr;   // rewritten by this launch
        // forward-substitution results, same tile layout as B
        const size_t ybytes = (size_t)(priv(B)->cm_view ? B->lda : B->lm) * B->ln * sizeof(float);
        if (ybytes > w.y_bytes) {
            dev_free(w.y);
            w.y_bytes = 0;
            if (!(w.y = dev_alloc(ybytes))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
            w.y_bytes = ybytes;
        }
        p.Y = w.y;
    }
    p.st = w.st;
    p.trace = (g_trace_buf && g_trace_cap >= p.ntasks) ? g_trace_buf : nullptr;
    p.wait_budget_ns = (unsigned long long)c.wait_budget_us * 1000ull;
    p.kgroup = G;
    p.utail = sh.tail;
    if (tc) {
        p.split_nrb = (NB + SUBB - 1) / SUBB;
        p.split_nkc = NB / tc05::BK;
        const size_t tile_bytes = (size_t)p.split_nrb * p.split_nkc * 2 * tc05::CHUNK_BYTES;
        const size_t bytes = (size_t)NT * (NT - 1) / 2 * tile_bytes;
        if (bytes > w.split_bytes) {
            dev_free(w.split);
            w.split_bytes = 0;
            if (!(w.split = (uint8_t *)dev_alloc(bytes))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
            w.split_bytes = bytes;
        }
        p.split = w.split;
    }
    ExecState init{};
    init.info = INT_MAX;
    init.stuck_task = -1;
    CHB_CUDA(cudaMemsetAsync(ctr, 0, nctr * sizeof(int), s));
    CHB_CUDA(cudaMemcpyAsync(w.st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
    CHB_CUDA(cudaEventRecord(w.e0, s));
    if (p.ntasks > 0) {
        CHB_LAUNCHED(1);
        if (!f32) rc = launch_dag_f64(p, grid, s);
        else if (split == SPLIT_TF32X3) rc = launch_dag_tf32(p, grid, s);
        else if (tc) rc = launch_dag_f32tc(p, grid, s);
        else rc = launch_dag_f32(p, grid, s);
        if (rc) return rc;
    }
    CHB_CUDA(cudaEventRecord(w.e1, s));
    ExecState out{};
    CHB_CUDA(cudaMemcpyAsync(&out, w.st, sizeof(out), cudaMemcpyDeviceToHost, s));
    CHB_CUDA(cudaStreamSynchronize(s));
    CHB_CUDA(cudaEventElapsedTime(&res->ms, w.e0, w.e1));
    res->info = (out.info == INT_MAX) ? 0 : out.info;
    res->error = out.error;
    if (xinv && !(mode & MODE_NOINV) && res->info == 0 && res->error == 0) {
        w.xinv_owner = A->mat;   // the inverses now match this factor
        w.xinv_n = N;
        w.xinv_nt = NT;
        w.xinv_nb = NB;
    }
    if (out.error) {
        char msg[160];
        snprintf(msg, sizeof msg, "device wait budget exhausted at task %d (%d of %d done)",
                 out.stuck_task, out.done, p.ntasks);
        warning("run_cholesky_dag", msg);
    }
    return 0;
}

}  // namespace chb

// Trace hooks (tracing subsystem): size the per-task trace buffer, read it back.
extern "C" int CHAM_B200_Trace_Enable(int capacity) {
    using namespace chb;
    if (g_trace_buf) { cudaFree(g_trace_buf); g_trace_buf = nullptr; g_trace_cap = 0; }
    if (capacity <= 0) return 0;
    if (cudaMalloc(&g_trace_buf, (size_t)capacity * sizeof(TraceRec)) != cudaSuccess) {
        g_trace_buf = nullptr;
        return CHAMELEON_ERR_OUT_OF_RESOURCES;
    }
    cudaMemset(g_trace_buf, 0, (size_t)capacity * sizeof(TraceRec));
    g_trace_cap = capacity;
    return 0;
}
extern "C" int CHAM_B200_Trace_Read(void *host_out, int count) {
    using namespace chb;
    if (!g_trace_buf || count > g_trace_cap) return CHAMELEON_ERR_ILLEGAL_VALUE;
    return cudaMemcpy(host_out, g_trace_buf, (size_t)count * sizeof(TraceRec), cudaMemcpyDeviceToHost) ==
                   cudaSuccess
               ? 0
               : CHAMELEON_ERR_UNEXPECTED;
}
// Copy the schedule of a shape into `out` (host only; used by the CPU tests of
// the DAG logic and by the trace tooling).  Returns the task count written.
extern "C" int CHAM_B200_Schedule_Build(int mode, int N, int NB, int nrhs, int NBB, int workers, int prof, int kgroup,
                                        void *out, int cap) {
    using namespace chb;
    const std::vector<Task> t =
        build_order(Shape{mode, N, NB, nrhs, NBB, workers, prof, std::max(1, kgroup), (mode & MODE_CAST) ? 50 : 0,
                          upd_tail(prof)});
    const int n = std::min<int>((int)t.size(), cap);
    memcpy(out, t.data(), sizeof(Task) * (size_t)n);
    return n;
}
// Number of tasks of the schedule of a given shape (for tests and tracing).
extern "C" int CHAM_B200_Schedule_Size(int mode, int N, int NB, int nrhs, int NBB, int workers, int prof, int kgroup) {
    using namespace chb;
    return (int)build_order(Shape{mode, N, NB, nrhs, NBB, workers, prof, std::max(1, kgroup),
                                  (mode & MODE_CAST) ? 50 : 0, upd_tail(prof)})
        .size();
}

// ---------------------------------------------------------------------------
// Recorded DAGs: tile tasks submitted by a caller (a Chameleon runtime plugin
// whose INSERT_TASK_* calls append here; chameleon_pzpotrf / chameleon_pztrsm
// run unchanged above it) and run by the persistent executor.
// ---------------------------------------------------------------------------
struct cham_b200_dag_s {
    std::vector<std::array<int, 5>> rec;   // kind, m, n, k, bn in submission order
};

namespace chb {
namespace {

// The executor's counter predicates (executor_kernel.cuh task_deps, update
// groups of one panel), replayed on a task list: true when every task's
// inputs are complete once every task before it has run, i.e. the list is
// deadlock-free for any number of CTAs.
bool replay_ok(const std::vector<Task> &tl, int mode, int N, int NB, int NTB) {
    const int NT = (N + NB - 1) / NB;
    auto tm = [&](int m) { return (m == NT - 1) ? N - m * NB : NB; };
    auto nbi = [&](int m) { return (tm(m) + SUBB - 1) / SUBB; };
    auto S = [&](int m, int n) { return m == n ? nbi(m) * (nbi(m) + 1) / 2 : nbi(m) * nbi(n); };
    const bool fact = mode & MODE_FACT;
    const size_t nb4 = (size_t)NT * std::max(NTB, 1);
    std::vector<int> upd((size_t)NT * NT, 0), pan((size_t)NT * NT, 0), fB(nb4, 0), fD(nb4, 0), bB(nb4, 0), bD(nb4, 0);
    for (const Task &t : tl) {
        bool ok = true;
        const size_t kb = t.k + (size_t)NT * t.bn, mb = t.m + (size_t)NT * t.bn;
        switch (t.kind) {
        case TK_POTRF: ok = upd[t.k + (size_t)NT * t.k] >= t.k * S(t.k, t.k); pan[t.k + (size_t)NT * t.k]++; break;
        case TK_INV: pan[t.k + (size_t)NT * t.k]++; break;
        case TK_TRSM:
            ok = pan[t.k + (size_t)NT * t.k] >= 1 && upd[t.m + (size_t)NT * t.k] >= t.k * S(t.m, t.k);
            pan[t.m + (size_t)NT * t.k]++;
            break;
        case TK_UPD:
            ok = t.bn == 1 && pan[t.m + (size_t)NT * t.k] >= nbi(t.m) && pan[t.n + (size_t)NT * t.k] >= nbi(t.n) &&
                 upd[t.m + (size_t)NT * t.n] >= t.k * S(t.m, t.n);
            upd[t.m + (size_t)NT * t.n]++;
            break;
        case TK_FWD_TRSM: ok = pan[t.k + (size_t)NT * t.k] >= 1 && fB[kb] >= t.k; fD[kb]++; break;
        case TK_FWD_UPD: ok = fD[kb] >= 1 && (!fact || pan[t.m + (size_t)NT * t.k] >= nbi(t.m)) && fB[mb] >= t.k; fB[mb]++; break;
        case TK_BWD_TRSM: ok = fD[kb] >= 1 && bB[kb] >= NT - 1 - t.k; bD[kb]++; break;
        case TK_BWD_UPD: ok = bD[kb] >= 1 && bB[mb] >= NT - 1 - t.k; bB[mb]++; break;
        default: ok = false;
        }
        if (!ok) return false;
    }
    return true;
}

}  // namespace
}  // namespace chb

extern "C" {

int CHAM_B200_Dag_Create(CHAM_b200_dag_t *dag) {
    if (!dag) return CHAMELEON_ERR_ILLEGAL_VALUE;
    *dag = new cham_b200_dag_s();
    return 0;
}
int CHAM_B200_Dag_Destroy(CHAM_b200_dag_t dag) {
    delete dag;
    return 0;
}
int CHAM_B200_Dag_Clear(CHAM_b200_dag_t dag) {
    if (!dag) return CHAMELEON_ERR_ILLEGAL_VALUE;
    dag->rec.clear();
    return 0;
}
int CHAM_B200_Dag_Record(CHAM_b200_dag_t dag, int kind, int m, int n, int k, int bn) {
    using namespace chb;
    if (!dag || kind < CHAM_B200_DAG_POTRF || kind > CHAM_B200_DAG_BWD_UPDATE || m < 0 || n < 0 || k < 0 || bn < 0)
        return CHAMELEON_ERR_ILLEGAL_VALUE;
    dag->rec.push_back({kind, m, n, k, bn});
    return 0;
}
int CHAM_B200_Dag_Size(CHAM_b200_dag_t dag) { return dag ? (int)dag->rec.size() : CHAMELEON_ERR_ILLEGAL_VALUE; }
int CHAM_B200_Dag_Get(CHAM_b200_dag_t dag, int *out, int cap) {
    if (!dag || !out) return CHAMELEON_ERR_ILLEGAL_VALUE;
    const int n = std::min<int>(cap, (int)dag->rec.size());
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < 5; ++j) out[5 * i + j] = dag->rec[i][j];
    return n;
}

// The recorded tasks as the executor's coarse DAG: every record's tiles (A's
// lower triangle, B's tile column bn) with read-after-write, write-after-read
// and write-after-write edges in submission order, then the same list
// scheduling as the built-in DAGs, and a replay of the device's wait
// predicates on the result.  Returns the sub-task list (empty + error code on
// a record the executor cannot run in that order).
static int dag_to_tasks(const cham_b200_dag_s &dag, int N, int NB, int nrhs, int NBB, int workers,
                        std::vector<chb::Task> *out, int *mode_out) {
    using namespace chb;
    const int NT = (N + NB - 1) / NB;
    const int NTB = nrhs > 0 ? (nrhs + NBB - 1) / NBB : 0;
    auto tm = [&](int m) { return (m == NT - 1) ? N - m * NB : NB; };
    auto nbi = [&](int m) { return (tm(m) + SUBB - 1) / SUBB; };
    int mode = 0;
    for (auto &r : dag.rec) mode |= (r[0] <= TK_UPD) ? MODE_FACT : MODE_SOLVE;
    std::vector<Coarse> ct;
    // tile ids: A (m, n) -> m + NT n; B (m, bn) -> NT NT + m + NT bn
    const size_t ntile = (size_t)NT * NT + (size_t)NT * std::max(NTB, 1);
    std::vector<int> last_w(ntile, -1);
    std::vector<std::vector<int>> readers(ntile);
    auto add = [&](int kind, int m, int n, int k, int bn, int nsub, double dur) {
        Coarse c;
        c.kind = kind; c.m = m; c.n = n; c.k = k; c.bn = bn; c.grp = 0; c.nsub = nsub; c.dur = dur;
        ct.push_back(c);
        return (int)ct.size() - 1;
    };
    auto edge = [&](int a, int b) {
        if (a < 0 || b < 0 || a == b) return;
        ct[a].succ.push_back(b);
        ct[b].npred++;
    };
    auto rd = [&](size_t tile, int id) {
        edge(last_w[tile], id);
        readers[tile].push_back(id);
    };
    auto wr = [&](size_t tile, int id) {
        edge(last_w[tile], id);
        for (int r : readers[tile]) edge(r, id);
        readers[tile].clear();
        last_w[tile] = id;
    };
    auto At = [&](int m, int n) { return (size_t)m + (size_t)NT * n; };
    auto Bt = [&](int m, int bn) { return (size_t)NT * NT + m + (size_t)NT * bn; };
    const double nb = NB;
    // FP64 path costs (flop model), as in build_order
    const Calib &cal = kCalib[PROF_FP64];
    std::vector<int> inv_id(NT, -1);
    if (!(mode & MODE_FACT)) {   // solve only: the executor inverts the diagonal blocks first
        for (int k = 0; k < NT; ++k) {
            inv_id[k] = add(TK_INV, k, k, k, 0, 1, 1.0 * tm(k) * IB * IB);
            rd(At(k, k), inv_id[k]);
        }
    }
    for (auto &r : dag.rec) {
        const int kind = r[0], m = r[1], n = r[2], k = r[3], bn = r[4];
        const bool inA = m < NT && n < NT && k < NT;
        const bool inB = bn < std::max(NTB, 1);
        if (!inA || !inB) return CHAMELEON_ERR_ILLEGAL_VALUE;
        int id = -1;
        const double w = NTB ? ((bn == NTB - 1) ? nrhs - bn * NBB : NBB) : 0;
        switch (kind) {
        case TK_POTRF:
            if (m != k || n != k) return CHAMELEON_ERR_ILLEGAL_VALUE;
            id = add(TK_POTRF, k, k, k, 0, 1, cal.potrf * 2.0 * tm(k) * tm(k) * tm(k));
            wr(At(k, k), id);
            break;
        case TK_TRSM:
            if (n != k || m <= k) return CHAMELEON_ERR_ILLEGAL_VALUE;
            id = add(TK_TRSM, m, k, k, 0, nbi(m), cal.trsm * 2.0 * SUBB * nb * nb);
            rd(At(k, k), id);
            wr(At(m, k), id);
            break;
        case TK_UPD:
            if (m < n || n <= k) return CHAMELEON_ERR_ILLEGAL_VALUE;
            id = add(TK_UPD, m, n, k, 1, m == n ? nbi(m) * (nbi(m) + 1) / 2 : nbi(m) * nbi(n),
                     cal.upd * SUBB * SUBB * nb * 2.0);
            ct[id].grp = k;
            rd(At(m, k), id);
            if (m != n) rd(At(n, k), id);
            wr(At(m, n), id);
            break;
        case TK_FWD_TRSM:
        case TK_BWD_TRSM:
            if (m != k || n != k || !NTB) return CHAMELEON_ERR_ILLEGAL_VALUE;
            id = add(kind, k, k, k, bn, 1, cal.strsm * 3.0 * tm(k) * tm(k) * w);
            rd(At(k, k), id);
            if (inv_id[k] >= 0) edge(inv_id[k], id);
            wr(Bt(k, bn), id);
            break;
        case TK_FWD_UPD:
        case TK_BWD_UPD:
            // forward: B(m) -= L(m,k) B(k), m > k; backward: B(m) -= L(k,m)^T B(k), m < k
            if (!NTB || (kind == TK_FWD_UPD ? m <= k : m >= k)) return CHAMELEON_ERR_ILLEGAL_VALUE;
            id = add(kind, m, k, k, bn, nbi(m), cal.supd * 2.0 * SUBB * tm(k) * w);
            rd(kind == TK_FWD_UPD ? At(m, k) : At(k, m), id);
            rd(Bt(k, bn), id);
            wr(Bt(m, bn), id);
            break;
        default:
            return CHAMELEON_ERR_ILLEGAL_VALUE;
        }
    }
    *out = list_schedule(ct, workers, nbi);
    *mode_out = mode;
    if (!replay_ok(*out, mode, N, NB, NTB)) {
        out->clear();
        return CHAMELEON_ERR_NOT_SUPPORTED;
    }
    return 0;
}

int CHAM_B200_Dag_Schedule(CHAM_b200_dag_t dag, int N, int NB, int nrhs, int NBB, int workers, void *out, int cap) {
    using namespace chb;
    if (!dag || N <= 0 || NB <= 0 || nrhs < 0 || (nrhs > 0 && NBB <= 0) || workers <= 0)
        return CHAMELEON_ERR_ILLEGAL_VALUE;
    std::vector<Task> tl;
    int mode = 0;
    if (int rc = dag_to_tasks(*dag, N, NB, nrhs, NBB, workers, &tl, &mode)) return rc;
    const int n = std::min<int>((int)tl.size(), cap);
    if (out) memcpy(out, tl.data(), sizeof(Task) * (size_t)std::max(0, n));
    return (int)tl.size();
}

int CHAM_B200_Dag_Run(CHAM_b200_dag_t dag, cham_uplo_t uplo, int N, int NB, double *A, const int64_t *a_off,
                      const int *a_ld, int nrhs, int NBB, double *B, const int64_t *b_off, const int *b_ld,
                      int *info) {
    using namespace chb;
    int rc = ensure_init();
    if (rc) return rc;
    if (!dag || !A || !a_off || !a_ld || N <= 0 || NB <= 0 || (uplo != ChamUpper && uplo != ChamLower) ||
        (nrhs > 0 && (!B || !b_off || !b_ld || NBB <= 0)))
        return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (info) *info = 0;
    if (dag->rec.empty()) return 0;
    Context &c = ctx();
    const int NT = (N + NB - 1) / NB, NTB = nrhs > 0 ? (nrhs + NBB - 1) / NBB : 0;
    auto sch = std::make_unique<Schedule>();
    int mode = 0;
    if ((rc = dag_to_tasks(*dag, N, NB, nrhs, NBB, c.num_sms, &sch->tasks, &mode))) return rc;
    if ((rc = upload_schedule(sch.get()))) return rc;
    CHAM_desc_t *dA = nullptr, *dB = nullptr;
    rc = desc_create_from_tables(&dA, A, NB, N, N, a_off, a_ld);
    if (!rc && NTB) rc = desc_create_from_tables(&dB, B, NB, N, nrhs, b_off, b_ld, NBB);
    ExecResult res;
    if (!rc) {
        t_given = sch.get();
        rc = run_cholesky_dag(mode, uplo, dA, dB, c.stream, &res, 0, nullptr, 0, 0, nullptr);
        t_given = nullptr;
    }
    if (dA) CHAMELEON_Desc_Destroy(&dA);
    if (dB) CHAMELEON_Desc_Destroy(&dB);
    dev_free(sch->d_tasks);
    if (rc) return rc;
    if (res.error) return res.error;
    if (info) *info = res.info;
    (void)NT;
    return 0;
}

}  // extern "C"
