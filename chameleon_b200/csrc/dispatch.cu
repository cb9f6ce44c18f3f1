// dispatch.cu -- host planning of independent SPD systems over several GPUs.
//
// Batches of systems and serving requests are independent units: spreading
// them over the GPUs of a node needs no collective, only a host dispatcher
// that decides which GPU solves which system (each GPU then runs the batched
// or the mixed-precision path on its share, and the results come back to the
// host).  The reference distributes one matrix's tiles over a P x Q grid
// (control/descriptor_helpers.c:51-56) for a single large solve; this is the
// other split, the one that needs no exchange.
//
// The plan is longest-processing-time-first list scheduling: systems sorted
// by estimated device time (largest first), each one placed on the live GPU
// whose estimated finish time is earliest among those whose free HBM still
// admits it.  A system pinned to a GPU (a serving request that reuses a factor
// kept there) goes to that GPU if it is alive.  When no GPU can admit a
// system next to what the current wave already holds, a new wave starts with
// every GPU's memory free again; the caller runs the waves one after another.
// Host code only.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "chameleon_b200.h"

namespace {

// Seconds a B200 needs for one system inside a batch or a serving wave: a
// launch-and-latency term plus the flops at the throughput of the path the
// library takes for that order (batched FP64 for small orders, the mixed
// BF16x3 solver with FP64 refinement for large ones).  Only ratios matter for
// balance; the figures are the library's measured throughputs, rounded.
double est_seconds(int n, int nrhs) {
    const double N = n, R = std::max(nrhs, 0);
    const double flops = N * N * N / 3.0 + 2.0 * N * N * R;
    double rate;
    if (n <= 512) rate = 3.0e12;
    else if (n <= 2048) rate = 12.0e12;
    else if (n <= 8192) rate = 40.0e12;
    else rate = 90.0e12;
    const double fixed = n <= 512 ? 2e-6 : 1.5e-3;
    return fixed + flops / rate;
}

// Device bytes one system holds while it is solved: the FP64 matrix and
// right-hand sides, the solution, and for orders above the batched range the
// mixed solver's FP32 copy, BF16 split panels and refinement vectors.
double est_bytes(int n, int nrhs) {
    const double N = n, R = std::max(nrhs, 0);
    const double fp64 = 8.0 * (N * N + 2.0 * N * R);
    return n <= 512 ? fp64 : fp64 + 8.0 * N * N + 24.0 * N * R;
}

}  // namespace

extern "C" {

double CHAM_B200_Dispatch_Cost(int n, int nrhs) { return n < 0 ? 0.0 : est_seconds(n, nrhs); }
double CHAM_B200_Dispatch_Bytes(int n, int nrhs) { return n < 0 ? 0.0 : est_bytes(n, nrhs); }

int CHAM_B200_Dispatch_Plan(int count, const int *n, const int *nrhs, const int *pin, int nranks, const int *alive,
                            const double *free_bytes, const double *load_s, int *owner, int *wave) {
    if (count < 0 || nranks <= 0 || (count > 0 && (!n || !nrhs || !owner)) || !alive || !free_bytes)
        return CHAMELEON_ERR_ILLEGAL_VALUE;
    std::vector<int> live;
    for (int r = 0; r < nranks; ++r)
        if (alive[r]) live.push_back(r);
    if (live.empty()) return CHAMELEON_ERR_NOT_INITIALIZED;
    for (int i = 0; i < count; ++i)
        if (n[i] < 0 || nrhs[i] < 0) return CHAMELEON_ERR_ILLEGAL_VALUE;

    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::vector<double> cost(count);
    for (int i = 0; i < count; ++i) cost[i] = est_seconds(n[i], nrhs[i]);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });

    std::vector<double> finish(nranks, 0.0), used(nranks, 0.0);
    for (int r = 0; r < nranks; ++r) finish[r] = load_s ? load_s[r] : 0.0;
    int cur_wave = 0;
    for (int i : order) {
        const double b = est_bytes(n[i], nrhs[i]);
        int best = -1;
        const int p = pin ? pin[i] : -1;
        if (p >= 0 && p < nranks && alive[p]) {
            if (b > free_bytes[p]) return CHAMELEON_ERR_OUT_OF_RESOURCES;
            if (used[p] + b > free_bytes[p]) {   // the pinned GPU is full in this wave
                ++cur_wave;
                std::fill(used.begin(), used.end(), 0.0);
            }
            best = p;
        } else {
            for (int pass = 0; pass < 2 && best < 0; ++pass) {
                for (int r : live)
                    if (used[r] + b <= free_bytes[r] && (best < 0 || finish[r] < finish[best])) best = r;
                if (best < 0) {
                    bool fits_alone = false;
                    for (int r : live) fits_alone |= b <= free_bytes[r];
                    if (!fits_alone) return CHAMELEON_ERR_OUT_OF_RESOURCES;
                    ++cur_wave;
                    std::fill(used.begin(), used.end(), 0.0);
                }
            }
        }
        owner[i] = best;
        if (wave) wave[i] = cur_wave;
        used[best] += b;
        finish[best] += cost[i];
    }
    return cur_wave + 1;
}

}  // extern "C"
