// sw2_shares.h -- CTA shares of a batched Krylov launch (host code, no CUDA).
//
// A batched Krylov launch lasts as long as its instance with the most work per CTA, so the
// shares minimise that maximum: every instance starts with one CTA, and each further CTA goes to
// the instance whose predicted work per CTA is then the largest (ties to the lower index), up to
// its virtual grid.  (Proportional shares rounded down left instances that should have 1.7 CTAs
// with one.)  The shares set only the speed: the results of an instance depend on its virtual
// grid alone.
#pragma once
#include <algorithm>
#include <queue>
#include <utility>
#include <vector>

namespace sw2 {

// Predicted work of an instance's solve: its blocks x its predicted iterations.  A resumed solve
// (`done` iterations behind it) is predicted to need the rest of its prediction, or half as many
// again as it has done once it is past the prediction.
inline double krylov_work(long long nnzb, int pred_its, int done) {
    const int pred = std::max(pred_its, 1);
    return (double)nnzb * (double)(done ? std::max(pred - done, (done + 1) / 2) : pred);
}

// The min-max integer allocation of `capacity` CTAs over instances of predicted work W[j] and
// virtual grid vgrid[j] (an instance never gets more CTAs than virtual ones, and at least one).
inline std::vector<int> krylov_shares_minmax(const std::vector<double>& W, const std::vector<int>& vgrid,
                                             int capacity) {
    const int n = (int)W.size();
    std::vector<int> P(n, 1);
    std::priority_queue<std::pair<double, int>> pq;   // (work per CTA, -j)
    for (int j = 0; j < n; j++)
        if (vgrid[j] > 1) pq.push({W[j], -j});
    for (int left = capacity - n; left > 0 && !pq.empty(); left--) {
        const int j = -pq.top().second;
        pq.pop();
        if (++P[j] < vgrid[j]) pq.push({W[j] / P[j], -j});
    }
    return P;
}

}  // namespace sw2
