// Host-side factorisation of an FFT axis into the radices of the line engine.
#pragma once

#include <vector>

#include "fft_engine.cuh"

namespace chfsi {

// Radices with a register codelet (fft_engine.cuh).
constexpr int kRadices[] = {15, 12, 10, 9, 8, 6, 5, 4, 3, 2};

namespace detail {
inline void search(int n, int rem, std::vector<int>& cur, std::vector<int>& best, int& best_tpl) {
    if (rem == 1) {
        int tpl = 0;
        for (int r : cur) tpl = tpl > n / r ? tpl : n / r;
        const bool better = best.empty() || cur.size() < best.size() ||
                            (cur.size() == best.size() && tpl < best_tpl);
        if (better) {
            best = cur;
            best_tpl = tpl;
        }
        return;
    }
    if ((int)cur.size() >= kMaxStages || (!best.empty() && cur.size() >= best.size())) return;
    for (int r : kRadices) {
        if (rem % r) continue;
        cur.push_back(r);
        search(n, rem / r, cur, best, best_tpl);
        cur.pop_back();
    }
}
}  // namespace detail

// Fewest stages first, then the fewest threads per line (one lane group of
// a warp per line when <= 32; larger plans run their stages CTA-wide).
// Returns false if n is not a product of the radices.
inline bool plan_axis(int n, AxisPlan& P) {
    P = AxisPlan{};
    P.n = n;
    if (n < 1) return false;
    if (n == 1) {
        P.nst = 0;
        P.tpl = 1;
        return true;
    }
    std::vector<int> cur, best;
    int best_tpl = 1 << 30;
    detail::search(n, n, cur, best, best_tpl);
    if (best.empty()) return false;
    P.nst = (int)best.size();
    for (int t = 0; t < P.nst; ++t) P.r[t] = best[t];
    P.tpl = best_tpl;
    return true;
}

}  // namespace chfsi
