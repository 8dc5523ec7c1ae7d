// Test infrastructure (oracle): sequential executor.
#pragma once

#include "par/for_each.h"

namespace par {

struct SequentialExecutor {
    template <typename T, typename F>
    void run_1d(T b, T e, const F& f) const { for (T i = b; i < e; ++i) f(i); }
    template <typename T, typename F>
    void run_2d(T x0, T x1, T y0, T y1, const F& f) const {
        for (T y = y0; y < y1; ++y) for (T x = x0; x < x1; ++x) f(x, y);
    }
    template <typename T, typename V, typename R, typename M>
    V run_reduce(T b, T e, V acc, const R& reduce, const M& map) const {
        for (T i = b; i < e; ++i) acc = reduce(acc, map(i));
        return acc;
    }
};

} // namespace par
