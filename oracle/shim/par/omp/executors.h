// Test infrastructure (oracle): OpenMP executors (static and dynamic schedules).
// The 2D range is split into rows; results per index do not depend on the
// schedule, only the order in which pixels are visited does.
#pragma once

#include <algorithm>
#include <omp.h>

#include "par/for_each.h"

namespace par::omp {

template <bool Dynamic>
struct Executor {
    template <typename T, typename F>
    void run_1d(T b, T e, const F& f) const {
        if constexpr (Dynamic) {
            #pragma omp parallel for schedule(dynamic, 64)
            for (long i = (long)b; i < (long)e; ++i) f((T)i);
        } else {
            #pragma omp parallel for schedule(static)
            for (long i = (long)b; i < (long)e; ++i) f((T)i);
        }
    }
    template <typename T, typename F>
    void run_2d(T x0, T x1, T y0, T y1, const F& f) const {
        const long w = (long)(x1 - x0), h = (long)(y1 - y0);
        if constexpr (Dynamic) {
            #pragma omp parallel for schedule(dynamic, 1) collapse(2)
            for (long ty = 0; ty < (h + 7) / 8; ++ty)
                for (long tx = 0; tx < (w + 7) / 8; ++tx)
                    for (long y = ty * 8; y < std::min(h, ty * 8 + 8); ++y)
                        for (long x = tx * 8; x < std::min(w, tx * 8 + 8); ++x) f(x0 + (T)x, y0 + (T)y);
        } else {
            #pragma omp parallel for schedule(static)
            for (long y = 0; y < h; ++y)
                for (long x = 0; x < w; ++x) f(x0 + (T)x, y0 + (T)y);
        }
    }
    template <typename T, typename V, typename R, typename M>
    V run_reduce(T b, T e, V init, const R& reduce, const M& map) const {
        V acc = init;
        #pragma omp parallel
        {
            V local = init;
            #pragma omp for schedule(static) nowait
            for (long i = (long)b; i < (long)e; ++i) local = reduce(local, map((T)i));
            #pragma omp critical(par_reduce)
            acc = reduce(acc, local);
        }
        return acc;
    }
};

using StaticExecutor = Executor<false>;
using DynamicExecutor = Executor<true>;

} // namespace par::omp
