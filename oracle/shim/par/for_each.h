// Test infrastructure (oracle): clean-room stand-in for the part of par
// (madmann91/par) that SoL uses: 1D/2D index ranges, for_each and
// transform_reduce over a sequential or OpenMP executor.
#pragma once

#include <cstddef>
#include <utility>

namespace par {

template <typename T> struct Range1 { T begin, end; };
template <typename T> struct Range2 { T x0, x1, y0, y1; };

template <typename T> Range1<T> range_1d(T b, T e) { return {b, e}; }
template <typename T> Range2<T> range_2d(T x0, T x1, T y0, T y1) { return {x0, x1, y0, y1}; }

template <typename Executor, typename T, typename F>
void for_each(const Executor& ex, const Range1<T>& r, const F& f) { ex.run_1d(r.begin, r.end, f); }

template <typename Executor, typename T, typename F>
void for_each(const Executor& ex, const Range2<T>& r, const F& f) { ex.run_2d(r.x0, r.x1, r.y0, r.y1, f); }

template <typename Executor, typename T, typename V, typename R, typename M>
V transform_reduce(const Executor& ex, const Range1<T>& r, V init, const R& reduce, const M& map) {
    return ex.run_reduce(r.begin, r.end, std::move(init), reduce, map);
}

} // namespace par
