// orc_common.hpp -- shared helpers of the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY.  The oracle is a plain C++ restatement of the
// XCALibre.jl CPU path for the finite-volume hot path.  Only tests/, the
// smoke check and the bench's CPU-baseline leg may load it; the library
// never links or calls it.
//
// Arithmetic rules (these define what "the reference's algorithm" means here):
//  * every floating-point operation is an individual IEEE-754 double op in the
//    order the Julia source writes it (Julia never contracts a*b+c into an
//    FMA), so this file is compiled with -ffp-contract=off;
//  * reductions whose order Julia leaves to a library (BLAS dot/nrm2, `sum`)
//    use the fixed blocked tree below, which the device kernels reproduce;
//  * per-row sums (SpMV, row walks) run sequentially in CSR order as in
//    src/Multithread/spmvm.jl:44-57.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>
#include <algorithm>
#include <limits>

namespace orc {

struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
// StaticArrays dot: ((a1*b1 + a2*b2) + a3*b3)
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// norm(SVector) = sqrt((x^2 + y^2) + z^2)
inline double norm(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
inline double comp(V3 a, int c) { return c == 0 ? a.x : (c == 1 ? a.y : a.z); }

// Julia's eps(x): spacing of floats at |x|
inline double jl_eps(double x) {
    x = std::fabs(x);
    return std::nextafter(x, std::numeric_limits<double>::infinity()) - x;
}
// Julia's max/min for floats (NaN propagating, -0.0 < 0.0)
inline double jl_max(double x, double y) {
    bool take_y = (y > x) || (std::signbit(y) < std::signbit(x));
    return take_y ? (std::isnan(x) ? x : y) : (std::isnan(y) ? y : x);
}
inline double jl_min(double x, double y) {
    bool take_y = (y < x) || (std::signbit(y) > std::signbit(x));
    return take_y ? (std::isnan(x) ? x : y) : (std::isnan(y) ? y : x);
}
inline double jl_clamp(double x, double lo, double hi) {
    return x > hi ? hi : (x < lo ? lo : x);
}

// ---- canonical blocked reduction -----------------------------------------
// The device reduces per-row contributions v[0..n) in tiles of
// RED_THREADS*RED_ITEMS rows.  Thread t of a tile accumulates rows
// tile*TILE + k*RED_THREADS + t (k = 0..RED_ITEMS-1) sequentially from 0.0,
// each warp combines its 32 lanes with an xor butterfly (16,8,4,2,1), and the
// 8 warp sums are combined by a second butterfly (4,2,1).  The tile partials
// are reduced by one tile-shaped pass with the same structure.
constexpr int RED_THREADS = 256;
constexpr int RED_ITEMS = 8;
constexpr int64_t RED_TILE = (int64_t)RED_THREADS * RED_ITEMS;

inline double block_tree(double* a /* [RED_THREADS] */) {
    double warp_sum[RED_THREADS / 32];
    for (int w = 0; w < RED_THREADS / 32; ++w) {
        double l[32];
        for (int i = 0; i < 32; ++i) l[i] = a[w * 32 + i];
        for (int off = 16; off >= 1; off >>= 1) {
            double nl[32];
            for (int i = 0; i < 32; ++i) nl[i] = l[i] + l[i ^ off];
            for (int i = 0; i < 32; ++i) l[i] = nl[i];
        }
        warp_sum[w] = l[0];
    }
    constexpr int NW = RED_THREADS / 32;
    double l[NW];
    for (int i = 0; i < NW; ++i) l[i] = warp_sum[i];
    for (int off = NW / 2; off >= 1; off >>= 1) {
        double nl[NW];
        for (int i = 0; i < NW; ++i) nl[i] = l[i] + l[i ^ off];
        for (int i = 0; i < NW; ++i) l[i] = nl[i];
    }
    return l[0];
}

template <class F>
inline double tile_partial(int64_t n, int64_t tile, F f) {
    double acc[RED_THREADS];
    for (int t = 0; t < RED_THREADS; ++t) {
        double s = 0.0;
        for (int k = 0; k < RED_ITEMS; ++k) {
            int64_t r = tile * RED_TILE + (int64_t)k * RED_THREADS + t;
            if (r < n) s = s + f(r);
        }
        acc[t] = s;
    }
    return block_tree(acc);
}

// Final pass over the tile partials: thread t sums partials t, t+256, ...
inline double reduce_partials(const std::vector<double>& part) {
    double acc[RED_THREADS];
    int64_t T = (int64_t)part.size();
    for (int t = 0; t < RED_THREADS; ++t) {
        double s = 0.0;
        for (int64_t idx = t; idx < T; idx += RED_THREADS) s = s + part[idx];
        acc[t] = s;
    }
    return block_tree(acc);
}

// Row order of the canonical reductions over cells: ascending 63-bit Morton
// key of the cell centre quantised to 21 bits per axis over the centres'
// bounding box, ties by index (order[s] = cell at position s).  This is a
// fixed summation order for the reference's `dot`/`sum`, whose own order is
// left to BLAS; the device stores cells in this order.
inline std::vector<int> morton_order(const std::vector<V3>& c) {
    int n = (int)c.size();
    double lo[3] = {c[0].x, c[0].y, c[0].z}, hi[3] = {c[0].x, c[0].y, c[0].z};
    for (int i = 1; i < n; ++i) {
        double v[3] = {c[i].x, c[i].y, c[i].z};
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], v[d]);
            hi[d] = std::max(hi[d], v[d]);
        }
    }
    auto bits = [](uint64_t q) {
        uint64_t r = 0;
        for (int b = 0; b < 21; ++b) r |= ((q >> b) & 1ULL) << (3 * b);
        return r;
    };
    std::vector<uint64_t> key(n);
    for (int i = 0; i < n; ++i) {
        double v[3] = {c[i].x, c[i].y, c[i].z};
        uint64_t q[3];
        for (int d = 0; d < 3; ++d) {
            double span = hi[d] - lo[d];
            double u = span > 0.0 ? (v[d] - lo[d]) / span : 0.0;
            double t = u * 2097151.0;
            uint64_t qq = t > 0.0 ? (uint64_t)t : 0;
            q[d] = qq > 2097151ULL ? 2097151ULL : qq;
        }
        key[i] = bits(q[0]) | (bits(q[1]) << 1) | (bits(q[2]) << 2);
    }
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return key[a] != key[b] ? key[a] < key[b] : a < b; });
    return order;
}

template <class F>
inline double creduce(int64_t n, F f) {
    int64_t T = (n + RED_TILE - 1) / RED_TILE;
    if (T == 0) T = 1;
    std::vector<double> part(T);
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < T; ++t) part[t] = tile_partial(n, t, f);
    return reduce_partials(part);
}


// exp(y) for y <= 0 and tanh(x) for x >= 0 from +, *, / and ldexp only, so
// the device restatement gives the same bits: Cody-Waite reduction
// y = k ln2 + r (ln2 split in a 12-bit head and its remainder), exp(r) by its
// Taylor series to r^14 / 14!; tanh(x) = (1 - e^-2x) / (1 + e^-2x), 1 past 20
inline double det_exp_neg(double y) {
    if (y < -745.0) return 0.0;
    const double LN2_HEAD = 0.693145751953125, LN2_TAIL = 1.4286068203094172321e-06;
    const double k = std::rint(y * 1.4426950408889634);
    const double r = (y - k * LN2_HEAD) - k * LN2_TAIL;
    double p = 1.0;
    for (int n = 14; n >= 1; --n) p = 1.0 + (r / (double)n) * p;
    return std::ldexp(p, (int)k);
}
// log(x) for x > 0 from frexp (exact) and +, *, /: x = 2^e m with
// m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s), s = (m - 1) / (m + 1), by
// its series to s^29
inline double det_log(double x) {
    int e = 0;
    double m = std::frexp(x, &e);  // m in [0.5, 1)
    if (m < 0.70710678118654752) {
        m = 2.0 * m;
        e -= 1;
    }
    const double s = (m - 1.0) / (m + 1.0), s2 = s * s;
    double t = 0.0;
    for (int n = 29; n >= 3; n -= 2) t = (t + 1.0 / (double)n) * s2;
    return (double)e * 0.6931471805599453 + 2.0 * (s + s * t);
}
inline double det_tanh_pos(double x) {
    if (x > 20.0) return 1.0;
    const double e = det_exp_neg(-2.0 * x);
    return (1.0 - e) / (1.0 + e);
}
// x^a for x >= 0 as exp(a log x) (Julia's ^ for a non-integer exponent):
// 0^a = Inf for a < 0, Inf^a = 0; the exp reduction also holds for y > 0,
// up to the overflow at 709.7
inline double det_pow(double x, double a) {
    if (x == 0.0) return a < 0.0 ? HUGE_VAL : 0.0;
    if (std::isinf(x)) return a < 0.0 ? 0.0 : HUGE_VAL;
    const double y = a * det_log(x);
    return y >= 709.7 ? HUGE_VAL : det_exp_neg(y);
}

}  // namespace orc
