// Host interaction plan (modules/bem/galerkin/interaction_plan.cpp:228-504,
// pair_quadrature.cpp:143-575): every unordered disjoint pair that is
// geometrically near, or that no qualified regular Dunavant rule covers at
// the planning wavenumber, gets an adaptive patch list from the
// largest-error refinement driven by embedded degree 6/8 (12/14) estimates.
// Candidate pairs come from a uniform grid over panel vertex 0 with cell
// width (ratio+2)*h_max; pairs are refined concurrently on host threads and
// flattened in (first, second) order, so the plan is independent of thread
// count and identical to the reference's.
#include "planner.hpp"
#include "planner_geom.cuh"

#include <algorithm>
#include <array>
#include <atomic>
#include <complex>
#include <exception>
#include <limits>
#include <mutex>
#include <sstream>
#include <thread>
#include <unordered_map>

namespace hsb {
namespace {

using cplx = std::complex<double>;
using Moments = std::array<cplx, 36>;
using Bary = std::array<double, 3>;

FanPanel fan(const HostPanel &p) { return FanPanel{{p.v[0], p.v[1], p.v[2]}, p.n, p.area}; }

// ---- embedded-rule patch estimate (pair_quadrature.cpp:143-226, 644-683) ----
std::array<cplx, 4> pointKernels(V3 d, double k, double scale) {
    const double r = std::sqrt(norm2(d));
    if (!(r > 0))
        throw InvalidArgument("Disjoint quadrature panels intersect or contain duplicate geometric nodes.");
    double sn, cs;  // exp(-i k r) = cos + i sin of the same argument
    ::sincos(-k * r, &sn, &cs);
    const cplx g = cplx(cs, sn) / r;
    // -g (1 + i k r), written out: the same products and sums as the complex
    // product, without the library's NaN-recovery call per point
    const double kr = k * r;
    const cplx der = cplx(-g.real() + g.imag() * kr, -g.real() * kr - g.imag()) * (scale / (r * r));
    return {g, der * d.x, der * d.y, der * d.z};
}

struct Rules {
    std::vector<TriPoint> r6, r8, r12, r14;
    std::vector<GaussPoint> g14, g20;
};
const Rules &rules() {
    static const Rules r{triangleRule(6), triangleRule(8), triangleRule(12), triangleRule(14), gaussLegendre01(14),
                         gaussLegendre01(20)};
    return r;
}

Moments tensorMoments(const HostPanel &t, const HostPanel &s, const Sub &a, const Sub &b,
                      const std::vector<TriPoint> &rule, double k, double scale) {
    Moments m{};
    const V3 origin = t.v[0] - s.v[0];
    // trial barycentrics and points, the same for every test point
    constexpr size_t kMaxRule = 64;
    if (rule.size() > kMaxRule)
        throw std::logic_error("pair rule larger than the planner's point table");
    double bsAll[kMaxRule][3];
    V3 lsAll[kMaxRule];
    for (size_t q = 0; q < rule.size(); ++q) {
        double *bs = bsAll[q];
        bs[0] = bs[1] = bs[2] = 0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                bs[i] += rule[q].b[j] * b.v[j][i];
        lsAll[q] = localPoint(s, bs);
    }
    for (const auto &x : rule) {
        double bt[3] = {0, 0, 0};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                bt[i] += x.b[j] * a.v[j][i];
        const V3 lt = localPoint(t, bt);
        for (size_t q = 0; q < rule.size(); ++q) {
            const auto &y = rule[q];
            const double *bs = bsAll[q];
            const double w = x.w * y.w * a.fraction * b.fraction;
            const auto ker = pointKernels(origin + (lt - lsAll[q]), k, scale);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    const double ww = w * bt[i] * bs[j];
                    for (int c = 0; c < 4; ++c)
                        m[c * 9 + i * 3 + j] += ker[c] * ww;
                }
        }
    }
    return m;
}

Moments projectionMoments(const HostPanel &t, const HostPanel &s, const Sub &a, const std::vector<TriPoint> &outer,
                          const std::vector<GaussPoint> &base, unsigned intervals, double k, double scale) {
    Patch patch{};
    patch.projection = 1;
    patch.areaFraction = a.fraction;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            patch.test[3 * i + j] = a.v[i][j];
    std::vector<GaussPoint> g;
    g.reserve(base.size() * intervals);
    for (unsigned iv = 0; iv < intervals; ++iv)
        for (const auto &p : base)
            g.push_back({(iv + p.x) / intervals, p.w / intervals});
    const FanPanel ft = fan(t), fs = fan(s);
    const V3 offset = t.v[0] - s.v[0];
    Moments m{};
    for (const auto &x : outer) {
        const ProjOuter po = projOuter(x.b, x.w, patch, ft, fs);
        const V3 lt = localPoint(t, po.test);
        std::array<cplx, 12> inner{};
        for (unsigned e = 0; e < 3; ++e) {
            const ProjEdge pe = projEdge(po, e, fs);
            for (const auto &u : g) {
                const ProjRay ray = projRay(po, pe, u);
                for (const auto &v : g) {
                    const PairPoint p = projPoint(po, ray, v);
                    const auto ker = pointKernels(offset + (lt - localPoint(s, p.s)), k, scale);
                    for (int j = 0; j < 3; ++j) {
                        const double w = p.w * p.s[j];
                        for (int c = 0; c < 4; ++c)
                            inner[3 * c + j] += ker[c] * w;
                    }
                }
            }
        }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int c = 0; c < 4; ++c)
                    m[9 * c + 3 * i + j] += po.test[i] * inner[3 * c + j];
    }
    return m;
}

double maxNorm(const Moments &m) {
    double r = 0;
    for (const auto &v : m) {
        const double a = std::abs(v);
        if (!std::isfinite(a))
            throw NumericError("Near-pair quadrature produced a non-finite moment.");
        r = std::max(r, a);
    }
    return r;
}

struct Estimate {
    Moments integral{};
    double error{}, inner{}, outer{};
};
Estimate estimate(const HostPanel &t, const HostPanel &s, const Sub &a, const Sub &b, unsigned degree,
                  bool projection, unsigned intervals, double k) {
    const Rules &R = rules();
    const double scale = std::max(t.maxEdge, s.maxEdge);
    const auto &lo = degree == 8 ? R.r6 : R.r12;
    const auto &hi = degree == 8 ? R.r8 : R.r14;
    Estimate e;
    const Moments low = projection ? projectionMoments(t, s, a, lo, R.g20, intervals, k, scale)
                                   : tensorMoments(t, s, a, b, lo, k, scale);
    e.integral = projection ? projectionMoments(t, s, a, hi, R.g20, intervals, k, scale)
                            : tensorMoments(t, s, a, b, hi, k, scale);
    Moments d;
    for (int i = 0; i < 36; ++i)
        d[i] = e.integral[i] - low[i];
    (void)maxNorm(e.integral);
    e.outer = maxNorm(d);
    if (projection) {
        const Moments il = projectionMoments(t, s, a, hi, R.g14, intervals, k, scale);
        for (int i = 0; i < 36; ++i)
            d[i] = e.integral[i] - il[i];
        e.inner = maxNorm(d);
    }
    e.error = e.outer + e.inner;
    return e;
}

// ---- projected partition (pair_quadrature.cpp:231-317) ----
std::vector<Sub> projectionPartition(const HostPanel &t, const HostPanel &s) {
    Bary proj[3];
    for (int i = 0; i < 3; ++i) {
        const V3 rel = t.v[i] - s.v[0];
        proj[i][1] = dot(rel, s.grad[1]);
        proj[i][2] = dot(rel, s.grad[2]);
        proj[i][0] = 1 - proj[i][1] - proj[i][2];
    }
    using Poly = std::vector<Bary>;
    std::vector<Poly> polys{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}};
    for (int e = 0; e < 3; ++e) {
        const auto value = [&](const Bary &p) { return p[0] * proj[0][e] + p[1] * proj[1][e] + p[2] * proj[2][e]; };
        std::vector<Poly> next;
        for (const auto &poly : polys) {
            bool pos = false, neg = false;
            for (const auto &p : poly) {
                pos |= value(p) > 0;
                neg |= value(p) < 0;
            }
            if (!(pos && neg)) {
                next.push_back(poly);
                continue;
            }
            Poly plus, minus;
            for (size_t i = 0; i < poly.size(); ++i) {
                const Bary a = poly[i], b = poly[(i + 1) % poly.size()];
                const double va = value(a), vb = value(b);
                if (va >= 0)
                    plus.push_back(a);
                if (va <= 0)
                    minus.push_back(a);
                if ((va < 0 && vb > 0) || (va > 0 && vb < 0)) {
                    const double f = va / (va - vb);
                    Bary x;
                    for (int j = 0; j < 3; ++j)
                        x[j] = a[j] + f * (b[j] - a[j]);
                    plus.push_back(x);
                    minus.push_back(x);
                }
            }
            if (plus.size() >= 3)
                next.push_back(std::move(plus));
            if (minus.size() >= 3)
                next.push_back(std::move(minus));
        }
        polys = std::move(next);
    }
    std::vector<Sub> out;
    double area = 0;
    for (const auto &poly : polys)
        for (size_t i = 1; i + 1 < poly.size(); ++i) {
            const Bary a = poly[0], b = poly[i], c = poly[i + 1];
            const double f = std::abs((b[1] - a[1]) * (c[2] - a[2]) - (b[2] - a[2]) * (c[1] - a[1]));
            if (f > 0) {
                Sub sub{};
                for (int i = 0; i < 3; ++i) {
                    sub.v[0][i] = a[i];
                    sub.v[1][i] = b[i];
                    sub.v[2][i] = c[i];
                }
                sub.fraction = f;
                out.push_back(sub);
                area += f;
            }
        }
    if (std::abs(area - 1) > 1024 * std::numeric_limits<double>::epsilon())
        throw NumericError("Projected near-pair partition lost reference area.");
    if (out.size() > 16)
        throw NumericError("Projected line partition exceeds its triangle bound.");
    return out;
}
// Largest-error refinement for one disjoint pair (pair_quadrature.cpp:329-575).
PairRule adaptivePair(const HostPanel &t, const HostPanel &s, const PlanSettings &st, double k,
                      const volatile int32_t *cancel) {
    struct Leaf {
        Sub a, b;
        Moments integral{};
        double error{}, da{}, db{}, inner{}, outer{};
        unsigned depth{}, degree{8}, intervals{1};
    };
    const auto byError = [](const Leaf &x, const Leaf &y) { return x.error < y.error; };
    const bool projection = useProjection(t, s, std::max(t.maxEdge, s.maxEdge));
    const bool promoteRoot = !projection && !isNearPair(t, s, 1.0);
    const std::vector<Sub> initial = projection ? projectionPartition(t, s) : std::vector<Sub>{wholeSub()};
    const auto makeLeaf = [&](const Sub &a, const Sub &b, unsigned depth, unsigned degree, unsigned intervals) {
        Leaf l;
        l.a = a;
        l.b = b;
        l.da = subDiameter(t, a, t.v[0]);
        l.db = subDiameter(s, b, t.v[0]);
        l.depth = depth;
        l.degree = degree;
        l.intervals = intervals;
        return l;
    };
    const auto patchOf = [&](const Leaf &l) {
        Patch p{};
        p.degree = l.degree;
        p.projection = projection ? 1 : 0;
        p.intervals = l.intervals;
        p.areaFraction = l.a.fraction * l.b.fraction;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                p.test[3 * i + j] = l.a.v[i][j];
                p.trial[3 * i + j] = l.b.v[i][j];
            }
        return p;
    };
    std::vector<Leaf> pending, atLimit, requested;
    Moments integral{};
    double absError = 0;
    size_t nextInitial = 0;
    const auto requestInitial = [&]() {
        while (nextInitial < initial.size() && requested.size() < 4)
            requested.push_back(makeLeaf(initial[nextInitial++], wholeSub(), 0, 8, 1));
    };
    requestInitial();
    for (;;) {
        if (cancel && *cancel)
            throw Cancelled();
        for (auto &l : requested) {
            Sub a = l.a;
            const Estimate e = estimate(t, s, a, l.b, l.degree, projection, l.intervals, k);
            if (!std::isfinite(e.error) || !(e.error >= 0))
                throw NumericError("Near-pair quadrature produced a non-finite error estimate.");
            l.integral = e.integral;
            l.error = e.error;
            l.inner = e.inner;
            l.outer = e.outer;
        }
        for (auto &l : requested) {
            absError += l.error;
            for (int i = 0; i < 36; ++i)
                integral[i] += l.integral[i];
            const bool outerLimit = l.depth == st.maxDepth && l.degree == 14;
            const unsigned nextInner = l.intervals * 2;
            const bool innerLimit = nextInner > (1u << st.maxDepth) ||
                                    uint64_t(192) * 400 * nextInner * nextInner > std::numeric_limits<unsigned>::max();
            if ((!projection && outerLimit) || (projection && (l.inner > l.outer ? innerLimit : outerLimit)))
                atLimit.push_back(l);
            else {
                pending.push_back(l);
                std::push_heap(pending.begin(), pending.end(), byError);
            }
        }
        requested.clear();
        if (nextInitial < initial.size()) {
            requestInitial();
            continue;
        }
        if (absError <= st.tol * .2 * maxNorm(integral)) {
            PairRule out;
            for (const auto &l : atLimit) {
                out.maxDepth = std::max(out.maxDepth, l.depth);
                out.patches.push_back(patchOf(l));
            }
            while (!pending.empty()) {
                out.maxDepth = std::max(out.maxDepth, pending.front().depth);
                out.patches.push_back(patchOf(pending.front()));
                std::pop_heap(pending.begin(), pending.end(), byError);
                pending.pop_back();
            }
            const double ref = maxNorm(integral);
            if (!(ref > 0))
                throw NumericError("Near-pair quadrature has no finite nonzero reference scale.");
            out.relError = absError / ref;
            if (!std::isfinite(out.relError) || out.relError > st.tol)
                throw NumericError("Near-pair quadrature global error estimate exceeds the requested tolerance.");
            return out;
        }
        if (pending.empty())
            throw NumericError("Near-pair quadrature did not attain the requested error tolerance before the "
                               "subdivision limit.");
        const Leaf v = pending.front();
        std::pop_heap(pending.begin(), pending.end(), byError);
        pending.pop_back();
        absError = std::max(0.0, absError - v.error);
        for (int i = 0; i < 36; ++i)
            integral[i] -= v.integral[i];
        if (projection && v.inner > v.outer)
            requested.push_back(makeLeaf(v.a, v.b, v.depth, v.degree, v.intervals * 2));
        else if (v.degree == 8 && (v.depth == st.maxDepth || (promoteRoot && v.depth == 0)))
            requested.push_back(makeLeaf(v.a, v.b, v.depth, 14, v.intervals));
        else {
            if (pending.size() + atLimit.size() + 4 > 50000)
                throw NumericError("Near-pair quadrature exceeds the fifty-thousand-patch safety limit.");
            Sub children[4];
            if (projection || v.da >= v.db) {
                quarter(v.a, children);
                for (const auto &c : children)
                    requested.push_back(makeLeaf(c, v.b, v.depth + 1, 8, v.intervals));
            } else {
                quarter(v.b, children);
                for (const auto &c : children)
                    requested.push_back(makeLeaf(v.a, c, v.depth + 1, 8, 1));
            }
        }
    }
}

// Uniform-grid candidates over vertex 0 (interaction_plan.cpp:129-220).
std::vector<std::pair<uint32_t, uint32_t>> candidates(const Space &sp, double ratio) {
    double maxEdge = 0;
    for (const auto &p : sp.panels)
        maxEdge = std::max(maxEdge, p.maxEdge);
    const V3 origin = sp.panels.front().v[0];
    double extent = 0;
    for (const auto &p : sp.panels)
        extent = std::max({extent, std::abs(p.v[0].x - origin.x), std::abs(p.v[0].y - origin.y),
                           std::abs(p.v[0].z - origin.z)});
    const double width = (ratio + 2) * maxEdge + 128 * std::numeric_limits<double>::epsilon() * extent;
    if (!(width > 0) || !std::isfinite(width))
        throw InvalidArgument("Interaction-plan grid scale is not finite.");
    struct Key {
        int64_t x, y, z;
        bool operator==(const Key &o) const { return x == o.x && y == o.y && z == o.z; }
    };
    struct KeyHash {
        size_t operator()(const Key &k) const {
            return size_t(k.x * 73856093) ^ size_t(k.y * 19349663) ^ size_t(k.z * 83492791);
        }
    };
    const auto cell = [&](V3 p) {
        return Key{int64_t(std::floor((p.x - origin.x) / width)), int64_t(std::floor((p.y - origin.y) / width)),
                   int64_t(std::floor((p.z - origin.z) / width))};
    };
    std::unordered_map<Key, std::vector<uint32_t>, KeyHash> grid;
    std::vector<Key> where(sp.panels.size());
    for (size_t i = 0; i < sp.panels.size(); ++i) {
        where[i] = cell(sp.panels[i].v[0]);
        grid[where[i]].push_back(uint32_t(i));
    }
    // Each panel's partners j > i, sorted, on host threads; concatenated in
    // panel order this is the sorted pair list.
    const size_t T = sp.panels.size();
    std::vector<std::vector<uint32_t>> partners(T);
    std::atomic<size_t> next{0};
    const unsigned workers = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < std::min<size_t>(workers, (T + 255) / 256); ++w)
        pool.emplace_back([&]() {
            for (;;) {
                const size_t begin = next.fetch_add(256);
                if (begin >= T)
                    return;
                for (size_t i = begin; i < std::min(T, begin + 256); ++i) {
                    const auto &a = sp.panels[i];
                    auto &mine = partners[i];
                    for (int dx = -1; dx <= 1; ++dx)
                        for (int dy = -1; dy <= 1; ++dy)
                            for (int dz = -1; dz <= 1; ++dz) {
                                const auto it = grid.find(Key{where[i].x + dx, where[i].y + dy, where[i].z + dz});
                                if (it == grid.end())
                                    continue;
                                for (uint32_t j : it->second) {
                                    if (j <= i)
                                        continue;
                                    const auto &b = sp.panels[j];
                                    const double bound =
                                        ratio * std::max(a.maxEdge, b.maxEdge) + a.maxEdge + b.maxEdge;
                                    if (std::abs(a.v[0].x - b.v[0].x) > bound ||
                                        std::abs(a.v[0].y - b.v[0].y) > bound ||
                                        std::abs(a.v[0].z - b.v[0].z) > bound)
                                        continue;
                                    if (panelsDisjoint(a, b))
                                        mine.push_back(j);
                                }
                            }
                    std::sort(mine.begin(), mine.end());
                }
            }
        });
    for (auto &th : pool)
        th.join();
    size_t total = 0;
    for (const auto &m : partners)
        total += m.size();
    std::vector<std::pair<uint32_t, uint32_t>> out;
    out.reserve(total);
    for (size_t i = 0; i < T; ++i)
        for (uint32_t j : partners[i])
            out.emplace_back(uint32_t(i), j);
    return out;
}

// The host planner's per-pair step: regular-rule qualification, the
// geometric near test, then adaptive refinement of the pairs that need it
// (interaction_plan.cpp:228-300). Appends (key, rule) to `out`.
void processPair(const Space &sp, const std::vector<Bounds> &bounds, const PlanSettings &st, double maxK, uint32_t i,
                 uint32_t j, const volatile int32_t *cancel, std::vector<std::pair<uint64_t, PairRule>> &out,
                 bool classify) {
    const HostPanel &a = sp.panels[i], &b = sp.panels[j];
    if (classify) {
        if (!panelsDisjoint(a, b))
            return;
        const unsigned degree = qualifiedDegree(bounds[i], bounds[j], maxK, st.tol, st.regularOrder);
        const double h = std::max(a.maxEdge, b.maxEdge);
        const double limit = bounds[i].radius + bounds[j].radius + st.nearRatio * h;
        const double dx = a.centroid.x - b.centroid.x, dy = a.centroid.y - b.centroid.y,
                     dz = a.centroid.z - b.centroid.z;
        const bool geometricNear = degree && st.nearRatio > 0 && dx * dx + dy * dy + dz * dz < limit * limit &&
                                   isNearPair(a, b, st.nearRatio);
        if (degree && !geometricNear)
            return;
    }
    try {
        out.emplace_back((uint64_t(i) << 32) | j, adaptivePair(a, b, st, maxK, cancel));
    } catch (const Cancelled &) {
        throw;
    } catch (const std::exception &e) {
        std::ostringstream msg;
        msg << "Near pair panels " << i << '/' << j << " (faces " << a.face << '/' << b.face << ", k=" << maxK
            << ", gap=" << panelDistance(a, b) << " m, depth=" << st.maxDepth << "): " << e.what();
        throw NumericError(msg.str());
    }
}

// Runs `work(unit, results[unit])` for units 0..count-1 on up to `threads`
// host threads (0 = hardware concurrency, at most 64); the first exception
// stops the workers and is rethrown.
template <class Work>
void parallelUnits(size_t count, unsigned threads, const volatile int32_t *cancel,
                   std::vector<std::vector<std::pair<uint64_t, PairRule>>> &results, Work work) {
    std::atomic<size_t> next{0};
    std::atomic<bool> failed{false};
    std::exception_ptr failure;
    std::mutex failureMutex;
    unsigned workers = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
    workers = unsigned(std::min<size_t>({size_t(workers), size_t(64), std::max<size_t>(count, 1)}));
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < workers; ++w)
        pool.emplace_back([&]() {
            try {
                for (;;) {
                    if (failed.load(std::memory_order_relaxed))
                        return;
                    if (cancel && *cancel)
                        throw Cancelled();
                    const size_t u = next.fetch_add(1);
                    if (u >= count)
                        return;
                    work(u, results[u]);
                }
            } catch (...) {
                std::lock_guard<std::mutex> lock(failureMutex);
                if (!failure)
                    failure = std::current_exception();
                failed = true;
            }
        });
    for (auto &th : pool)
        th.join();
    if (failure)
        std::rethrow_exception(failure);
}

}  // namespace

Bounds makeBounds(const HostPanel &p) {
    Bounds b{p.centroid, 0, p.maxEdge, 1, 0};
    double e[3];
    for (int i = 0; i < 3; ++i) {
        const V3 a = p.v[i], c = p.v[(i + 1) % 3];
        e[i] = std::hypot(a.x - c.x, a.y - c.y, a.z - c.z);
        b.radius = std::max(b.radius, std::hypot(a.x - p.centroid.x, a.y - p.centroid.y, a.z - p.centroid.z));
    }
    b.radius = std::nextafter(b.radius * (1 + 8 * std::numeric_limits<double>::epsilon()),
                              std::numeric_limits<double>::infinity());
    constexpr double cos20 = .939692620785908384;
    bool q = true;
    for (int i = 0; i < 3; ++i) {
        const double x = e[i], y = e[(i + 1) % 3], z = e[(i + 2) % 3];
        q = q && x > 0 && y > 0 && (x * x + y * y - z * z) <= 2 * x * y * cos20;
    }
    b.qualified = q && std::isfinite(b.radius) && b.maxEdge > 0;
    return b;
}

PlanFrame beginPlan(const Space &sp, const PlanSettings &st, double maxK) {
    const size_t T = sp.panels.size();
    if (!T || !std::isfinite(maxK) || maxK < 0 || !std::isfinite(st.nearRatio) || st.nearRatio < 0 ||
        !std::isfinite(st.tol) || st.tol <= 0 || st.maxDepth > 16 || (st.regularOrder != 2 && st.regularOrder != 4) ||
        st.singularOrder < 2 || st.singularOrder > 20)
        throw InvalidArgument("Invalid BEM interaction-plan input or quadrature settings.");
    PlanFrame f;
    f.bounds.resize(T);
    f.allPairs = !((1e-6 + 4 * 3.5e-8) <= .2 * st.tol);
    for (size_t i = 0; i < T; ++i) {
        f.bounds[i] = makeBounds(sp.panels[i]);
        f.allPairs = f.allPairs || !f.bounds[i].qualified || maxK * sp.panels[i].maxEdge > 2;
    }
    Plan &plan = f.plan;
    if (f.allPairs)
        plan.wholePanelDegrees.assign(T * (T - 1) / 2, 0);
    plan.nearOffsets.assign(T + 1, 0);
    for (size_t t = 0; t < T; ++t) {
        std::vector<uint32_t> adj;
        for (int i = 0; i < 3; ++i) {
            const uint32_t n = sp.panels[t].nodes[i];
            for (uint32_t o = sp.incOffsets[n]; o < sp.incOffsets[n + 1]; ++o)
                adj.push_back(sp.incPanel[o]);
        }
        std::sort(adj.begin(), adj.end());
        adj.erase(std::unique(adj.begin(), adj.end()), adj.end());
        for (uint32_t s : adj)
            plan.touching.push_back({uint32_t(t), s, classifyNodes(sp.panels[t].nodes, sp.panels[s].nodes)});
    }
    if (!f.allPairs)
        f.candidates = candidates(sp, std::max(2.0, st.nearRatio));
    return f;
}

void appendPairRule(Plan &plan, bool allPairs, uint32_t i, uint32_t j, const Patch *patches, uint32_t count,
                    unsigned maxDepth, double relError) {
    if (allPairs && maxDepth == 0 && count == 1 && !patches[0].projection) {
        plan.wholePanelDegrees[unorderedPairIndex(i, j)] = uint8_t(patches[0].degree);
        plan.maxRelError = std::max(plan.maxRelError, relError);
        return;
    }
    const uint32_t first = uint32_t(plan.patches.size());
    plan.patches.insert(plan.patches.end(), patches, patches + count);
    plan.near.push_back({i, j, first, count, 0});
    plan.near.push_back({j, i, first, count, 1});
    plan.maxDepth = std::max(plan.maxDepth, maxDepth);
    plan.maxRelError = std::max(plan.maxRelError, relError);
}

void finishPlan(Plan &plan, size_t T) {
    // jobs by (test, trial): a counting sort by test, then each test's jobs by
    // trial (keys are unique, so this is the order of a full sort)
    std::vector<uint32_t> start(T + 1, 0);
    for (const auto &j : plan.near)
        ++start[j.test + 1];
    for (size_t r = 1; r <= T; ++r)
        start[r] += start[r - 1];
    std::vector<NearJob> sorted(plan.near.size());
    std::vector<uint32_t> fill(start.begin(), start.end() - 1);
    for (const auto &j : plan.near)
        sorted[fill[j.test]++] = j;
    for (size_t r = 0; r < T; ++r)
        std::sort(sorted.begin() + start[r], sorted.begin() + start[r + 1],
                  [](const NearJob &x, const NearJob &y) { return x.trial < y.trial; });
    plan.near = std::move(sorted);
    plan.nearTrials.reserve(plan.near.size());
    for (const auto &j : plan.near)
        plan.nearTrials.push_back(j.trial);
    plan.nearOffsets.assign(start.begin(), start.end());
}

std::vector<PairRule> planPairsOnHost(const Space &sp, const PlanSettings &st, double maxK,
                                      const std::vector<std::pair<uint32_t, uint32_t>> &pairs, unsigned threads,
                                      const volatile int32_t *cancel) {
    std::vector<std::vector<std::pair<uint64_t, PairRule>>> results(pairs.size());
    const std::vector<Bounds> none;
    parallelUnits(pairs.size(), threads, cancel, results, [&](size_t u, auto &out) {
        processPair(sp, none, st, maxK, pairs[u].first, pairs[u].second, cancel, out, false);
    });
    std::vector<PairRule> rules(pairs.size());
    for (size_t u = 0; u < pairs.size(); ++u)
        rules[u] = std::move(results[u].front().second);
    return rules;
}

double hostPatchError(const HostPanel &t, const HostPanel &s, const Patch &p, double k) {
    // a tensor patch's sub-triangles; fractions are powers of 1/4, so the
    // product in the sample weight is the same with the whole fraction on the
    // test side
    Sub a{}, b{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            a.v[i][j] = p.test[3 * i + j];
            b.v[i][j] = p.trial[3 * i + j];
        }
    a.fraction = p.areaFraction;
    b.fraction = 1;
    return estimate(t, s, a, b, p.degree, false, 1, k).error;
}

Plan makePlan(const Space &sp, const PlanSettings &st, double maxK, unsigned threads, const volatile int32_t *cancel) {
    PlanFrame f = beginPlan(sp, st, maxK);
    const size_t T = sp.panels.size();
    const size_t units = f.allPairs ? T : f.candidates.size();
    // Results per candidate (or per all-pairs row) keep the flattening order
    // independent of which worker integrated which pair.
    std::vector<std::vector<std::pair<uint64_t, PairRule>>> results(units);
    parallelUnits(units, threads, cancel, results, [&](size_t u, auto &out) {
        if (f.allPairs)
            for (uint32_t j = uint32_t(u) + 1; j < T; ++j)
                processPair(sp, f.bounds, st, maxK, uint32_t(u), j, cancel, out, true);
        else
            processPair(sp, f.bounds, st, maxK, f.candidates[u].first, f.candidates[u].second, cancel, out, true);
    });
    for (auto &row : results)
        for (auto &[key, rule] : row)
            appendPairRule(f.plan, f.allPairs, uint32_t(key >> 32), uint32_t(key & 0xffffffffu), rule.patches.data(),
                           uint32_t(rule.patches.size()), rule.maxDepth, rule.relError);
    finishPlan(f.plan, T);
    return std::move(f.plan);
}

}  // namespace hsb
