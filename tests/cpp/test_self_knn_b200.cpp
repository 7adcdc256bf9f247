// C++ parity test through the drop-in header include/fasttree/hlbvh.hpp, written like the
// reference's test/test_self_knn.cpp and test/main.cpp: host brute force over the sorted
// leaves, exact integer distances / 1e-4 relative float tolerance, indices compared at
// untied ranks only, no duplicate indices, sentinels beyond the available count; range
// count and kNN on the 10^3 grid; ghost visibility; a refit-only update and a save / load
// round trip (this library's additions).  Built once per configuration macro set
// (tests/test_cpp_api.py) and run on the GPU.  Exit code 0 = all passed.
#include <fasttree/hlbvh.hpp>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <numeric>
#include <random>
#include <string>
#include <vector>

using namespace fasttree;

static const double BOX = 100.0;

static coord_t to_coord(double v) {
#if defined(FASTTREE_INTEGER_COORDS)
    double n = std::min(std::max(v / BOX, 0.0), std::nextafter(1.0, 0.0));
    return static_cast<coord_t>(std::floor(n * std::ldexp(1.0, BITS_PER_DIMENSION)));
#else
    return static_cast<coord_t>(v);
#endif
}

static dist_t point_dist(coord_t ax, coord_t ay, coord_t az, coord_t bx, coord_t by, coord_t bz) {
#if defined(FASTTREE_INTEGER_COORDS)
    constexpr int      shift = BITS_PER_DIMENSION > 31 ? BITS_PER_DIMENSION - 31 : 0;
    auto axis = [](coord_t a, coord_t b) -> uint64_t {
#if defined(PERIODIC_BC)
        constexpr int sb = (sizeof(coord_t) == 8 ? 64 : 32) - BITS_PER_DIMENSION;
        if constexpr (sizeof(coord_t) == 8) a &= (coord_t)((coord_t(1) << BITS_PER_DIMENSION) - 1);
        if (a == b) return 0;
        using S  = std::conditional_t<sizeof(coord_t) == 8, int64_t, int32_t>;
        S    d   = static_cast<S>(static_cast<coord_t>(a - b) << sb) >> sb;
        uint64_t g = static_cast<uint64_t>(d < 0 ? -d : d);
        return g >> shift;
#else
        return (a < b ? (uint64_t)(coord_t)(b - a) : (uint64_t)(coord_t)(a - b)) >> shift;
#endif
    };
    uint64_t dx = axis(ax, bx), dy = axis(ay, by), dz = axis(az, bz);
    return dx * dx + dy * dy + dz * dz;
#else
    coord_t dx = ax - bx, dy = ay - by, dz = az - bz;
    dx = dx < 0 ? -dx : dx;
    dy = dy < 0 ? -dy : dy;
    dz = dz < 0 ? -dz : dz;
    coord_t s = dx * dx;
    s         = s + dy * dy;
    s         = s + dz * dz;
    return static_cast<double>(s);
#endif
}

struct BF {
    dist_t d;
    size_t idx;
    bool   tied;
};

static std::vector<std::vector<BF>> brute_force(const TreeSoA &t, const std::vector<int> &ranks, int k, bool excl) {
    size_t                       n  = t.num_leaves, ni = t.num_internal;
    std::vector<std::vector<BF>> out;
    for (int q : ranks) {
        std::vector<BF> c;
        for (size_t j = 0; j < n; ++j) {
            if (excl && (int)j == q) continue;
            dist_t d = point_dist(t.min_x[ni + q], t.min_y[ni + q], t.min_z[ni + q], t.min_x[ni + j], t.min_y[ni + j],
                                  t.min_z[ni + j]);
#if defined(RETURN_ORIG_INDICES)
            size_t r = (size_t)t.orig_idx[ni + j];
#else
            size_t r = j;
#endif
            c.push_back({d, r, false});
        }
        std::sort(c.begin(), c.end(), [](const BF &a, const BF &b) { return a.d != b.d ? a.d < b.d : a.idx < b.idx; });
        for (size_t i = 0; i < c.size(); ++i) {
            auto near = [](dist_t a, dist_t b) {
#if defined(FASTTREE_INTEGER_COORDS)
                return a == b;
#else
                return std::abs((double)a - (double)b) <= 1e-4 * std::max((double)a, 1.0) + 1e-9;
#endif
            };
            c[i].tied = (i > 0 && near(c[i].d, c[i - 1].d)) || (i + 1 < c.size() && near(c[i].d, c[i + 1].d));
        }
        if (c.size() > (size_t)k) c.resize(k);
        out.push_back(c);
    }
    return out;
}

static int failures = 0;

static void verify(const std::string &name, const size_t *idx, const dist_t *dist, const std::vector<std::vector<BF>> &exp,
                   int k) {
    int bad = 0;
    for (size_t q = 0; q < exp.size(); ++q) {
        std::vector<size_t> seen;
        for (int i = 0; i < k; ++i)
            if (idx[q * k + i] != (size_t)-1) seen.push_back(idx[q * k + i]);
        std::sort(seen.begin(), seen.end());
        if (std::adjacent_find(seen.begin(), seen.end()) != seen.end()) ++bad;
        for (int i = 0; i < k; ++i) {
            if (i < (int)exp[q].size()) {
#if defined(FASTTREE_INTEGER_COORDS)
                if (dist[q * k + i] != exp[q][i].d) ++bad;
#else
                double a = dist[q * k + i], b = exp[q][i].d;
                if (std::abs(a - b) > 1e-4 * std::max(b, 1.0) + 1e-9) ++bad;
#endif
                if (!exp[q][i].tied && idx[q * k + i] != exp[q][i].idx) ++bad;
            } else if (idx[q * k + i] != (size_t)-1) {
                ++bad;
            }
        }
    }
    std::printf("  %s: %s (%d mismatches)\n", name.c_str(), bad ? "FAILED" : "PASSED", bad);
    failures += bad != 0;
}

static particles<coord_t> generate(const std::string &kind, size_t n, unsigned seed) {
    particles<coord_t> p;
    std::mt19937       g(seed);
    std::uniform_real_distribution<double> u(0.0, BOX), u2(0.1 * BOX, 0.9 * BOX);
    std::normal_distribution<double>       c1(0.25 * BOX, 0.04 * BOX), c2(0.75 * BOX, 0.04 * BOX);
    std::vector<std::array<double, 3>>     centres(10);
    for (auto &c : centres) c = {u2(g), u2(g), u2(g)};
    for (size_t i = 0; i < n; ++i) {
        double x, y, z;
        if (kind == "uniform") {
            x = u(g), y = u(g), z = u(g);
        } else if (kind == "clustered") {
            if (i < n * 0.45) x = c1(g), y = c1(g), z = c1(g);
            else if (i < n * 0.85) x = c2(g), y = c2(g), z = c2(g);
            else x = u(g), y = u(g), z = u(g);
            x = std::clamp(x, 1e-4, BOX - 1e-4);
            y = std::clamp(y, 1e-4, BOX - 1e-4);
            z = std::clamp(z, 1e-4, BOX - 1e-4);
        } else {
            if (i < n * 0.6) x = centres[i % 10][0], y = centres[i % 10][1], z = centres[i % 10][2];
            else x = u2(g), y = u2(g), z = u2(g);
        }
        p.pos_x.push_back(to_coord(x));
        p.pos_y.push_back(to_coord(y));
        p.pos_z.push_back(to_coord(z));
        p.id.push_back((uint32_t)i);
    }
    return p;
}

template <int MAXK> static void self_knn_case(queue &q, const TreeSoA &t, int k, bool excl, const std::string &label) {
    size_t  n = t.num_leaves;
    size_t *r = malloc_shared<size_t>(n * k, q);
    dist_t *d = malloc_shared<dist_t>(n * k, q);
    self_knn_query<MAXK>(q, t, k, r, d, excl);
    q.wait();
    std::vector<int> ranks(n);
    std::iota(ranks.begin(), ranks.end(), 0);
    verify(label, r, d, brute_force(t, ranks, k, excl), k);
    free(r, q);
    free(d, q);
}

int main() {
    queue q(0);
    std::printf("fasttree_b200 C++ API parity test (coord bytes %zu)\n", sizeof(coord_t));
    for (std::string kind : {"uniform", "clustered", "degenerate"}) {
        auto    p = generate(kind, 1000, 42);
        TreeSoA tree(q, p.pos_x.size());
        build_bvh(q, p, tree);
        for (bool excl : {true, false}) {
            std::string e = excl ? " excl" : " incl";
            self_knn_case<32>(q, tree, 16, excl, kind + " k=16" + e);
            self_knn_case<32>(q, tree, 32, excl, kind + " k=32" + e);
            self_knn_case<256>(q, tree, 33, excl, kind + " k=33" + e);
            self_knn_case<256>(q, tree, 64, excl, kind + " k=64" + e);
        }
        // subset: every n/17th plus the boundaries (test/test_self_knn.cpp:613-677)
        std::vector<int> ids;
        for (size_t i = 0; i < tree.num_leaves; i += tree.num_leaves / 17) ids.push_back((int)i);
        ids.push_back(0);
        ids.push_back((int)tree.num_leaves - 1);
        std::sort(ids.begin(), ids.end());
        ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
        int *dids = malloc_shared<int>(ids.size(), q);
        std::copy(ids.begin(), ids.end(), dids);
        size_t *r = malloc_shared<size_t>(ids.size() * 40, q);
        dist_t *d = malloc_shared<dist_t>(ids.size() * 40, q);
        self_knn_query_subset(q, tree, dids, (int)ids.size(), 40, r, d, true);
        q.wait();
        verify(kind + " subset k=40", r, d, brute_force(tree, ids, 40, true), 40);
        free(r, q);
        free(d, q);
        free(dids, q);
        // MAXK guard (src/hlbvh.hpp:1940-1944)
        bool threw = false;
        try {
            self_knn_query<32>(q, tree, 33, nullptr, nullptr, true);
        } catch (const std::invalid_argument &) {
            threw = true;
        }
        std::printf("  %s k > MAXK throws invalid_argument: %s\n", kind.c_str(), threw ? "PASSED" : "FAILED");
        failures += !threw;
        // refit-only update (new positions for the same points, topology kept), then a
        // save / load round trip of the refit tree
        {
            auto p2 = generate(kind, 1000, 43);
            refit_bvh(q, p2, tree);
            self_knn_case<32>(q, tree, 16, true, kind + " refit k=16");
            std::vector<unsigned char> blob = save_tree(q, tree);
            TreeSoA                    t2(q, tree.num_leaves);
            load_tree(q, blob, t2);
            self_knn_case<32>(q, t2, 16, true, kind + " loaded k=16");
        }
    }
    // 10^3 grid (test/main.cpp:84-241): range count vs brute force at (52,52,52), r <= 20
    {
        particles<coord_t> p;
        for (int ix = 0; ix < 10; ++ix)
            for (int iy = 0; iy < 10; ++iy)
                for (int iz = 0; iz < 10; ++iz) {
                    p.pos_x.push_back(to_coord((ix + 0.5) * 10));
                    p.pos_y.push_back(to_coord((iy + 0.5) * 10));
                    p.pos_z.push_back(to_coord((iz + 0.5) * 10));
                }
        TreeSoA tree(q, 1000);
        build_bvh(q, p, tree);
        coord_t qx = to_coord(52.0), rm = to_coord(0.0);
#if defined(FASTTREE_INTEGER_COORDS)
        coord_t RM = (coord_t)(20.0 / BOX * std::ldexp(1.0, BITS_PER_DIMENSION));
#else
        coord_t RM = 20.0;
#endif
        std::vector<int> res(1000);
        int              cnt = 0;
        range_query(q, tree, &qx, &qx, &qx, &rm, &RM, 1, res.data(), &cnt, 1000);
        int    expect = 0;
        size_t ni     = tree.num_internal;
#if defined(FASTTREE_INTEGER_COORDS)
        constexpr int shift = BITS_PER_DIMENSION > 31 ? BITS_PER_DIMENSION - 31 : 0;
        uint64_t      r2    = (uint64_t)(RM >> shift) * (uint64_t)(RM >> shift);
#else
        double r2 = 400.0;
#endif
        for (size_t i = 0; i < 1000; ++i)
            if ((double)point_dist(qx, qx, qx, tree.min_x[ni + i], tree.min_y[ni + i], tree.min_z[ni + i]) <= (double)r2)
                ++expect;
        std::printf("  grid range count %d expected %d: %s\n", cnt, expect, cnt == expect ? "PASSED" : "FAILED");
        failures += cnt != expect;
        size_t idx[48];
        dist_t dd[48];
        knn_query<128>(q, tree, &qx, &qx, &qx, 48, 1, idx, dd);
        std::vector<int> all(1);
        std::vector<BF>  bf;
        for (size_t i = 0; i < 1000; ++i)
            bf.push_back({point_dist(qx, qx, qx, tree.min_x[ni + i], tree.min_y[ni + i], tree.min_z[ni + i]), i, false});
        std::sort(bf.begin(), bf.end(), [](const BF &a, const BF &b) { return a.d < b.d; });
        int bad = 0;
        for (int i = 0; i < 48; ++i) bad += dd[i] != bf[i].d;
        std::printf("  grid knn_query<128> k=48 distances: %s\n", bad ? "FAILED" : "PASSED");
        failures += bad != 0;
    }
    std::printf("%s\n", failures ? "SOME TESTS FAILED" : "ALL TESTS PASSED");
    return failures ? 1 : 0;
}
