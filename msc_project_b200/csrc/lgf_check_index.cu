// CPU check of the engine's index arithmetic and work lists, built with
// -DLGF_CHECKED (every coordinate, direction and site index the helpers of
// lgf_lattice.cuh touch is asserted in range) and run on small lattices with
// every extent distinct, odd slice sizes and tails shorter than a layout block.
// Host code only: no GPU is needed.  Checked against plain coordinate
// arithmetic (periodic wrap, LGF/Lattice/Lattice.cpp:423-459):
//   - site <-> coordinates, forward/backward neighbours in every direction;
//   - the staple's neighbour sites x+mu, x+nu, x-nu, x-nu+mu (k_rk3_stage);
//   - the loop walks of the measurement (Plane::advance) for every plane,
//     quadrant and length 1..3;
//   - the device layouts of both precisions (link_offset, alg_offset) are
//     bijections into the padded buffers with 16-byte aligned vector loads;
//   - the stage and measurement tile lists cover every tile exactly once for
//     row-block and column orders and a range of budgets and block sizes, and
//     the measurement's strips or patches cover every site of a slice once;
//   - the launch segments of a group (member_runs) split a list of members
//     into at most `slots` back-to-back runs of whole members covering it.
// Prints one line and exits 0 when everything holds.
#include <cstdio>
#include <cstdlib>
#include <set>
#include <vector>

// both measurement geometries are checked: strips by default builds, patches here
#ifndef LGF_MEAS_PATCH
#define LGF_MEAS_PATCH 1
#endif
#include "lgf_tiles.h"

using namespace lgf;

static int g_fail = 0;
#define CHECK(cond)                                                                     \
    do {                                                                                \
        if (!(cond)) {                                                                  \
            std::fprintf(stderr, "check failed: %s (%s:%d)\n", #cond, __FILE__, __LINE__); \
            if (++g_fail > 20) std::exit(1);                                            \
        }                                                                               \
    } while (0)

static int idx(const Geom& g, const int x[4]) {
    int s = 0;
    for (int d = 0; d < 4; ++d) s = s * g.n[d] + ((x[d] % g.n[d]) + g.n[d]) % g.n[d];
    return s;
}

static void check_neighbours(const Geom& g) {
    for (int s = 0; s < g.V; ++s) {
        const Coord c = site_coord(g, s);
        CHECK(idx(g, c.x) == s);
        for (int d = 0; d < 4; ++d) {
            int y[4] = {c.x[0], c.x[1], c.x[2], c.x[3]};
            y[d] += 1;
            CHECK(fwd(g, s, d, c.x[d]) == idx(g, y));
            CHECK(fwd(s, dir_of(g, c, d)) == idx(g, y));
            y[d] -= 2;
            CHECK(bwd(g, s, d, c.x[d]) == idx(g, y));
            CHECK(bwd(s, dir_of(g, c, d)) == idx(g, y));
        }
        // the staple's neighbour sites, as k_rk3_stage forms them
        for (int mu = 0; mu < 4; ++mu) {
            const Dir dm = dir_of(g, c, mu);
            const int xpm = fwd(s, dm);
            for (int nu = 0; nu < 4; ++nu) {
                if (nu == mu) continue;
                const int xpn = fwd(g, s, nu, c.x[nu]), xmn = bwd(g, s, nu, c.x[nu]);
                const int xmnpm = fwd(xmn, dm);
                int y[4] = {c.x[0], c.x[1], c.x[2], c.x[3]};
                y[mu] += 1;
                CHECK(xpm == idx(g, y));
                y[mu] -= 1;
                y[nu] += 1;
                CHECK(xpn == idx(g, y));
                y[nu] -= 2;
                CHECK(xmn == idx(g, y));
                y[mu] += 1;
                CHECK(xmnpm == idx(g, y));
            }
        }
    }
}

// Plane::advance walks (the measurement's loop corners)
static void check_plane_walks(const Geom& g) {
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = mu + 1; nu < 4; ++nu)
            for (int s = 0; s < g.V; s += 7) {
                const Coord c = site_coord(g, s);
                Plane<double> P;
                P.U = nullptr;
                P.V = g.V;
                P.mu = mu;
                P.nu = nu;
                P.dm = dir_of(g, c, mu);
                P.dn = dir_of(g, c, nu);
                for (int sm = -1; sm <= 1; sm += 2)
                    for (int sn = -1; sn <= 1; sn += 2)
                        for (int a = 1; a <= 3; ++a)
                            for (int b = 1; b <= 3; ++b) {
                                PlanePos p = {s, P.dm.x, P.dn.x};
                                P.advance(p, true, sm, a);
                                P.advance(p, false, sn, b);
                                int y[4] = {c.x[0], c.x[1], c.x[2], c.x[3]};
                                y[mu] += sm * a;
                                y[nu] += sn * b;
                                CHECK(p.s == idx(g, y));
                                CHECK(p.xm == ((y[mu] % g.n[mu]) + g.n[mu]) % g.n[mu]);
                                CHECK(p.xn == ((y[nu] % g.n[nu]) + g.n[nu]) % g.n[nu]);
                            }
            }
}

// the device layout of precision R is a bijection into the padded buffers,
// and every vector load starts on a 16-byte boundary
template <typename R> static void check_layout(const Geom& g) {
    const size_t Vp = padded_sites(g.V);
    std::vector<char> seen(Vp * 36, 0), seen_a(Vp * 32, 0);
    for (int s = 0; s < g.V; ++s)
        for (int mu = 0; mu < 4; ++mu) {
            for (int k = 0; k < 9; ++k) {
                const size_t o = link_offset<R>(mu, k, s);
                CHECK(o < Vp * 36);
                if (o < Vp * 36) CHECK(!seen[o]++);
            }
            // double: every entry is a 16-byte load; float: entries 0, 2, 4, 6 start float4 loads
            for (int k = 0; k < 9; ++k)
                if (sizeof(R) == 8 || (k < 8 && k % 2 == 0)) CHECK((link_offset<R>(mu, k, s) * 2 * sizeof(R)) % 16 == 0);
            if (sizeof(R) == 4)
                for (int k = 0; k < 8; k += 2) CHECK(link_offset<R>(mu, k + 1, s) == link_offset<R>(mu, k, s) + 1);
            for (int a = 0; a < 8; ++a) {
                const size_t o = alg_offset<R>(mu, a, s);
                CHECK(o < Vp * 32);
                if (o < Vp * 32) CHECK(!seen_a[o]++);
            }
            const int per = 16 / sizeof(R);  // reals of one vector load
            for (int a = 0; a < 8; a += per) {
                CHECK((alg_offset<R>(mu, a, s) * sizeof(R)) % 16 == 0);
                for (int b = 1; b < per; ++b) CHECK(alg_offset<R>(mu, a + b, s) == alg_offset<R>(mu, a, s) + b);
            }
        }
}

static void check_tiles(const Geom& g) {
    const double bps_stage = 4.0 * (2 * 18 + 8) * 8, bps_meas = 4.0 * 18 * 8;
    for (int T : {32, 64, 96}) {
        std::set<int> want;
        for (int s0 = 0; s0 < g.V; s0 += T) want.insert(s0);
        for (double budget : {1.0e3, 2.0e4, 3.0e5, 8.0e6}) {
            std::vector<int2> tiles;
            append_stage_tiles(tiles, 3, g, T, budget, bps_stage);
            std::multiset<int> got;
            for (const int2& t : tiles) {
                CHECK(t.x == 3);
                got.insert(t.y);
            }
            CHECK(got.size() == want.size() && std::set<int>(got.begin(), got.end()) == want);
        }
        for (int G : {1, 16, 148, 4096}) {
            std::vector<int2> tiles;
            if (!append_stage_tiles_columns(tiles, 1, g, T, G)) continue;
            std::multiset<int> got;
            for (const int2& t : tiles) got.insert(t.y);
            CHECK(got.size() == want.size() && std::set<int>(got.begin(), got.end()) == want);
        }
    }
    const int nchunk = (g.Vs + MEAS_SITES - 1) / MEAS_SITES;
    // every site of a slice is exactly one lane of one chunk
    {
        std::vector<char> hit(g.Vs, 0);
        for (int c = 0; c < nchunk; ++c)
            for (int l = 0; l < MEAS_SITES; ++l) {
                const int off = meas_site_offset(g, meas_patched(g), c, l);
                if (off < g.Vs) CHECK(!hit[off]++);
                else CHECK(!meas_patched(g));  // only a strip's last chunk runs past the slice
            }
        for (int o = 0; o < g.Vs; ++o) CHECK(hit[o] == 1);
    }
    for (double budget : {1.0e3, 2.0e4, 3.0e5, 2.0e6, 6.4e7}) {
        std::vector<int4> tiles;
        append_measure_tiles(tiles, 2, g, budget, bps_meas);
        std::set<long long> got;
        for (const int4& t : tiles) {
            CHECK(t.x == 2 && t.y >= 0 && t.y < g.n[0] && t.z >= 0 && t.z < nchunk);
            CHECK(got.insert((long long)t.y * nchunk + t.z).second);
        }
        CHECK((long long)got.size() == (long long)g.n[0] * nchunk);
    }
}

static void check_member_runs() {
    const std::vector<std::vector<int>> lists = {
        {}, {0}, {5}, {20736}, {43, 43, 43}, {683, 20736, 683, 683, 2048, 165888, 1},
        std::vector<int>(64, 43), std::vector<int>(16, 20736), {0, 7, 0, 9}};
    for (const auto& lens : lists)
        for (int slots : {1, 2, 3, 16, 32})
            for (long long min_run : {0LL, 1LL, 1184LL, 3552LL, 100000LL}) {
                const std::vector<int2> runs = member_runs(lens, slots, min_run);
                CHECK(!runs.empty() && (int)runs.size() <= slots);
                // runs are back to back, cover the list, and end on member boundaries
                std::set<long long> bounds;
                long long acc = 0;
                bounds.insert(0);
                for (int t : lens) bounds.insert(acc += t);
                long long next = 0;
                for (const int2& r : runs) {
                    CHECK(r.x == next && r.y >= 0);
                    next += r.y;
                    CHECK(bounds.count(next) == 1);
                }
                CHECK(next == acc);
            }
}

int main() {
    check_member_runs();
    const int shapes[][4] = {{4, 4, 4, 4}, {4, 6, 8, 10}, {6, 6, 6, 6}, {4, 4, 6, 6}, {8, 4, 6, 4},
                             {10, 4, 4, 8}, {4, 20, 18, 18}, {4, 6, 6, 10}, {4, 6, 8, 16}, {6, 4, 12, 8}};
    int n = 0;
    for (const auto& sh : shapes) {
        const Geom g = make_geom(sh);
        check_neighbours(g);
        check_plane_walks(g);
        check_layout<double>(g);
        check_layout<float>(g);
        check_tiles(g);
        ++n;
    }
    if (g_fail) {
        std::printf("index check FAILED: %d failures\n", g_fail);
        return 1;
    }
    std::printf("index check ok: %d lattices\n", n);
    return 0;
}
