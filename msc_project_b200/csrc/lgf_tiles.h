// Work lists of the persistent kernels: the order in which the RK3 stage and
// measurement kernels take their tiles (host code; tested on the CPU by
// tests/test_index_checked.py through lgf_check_index.cu).
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

#include "lgf_kernels.cuh"

namespace lgf {

// ------------------------------------------------------------ work order
// The persistent kernels take tiles in list order, so the list order sets the
// L2 reuse distance of the stencil.  In plain site order the x0 +- 1 (and, in
// the measurement, up to +- 3) neighbours of a site are reused one slice of
// work later; once a slice of work exceeds the L2 budget they come from HBM
// again.  Large lattices are therefore ordered in blocks of x1 (and x2) rows,
// each block swept through every x0 slice before the next block starts.  Only
// the order changes: the set of tiles is the same, and no result depends on
// it (no reduction runs in tile order).
// Block budgets, measured on 16^4 .. 48^4 (FP64, 100 steps): 8 MB / 2 MB gave
// +5% on 24^3x48 and +7% on 32^4 over the plain site order; 24/8, 12/4, 4/1
// and smaller were between the two.
// (The budgets are fields of TileShape: stage bytes, default 8 MB, and
// measurement link bytes, default 2 MB, per block and slice; x0 +- 3 keeps
// 7 slices of a measurement block live.)

// A block: x1 in [a1, b1), x2 in [a2, b2), all x3.  One block per slice when
// a slice of work fits the budget; else blocks of whole x1 rows, at least
// MIN_ROWS deep so that most x1 neighbours stay inside; else (lattices whose
// x1 rows are themselves large) square (x1, x2) blocks.
struct SiteBlock { int a1, b1, a2, b2; };
#ifndef LGF_MIN_ROWS
#define LGF_MIN_ROWS 4
#endif
constexpr int MIN_ROWS = LGF_MIN_ROWS;

inline std::vector<SiteBlock> site_blocks(const Geom& g, double budget, double bytes_per_site, int align2 = 1) {
    std::vector<SiteBlock> out;
    const int N1 = g.n[1], N2 = g.n[2], N3 = g.n[3];
    const double sites = budget / bytes_per_site;  // sites of one block and slice
    if ((double)g.Vs <= sites) {
        out.push_back({0, N1, 0, N2});
    } else if ((double)MIN_ROWS * N2 * N3 <= sites) {
        const int r = std::max(1, (int)(sites / ((double)N2 * N3)));
        for (int a = 0; a < N1; a += r) out.push_back({a, std::min(a + r, N1), 0, N2});
    } else {
        // square blocks; x2 boundaries on multiples of align2 (the measurement's patch rows)
        const int side = std::max(align2, (int)std::sqrt(sites / N3) / align2 * align2);
        for (int a = 0; a < N1; a += side)
            for (int c = 0; c < N2; c += side) out.push_back({a, std::min(a + side, N1), c, std::min(c + side, N2)});
    }
    return out;
}

// stage tiles of T consecutive sites (first site a multiple of T) of lattice
// i, each assigned to the block row that holds its first site
inline void append_stage_tiles(std::vector<int2>& tiles, int i, const Geom& g, int T, double budget,
                               double bytes_per_site) {
    const long long N3 = g.n[3], row = (long long)g.n[2] * N3;
    for (const SiteBlock& b : site_blocks(g, budget, bytes_per_site))
        for (long long x0 = 0; x0 < g.n[0]; ++x0)
            for (long long x1 = b.a1; x1 < b.b1; ++x1) {
                const long long base = x0 * g.Vs + x1 * row;
                const long long lo = base + b.a2 * N3, hi = base + b.b2 * N3;
                for (long long s0 = (lo + T - 1) / T * T; s0 < hi; s0 += T) tiles.push_back(make_int2(i, (int)s0));
            }
}

// Column order: a column is the tiles at one (x0, position in the x1 row) for
// x1 = 0..N1-1.  Columns are taken G at a time (G = the persistent grid) and
// listed row by row, so CTA b walks column b along x1: the x1 - 1 neighbours
// of its tile are the links of the tile it did before.  Needs tiles that lie
// inside one x1 row (N2 N3 a multiple of T) and bands of G columns that span
// at least 8 x0 slices (else most x0 neighbours fall on a band edge: 48^4
// with 64-site tiles spans 4); returns false otherwise.  Measured against the
// blocked order: +3-4% flow-only on 24^3x48 and 32^4.
inline bool append_stage_tiles_columns(std::vector<int2>& tiles, int i, const Geom& g, int T, int G) {
    const long long row = (long long)g.n[2] * g.n[3];
    if (row % T || G < 1) return false;
    const long long per_row = row / T, ncol = g.n[0] * per_row;
    if (8 * per_row > G && ncol > G) return false;
    for (long long c0 = 0; c0 < ncol; c0 += G) {
        const long long c1 = std::min(c0 + (long long)G, ncol);
        for (long long x1 = 0; x1 < g.n[1]; ++x1)
            for (long long c = c0; c < c1; ++c)
                tiles.push_back(make_int2(i, (int)((c / per_row) * g.Vs + x1 * row + (c % per_row) * T)));
    }
    return true;
}

// measurement tiles (lattice, slice, chunk of the slice) of lattice i; a
// chunk is a 32-site strip or a 4 x 8 patch (meas_patched, lgf_kernels.cuh)
inline void append_measure_tiles(std::vector<int4>& tiles, int i, const Geom& g, double budget,
                                 double bytes_per_site) {
    const long long N3 = g.n[3], row = (long long)g.n[2] * N3;
    if (meas_patched(g)) {
        const int nb3 = g.n[3] / MEAS_PATCH_COLS, nb2 = g.n[2] / MEAS_PATCH_ROWS;
        for (const SiteBlock& b : site_blocks(g, budget, bytes_per_site, MEAS_PATCH_ROWS))
            for (int t = 0; t < g.n[0]; ++t)
                for (int x1 = b.a1; x1 < b.b1; ++x1)
                    for (int c2 = b.a2 / MEAS_PATCH_ROWS; c2 * MEAS_PATCH_ROWS < b.b2; ++c2)
                        for (int c3 = 0; c3 < nb3; ++c3) tiles.push_back(make_int4(i, t, (x1 * nb2 + c2) * nb3 + c3, 0));
        return;
    }
    for (const SiteBlock& b : site_blocks(g, budget, bytes_per_site))
        for (int t = 0; t < g.n[0]; ++t)
            for (long long x1 = b.a1; x1 < b.b1; ++x1) {
                const long long lo = x1 * row + b.a2 * N3, hi = x1 * row + b.b2 * N3;
                for (long long c = (lo + MEAS_SITES - 1) / MEAS_SITES; c * MEAS_SITES < hi; ++c)
                    tiles.push_back(make_int4(i, t, (int)c, 0));
            }
}

// Launch segments: a group's members (in list order, each a contiguous run
// of the tile list) split into at most `slots` runs of whole members, each
// closed once it holds max(total / slots, min_run) tiles.  Each run is one
// launch of its own: on one B200 a launch over many large lattices ran its
// stages 6-15% and its measurements 7-200% slower per lattice than launches
// of one lattice each (measured on 8 x 24^3x48), while small lattices still
// share a launch (min_run keeps every launch several tiles per block deep).
inline std::vector<int2> member_runs(const std::vector<int>& tiles_per_member, int slots, long long min_run) {
    long long total = 0;
    for (int t : tiles_per_member) total += t;
    const long long target = std::max((total + slots - 1) / std::max(slots, 1), min_run);
    std::vector<int2> runs;
    long long first = 0, cur = 0;
    for (int t : tiles_per_member) {
        cur += t;
        if (cur >= target && (int)runs.size() < slots - 1) {
            runs.push_back(make_int2((int)first, (int)cur));
            first += cur;
            cur = 0;
        }
    }
    if (cur > 0 || runs.empty()) runs.push_back(make_int2((int)first, (int)cur));
    return runs;
}

}  // namespace lgf
