// Host-side check of the tile plan of the two-step launches (psdm::plan_pair,
// psdm::pair_tile_rect, psdm::pair_rec_lists), linked against the built
// engine library and run on the CPU.
//
// Usage: pair_plan_check ny nx dPML fs nrec [injection rows (0-based interior rows)...]
// Prints: ntiles nclean cover_errors shape_errors clean_errors reach_errors rec_errors
//
// x-strip tiles (type 2): rows of a clean run, float4-aligned, at most 56 x 28.
//
// reach: every read of a tile's second step (the clamped x / z stencils of
// level n+1 and the strip-local phi stencils, rtm_pair.cu) lies in the tile
// plus a 3-cell ring, where the first step computes level n+1, and every
// stencil read of the first step on that ring lies in the cells loaded from
// level n (tile plus 6 cells for generic tiles, the staged rows and columns
// for clean tiles).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "rtm_internal.h"

using namespace psdm;

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

int main(int argc, char** argv) {
    if (argc < 6) return 2;
    const int ny = atoi(argv[1]), nx = atoi(argv[2]), dPML = atoi(argv[3]), fs = atoi(argv[4]);
    const int nrec = atoi(argv[5]);
    PairArgs P;
    std::memset(&P, 0, sizeof P);
    StepArgs& a = P.a;
    const Grid g = make_grid(dPML, ny, nx);
    a.ny = ny;
    a.nx = nx;
    a.dn = g.dn;
    a.nyt = g.nyt;
    a.nxt = g.nxt;
    a.zoff = g.zoff;
    a.ldz = g.ldz;
    a.fs = fs;
    const int dn = a.dn;
    std::vector<int> row_slot(a.ldz, -1);
    std::vector<char> inj_row(a.nyt, 0);
    for (int k = 6; k < argc; ++k) {
        const int z = dn + atoi(argv[k]);
        row_slot[a.zoff + z] = 0;
        inj_row[z] = 1;
    }
    if (!plan_pair(&P, row_slot.data())) {
        printf("0 0 1 0 0 0 0\n");
        return 0;
    }
    const int n = P.r_first[P.nrect];
    const int live0 = fs ? dn : 0;
    auto live = [&](int zd, int x) {
        const int z = zd - a.zoff;
        return z >= live0 && z < a.nyt && x >= 0 && x < a.nxt;
    };
    std::vector<int> cover((size_t)a.ldz * a.nxt, 0);
    long cover_err = 0, shape_err = 0, clean_err = 0, reach_err = 0, rec_err = 0;
    int nclean = 0;
    for (int b = 0; b < n; ++b) {
        int z0, z1, x0, x1;
        pair_tile_rect(P, b, &z0, &z1, &x0, &x1);
        int r = 0;
        while (r + 1 < P.nrect && b >= P.r_first[r + 1]) ++r;
        const bool clean = P.r_type[r] == 0, xs = P.r_type[r] == 2;
        nclean += clean;
        if (z0 >= z1 || x0 >= x1 || z0 < 0 || x0 < 0 || z1 > a.ldz || x1 > a.nxt) {
            ++shape_err;
            continue;
        }
        if (clean) {
            if (z0 % 4 || (z1 - z0) % 4 || z1 - z0 > 120 || x1 - x0 > P.txc) ++shape_err;
            // bulk copies and the first step's reads of level n-1 inside the arrays
            if (z0 - 8 < 0 || z1 + 8 > a.ldz || x0 - 6 < 0 || x1 + 6 > a.nxt) ++shape_err;
            // the tile and its 3-cell ring: interior cells, no free surface, no injection
            for (int zd = z0 - 3; zd < z1 + 3; ++zd)
                for (int x = x0 - 3; x < x1 + 3; ++x) {
                    const int z = zd - a.zoff;
                    if (z < dn || z >= dn + ny || x < dn || x >= dn + nx || (fs && z == dn) || inj_row[z])
                        ++clean_err;
                }
        } else if (xs) {
            if (z0 % 4 || (z1 - z0) % 4 || z1 - z0 > 56 || x1 - x0 > 28) ++shape_err;
            // float4 loads of level n on rows [z0-8, z1+8) inside the arrays
            if (z0 - 8 < 0 || z1 + 8 > a.ldz) ++shape_err;
            // rows of the tile and its ring: interior, no free surface, no injection
            for (int zd = z0 - 3; zd < z1 + 3; ++zd) {
                const int z = zd - a.zoff;
                if (z < dn || z >= dn + ny || (fs && z == dn) || inj_row[z]) ++clean_err;
            }
        } else if (z1 - z0 > 26 || x1 - x0 > 32) {
            ++shape_err;
        }
        // level-n cells a tile has: generic tile + 6; clean and x-strip: rows + 8
        const int lz0 = (clean || xs) ? z0 - 8 : z0 - 6, lz1 = (clean || xs) ? z1 + 8 : z1 + 6;
        const int lx0 = x0 - 6, lx1 = x1 + 6;
        auto in_ring3 = [&](int zd, int x) { return zd >= z0 - 3 && zd < z1 + 3 && x >= x0 - 3 && x < x1 + 3; };
        auto in_load = [&](int zd, int x) { return zd >= lz0 && zd < lz1 && x >= lx0 && x < lx1; };
        // stencil reads of a cell (clamped x / z stencils, strip-local phi)
        auto reads = [&](int zd, int x, bool with_phi, auto&& inside) {
            long bad = 0;
            const int z = zd - a.zoff;
            const int cx = clampi(x, 3, a.nxt - 4), czd = clampi(z, 3, a.nyt - 4) + a.zoff;
            for (int k = -3; k <= 3; ++k) {
                bad += !inside(zd, cx + k);
                bad += !inside(czd + k, x);
            }
            bad += !inside(zd, x);
            if (with_phi) {
                const int kz = (z < dn) ? (dn - z) : (z >= dn + ny ? z - (dn + ny) + 1 : 0);
                const int kx = (x < dn) ? (dn - x) : (x >= dn + nx ? x - (dn + nx) + 1 : 0);
                if (kx > 0) {
                    const int sb = (x < dn) ? 0 : dn + nx;
                    const int ci = clampi(x - sb, 3, dn - 4) + sb;
                    for (int k = -3; k <= 3; ++k) bad += !inside(zd, ci + k);
                }
                if (kz > 0) {
                    const int sb = (z < dn) ? 0 : dn + ny;
                    const int cj = clampi(z - sb, 3, dn - 4) + sb + a.zoff;
                    for (int k = -3; k <= 3; ++k) bad += !inside(cj + k, x);
                }
            }
            return bad;
        };
        for (int zd = z0; zd < z1; ++zd)
            for (int x = x0; x < x1; ++x) {
                if (!live(zd, x)) {
                    if (zd - a.zoff >= 0 && zd - a.zoff < a.nyt) ++cover_err;  // a dead row in a tile
                    continue;
                }
                ++cover[(size_t)x * a.ldz + zd];
                reach_err += reads(zd, x, true, in_ring3);
            }
        for (int zd = z0 - 3; zd < z1 + 3; ++zd)
            for (int x = x0 - 3; x < x1 + 3; ++x)
                if (live(zd, x)) reach_err += reads(zd, x, false, in_load);
    }
    for (int x = 0; x < a.nxt; ++x)
        for (int zd = 0; zd < a.ldz; ++zd) {
            const int c = cover[(size_t)x * a.ldz + zd];
            if (live(zd, x) ? c != 1 : c != 0) ++cover_err;
        }
    // receivers on the first interior row, spread over the window
    std::vector<int> cells(nrec);
    for (int i = 0; i < nrec; ++i) {
        const int x = dn + (int)((long)i * (nx - 1) / std::max(nrec - 1, 1));
        cells[i] = x * a.ldz + (dn + (fs ? 1 : 0)) + a.zoff;
    }
    std::vector<int> first, idx;
    pair_rec_lists(P, nrec, cells.data(), &first, &idx);
    std::vector<int> seen(nrec, 0);
    for (int b = 0; b < n; ++b) {
        int z0, z1, x0, x1;
        pair_tile_rect(P, b, &z0, &z1, &x0, &x1);
        for (int j = first[b]; j < first[b + 1]; ++j) {
            const int i = idx[j];
            const int x = cells[i] / a.ldz, zd = cells[i] % a.ldz;
            if (zd < z0 || zd >= z1 || x < x0 || x >= x1) ++rec_err;
            ++seen[i];
        }
    }
    for (int i = 0; i < nrec; ++i) rec_err += seen[i] != 1;
    printf("%d %d %ld %ld %ld %ld %ld\n", n, nclean, cover_err, shape_err, clean_err, reach_err, rec_err);
    return 0;
}
