// Host-side check of the resident form's planner (psdm::plan_resident),
// linked against the built engine library and run on the CPU.
//
// Usage: res_plan_check ny nx dPML fs max_regions max_sw nrec [injection rows (0-based interior rows)...]
// Prints: fits nregions cover_errors kind_errors shape_errors nbr_errors rec_errors max_lanes_per_warp
//   cover: live cells of the padded grid not updated exactly once, or cells
//          above a free surface updated;
//   kind:  interior float4 items outside interior rows without injection or
//          the free surface, x-strip items outside the band rows or the
//          C-PML x-strips, z-strip items outside the interior columns of a
//          z-strip or within 3 rows of its edges, or items leaving their
//          region;
//   shape: regions not on 4-row boundaries, smaller than 8 x 8, taller than
//          384 rows or wider than max_sw - 6 columns, overlapping, or a
//          shared window leaving the allocation's rows;
//   nbr:   neighbour lists not symmetric or missing a region within the
//          read halo;
//   rec:   receivers not in the region that owns their cell.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "rtm_internal.h"

using namespace psdm;

int main(int argc, char** argv) {
    if (argc < 8) return 2;
    const int ny = atoi(argv[1]), nx = atoi(argv[2]), dPML = atoi(argv[3]), fs = atoi(argv[4]);
    const int max_regions = atoi(argv[5]), max_sw = atoi(argv[6]), nrec = atoi(argv[7]);
    StepArgs a;
    std::memset(&a, 0, sizeof a);
    a.ny = ny;
    a.nx = nx;
    a.dn = dPML + 2 * kAcc;
    a.nyt = ny + 2 * a.dn;
    a.nxt = nx + 2 * a.dn;
    a.zoff = (4 - a.dn % 4) % 4;
    a.ldz = (a.zoff + a.nyt + 31) / 32 * 32;
    a.fs = fs;
    std::vector<int> row_slot(a.ldz, -1);
    std::vector<char> inj(a.ldz, 0);
    for (int k = 8; k < argc; ++k) {
        row_slot[a.zoff + a.dn + atoi(argv[k])] = 0;
        inj[a.zoff + a.dn + atoi(argv[k])] = 1;
    }
    plan_tiles(&a, row_slot.data(), false);
    // receivers spread along an interior row near the top
    std::vector<int> rec_cell(nrec);
    for (int i = 0; i < nrec; ++i) {
        const int x = a.dn + (int)((long long)i * (nx - 1) / (nrec > 1 ? nrec - 1 : 1));
        rec_cell[i] = x * a.ldz + a.zoff + a.dn + 2;
    }
    ResPlan plan;
    const bool fits = plan_resident(a, max_regions, max_sw, nrec, rec_cell.data(), &plan);
    const int nreg = (int)plan.reg.size();
    if (!fits) {
        printf("0 %d 0 0 0 0 0 0\n", nreg);
        return 0;
    }
    long cover_err = 0, kind_err = 0, shape_err = 0, nbr_err = 0, rec_err = 0;
    int max_lanes = 0;
    std::vector<int> cover((size_t)a.ldz * a.nxt, 0);
    std::vector<int> owner((size_t)a.ldz * a.nxt, -1);
    for (int b = 0; b < nreg; ++b) {
        const ResRegion& R = plan.reg[b];
        if (R.zr0 % 4 || R.nrows % 4 || R.nrows < kResMinSide || R.nrows > kResRows || R.w < kResMinSide ||
            R.w + 6 > plan.sw || plan.sw > max_sw || R.zr0 < 0 || R.zr0 + R.nrows > a.ldz || R.x0 < 0 ||
            R.x0 + R.w > a.nxt)
            ++shape_err;
        for (int x = R.x0; x < R.x0 + R.w; ++x)
            for (int zd = R.zr0; zd < R.zr0 + R.nrows; ++zd) {
                if (zd < 0 || zd >= a.ldz || x < 0 || x >= a.nxt) continue;
                int& o = owner[(size_t)x * a.ldz + zd];
                if (o >= 0) ++shape_err;
                o = b;
            }
        for (int w = 0; w < kResWarps; ++w)
            for (int it = plan.warp_first[b * kResWarps + w]; it < plan.warp_first[b * kResWarps + w + 1]; ++it) {
                const int w0 = plan.items[2 * it], w1 = plan.items[2 * it + 1];
                const int kind = w0 & 15;
                const int first = w1 >> 16, c0 = w1 & 0xffff;
                // the cells of each lane: rows [zs, zs+nr) x columns [xa, xb)
                struct Lane { int zs, nr, xa, xb; };
                std::vector<Lane> lanes;
                if (kind == kResGen) {
                    const int ng = (w0 >> 4) & 15, nr = (w0 >> 8) & 255, span = w0 >> 16;
                    if (nr < 1 || ng < 1 || nr * ng > 32 || span < ng || span > 8 * ng) ++kind_err;
                    for (int l = 0; l < nr * ng && l < 32; ++l) {
                        const int k = l / nr;
                        lanes.push_back({R.zr0 + first + l % nr, 1, R.x0 + c0 + span * k / ng,
                                         R.x0 + c0 + span * (k + 1) / ng});
                        if (lanes.back().xb - lanes.back().xa > 8) ++kind_err;
                    }
                    if (nr * ng > max_lanes) max_lanes = nr * ng;
                } else {
                    const int ncol = (w0 >> 4) & 15, nl = w0 >> 8;
                    if (nl < 1 || nl > 32 || ncol < 1 || ncol > 10) ++kind_err;
                    if (nl > max_lanes) max_lanes = nl;
                    for (int l = 0; l < nl && l < 32; ++l)
                        lanes.push_back({R.zr0 + 4 * (first + l), 4, R.x0 + c0, R.x0 + c0 + ncol});
                }
                for (const Lane& L : lanes)
                    for (int x = L.xa; x < L.xb; ++x) {
                        if (x >= R.x0 + R.w || L.zs + L.nr > R.zr0 + R.nrows) ++kind_err;
                        for (int zd = L.zs; zd < L.zs + L.nr; ++zd) {
                            const int z = zd - a.zoff;
                            const bool in_x = x >= a.dn && x < a.dn + nx;
                            const bool band = z >= a.dn && z < a.dn + (ny & ~3);
                            if (kind == kResFast && (!in_x || !band || inj[zd] || (fs && z == a.dn))) ++kind_err;
                            if (kind == kResXpml && (in_x || !band)) ++kind_err;
                            if (kind == kResZpml) {
                                const int sb = z < a.dn ? 0 : a.dn + ny;
                                const bool strip = z >= 0 && z < a.nyt && (z < a.dn || z >= a.dn + ny) &&
                                                   !(fs && z < a.dn);
                                if (!in_x || !strip || z - sb < 3 || z - sb > a.dn - 4) ++kind_err;
                            }
                            if (zd >= 0 && zd < a.ldz && x >= 0 && x < a.nxt) ++cover[(size_t)x * a.ldz + zd];
                        }
                    }
            }
    }
    const int zlive0 = a.zoff + (fs ? a.dn : 0), zlive1 = a.zoff + a.nyt;
    for (int x = 0; x < a.nxt; ++x)
        for (int zd = 0; zd < a.ldz; ++zd) {
            const int c = cover[(size_t)x * a.ldz + zd];
            const bool live = zd >= zlive0 && zd < zlive1;
            if (live && c != 1) ++cover_err;
            if (!live && fs && zd < zlive0 && c != 0) ++cover_err;
        }
    // neighbours: symmetric, and every region within kTileReadHalo listed
    for (int b = 0; b < nreg; ++b) {
        const ResRegion& R = plan.reg[b];
        for (int o = 0; o < nreg; ++o) {
            if (o == b) continue;
            const ResRegion& Q = plan.reg[o];
            const bool near = Q.zr0 < R.zr0 + R.nrows + kTileReadHalo && R.zr0 < Q.zr0 + Q.nrows + kTileReadHalo &&
                              Q.x0 < R.x0 + R.w + kTileReadHalo && R.x0 < Q.x0 + Q.w + kTileReadHalo;
            bool listed = false, back = false;
            for (int k = R.nbr0; k < R.nbr0 + R.nnbr; ++k) listed = listed || plan.nbr[k] == o;
            for (int k = Q.nbr0; k < Q.nbr0 + Q.nnbr; ++k) back = back || plan.nbr[k] == b;
            if (near != listed || listed != back) ++nbr_err;
        }
        for (int k = R.rec0; k < R.rec0 + R.nrec; ++k) {
            const int cell = rec_cell[plan.rec[k]];
            const int x = cell / a.ldz, zd = cell % a.ldz;
            if (owner[(size_t)x * a.ldz + zd] != b) ++rec_err;
        }
    }
    if ((int)plan.rec.size() != nrec) ++rec_err;
    printf("1 %d %ld %ld %ld %ld %ld %d\n", nreg, cover_err, kind_err, shape_err, nbr_err, rec_err, max_lanes);
    return 0;
}
