// Host-side check of the engine's tile planner (psdm::plan_tiles,
// psdm::tile_rect) and of the neighbour and receiver lists of the
// one-launch-per-pass form (psdm::pass_lists), linked against the built
// engine library and run on the CPU.
//
// Usage: plan_check ny nx dPML fs form nrec [injection rows (0-based interior rows)...]
//   form: 0 one-shot backward pass, 1 batched launch, 2 one-shot forward pass
// Prints: ntiles itx ixb cover_errors dead_errors type_errors sym_errors rec_errors
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "rtm_internal.h"

using namespace psdm;

int main(int argc, char** argv) {
    if (argc < 7) return 2;
    const int ny = atoi(argv[1]), nx = atoi(argv[2]), dPML = atoi(argv[3]), fs = atoi(argv[4]);
    const int form = atoi(argv[5]);
    const bool batched = form == 1;
    const int nrec = atoi(argv[6]);
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
    for (int k = 7; k < argc; ++k) row_slot[a.zoff + a.dn + atoi(argv[k])] = 0;
    plan_tiles(&a, row_slot.data(), batched, form == 2);
    const int n = a.r_first[a.nrect];
    // every live cell of the padded grid in exactly one tile; the rows above
    // a free surface in none
    std::vector<int> cover((size_t)a.ldz * a.nxt, 0);
    std::vector<int> owner((size_t)a.ldz * a.nxt, -1);
    long type_err = 0;
    for (int b = 0; b < n; ++b) {
        int z0, z1, x0, x1;
        tile_rect(a, b, &z0, &z1, &x0, &x1);
        if (z0 >= z1 || x0 >= x1 || z0 < 0 || x0 < 0 || z1 > a.ldz || x1 > a.nxt) ++type_err;
        int r = 0;
        while (r + 1 < a.nrect && b >= a.r_first[r + 1]) ++r;
        for (int x = x0; x < x1; ++x)
            for (int zd = z0; zd < z1; ++zd) {
                if (zd < 0 || zd >= a.ldz) continue;
                ++cover[(size_t)x * a.ldz + zd];
                owner[(size_t)x * a.ldz + zd] = b;
                const int z = zd - a.zoff;
                const bool special = (fs && z == a.dn) || row_slot[zd] >= 0;
                // interior tiles hold neither injection rows nor the free surface
                if (a.r_type[r] == 0 && special) ++type_err;
                if (a.r_type[r] == 0 && (z < a.dn || z >= a.dn + ny || x < a.dn || x >= a.dn + nx)) ++type_err;
            }
        if (a.r_type[r] == 0 && x1 - x0 > a.itx) ++type_err;
    }
    long cover_err = 0, dead_err = 0;
    for (int x = 0; x < a.nxt; ++x)
        for (int z = 0; z < a.nyt; ++z) {
            const int c = cover[(size_t)x * a.ldz + z + a.zoff];
            if (fs && z < a.dn) {
                if (c != 0) ++dead_err;
            } else if (c != 1) {
                ++cover_err;
            }
        }
    // neighbour lists: symmetric, no self, and every tile whose cells lie
    // within the halo of another is its neighbour
    std::vector<int> rec(nrec);
    for (int i = 0; i < nrec; ++i) {
        const int x = a.dn + (i * 7) % nx, z = a.dn + (i * 3) % ny;
        rec[i] = x * a.ldz + z + a.zoff;
    }
    std::vector<int> nf, nb, rf, ri;
    pass_lists(a, nrec, rec.data(), &nf, &nb, &rf, &ri);
    long sym_err = 0;
    std::vector<std::vector<char>> adj(n, std::vector<char>(n, 0));
    for (int b = 0; b < n; ++b)
        for (int k = nf[b]; k < nf[b + 1]; ++k) {
            if (nb[k] == b) ++sym_err;
            adj[b][nb[k]] = 1;
        }
    for (int b = 0; b < n; ++b)
        for (int c = 0; c < n; ++c)
            if (adj[b][c] != adj[c][b]) ++sym_err;
    const int H = kTileReadHalo;
    for (int b = 0; b < n; ++b) {
        int z0, z1, x0, x1;
        tile_rect(a, b, &z0, &z1, &x0, &x1);
        for (int x = x0 - H; x < x1 + H; ++x)
            for (int zd = z0 - H; zd < z1 + H; ++zd) {
                if (x < 0 || x >= a.nxt || zd < 0 || zd >= a.ldz) continue;
                const int o = owner[(size_t)x * a.ldz + zd];
                if (o >= 0 && o != b && !adj[b][o]) ++sym_err;
            }
    }
    long rec_err = 0;
    std::vector<int> seen(nrec, 0);
    for (int b = 0; b < n; ++b)
        for (int k = rf[b]; k < rf[b + 1]; ++k) {
            const int i = ri[k];
            ++seen[i];
            if (owner[(size_t)rec[i]] != b) ++rec_err;
        }
    for (int i = 0; i < nrec; ++i)
        if (seen[i] != 1) ++rec_err;
    printf("%d %d %d %ld %ld %ld %ld %ld\n", n, a.itx, a.ixb, cover_err, dead_err, type_err, sym_err, rec_err);
    return 0;
}
