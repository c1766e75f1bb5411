// Survey geometry on the host, before any shot reaches the GPU: the
// navigation file of the shots, the channel positions of a shot, their grid
// indices, the velocity model on the propagation grid and the sea-floor
// depth the trace windows are cut from.  Each function follows one routine
// of the reference in its FP32 operation order:
//   psdm_nav_read            read_nav_shot_mcs   src/get_mcs_data.f90:30-126
//   psdm_channel_positions   get_pos_channels    src/get_mcs_data.f90:418-510
//   psdm_geometry_mcs        get_geometry_mcs    src/get_mcs_data.f90:128-148
//   psdm_linear_2d           linear_2D, linear_interpolation_1D
//                                                src/linear_interpolation.f90:1-117
//   psdm_batmodel_from_velocity                  src/00-main.f90:146-158
// The navigation file is read as Fortran list-directed input: one record per
// line, values separated by blanks or commas, reals in any Fortran form
// (including a D exponent).

#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/psdm_rtm.h"
#include "rtm_internal.h"

namespace {

int fail_arg(const std::string& msg) {
    psdm::set_last_error(msg.c_str());
    return PSDM_ERR_ARG;
}

// Split one record into its values (blank or comma separated; a slash ends
// the record, as in list-directed input).
std::vector<std::string> fields(const std::string& line) {
    std::vector<std::string> out;
    std::string cur;
    for (char ch : line) {
        if (ch == '/') break;
        if (ch == ',' || std::isspace((unsigned char)ch)) {
            if (!cur.empty()) out.push_back(cur);
            cur.clear();
        } else {
            cur.push_back(ch);
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

bool to_int(const std::string& s, int* v) {
    errno = 0;
    char* end = nullptr;
    const long x = std::strtol(s.c_str(), &end, 10);
    if (errno || end == s.c_str() || *end != '\0' || x < INT32_MIN || x > INT32_MAX) return false;
    *v = (int)x;
    return true;
}

bool to_real(std::string s, float* v) {
    for (char& ch : s)
        if (ch == 'd' || ch == 'D') ch = 'e';  // Fortran double-precision exponent
    errno = 0;
    char* end = nullptr;
    const float x = std::strtof(s.c_str(), &end);  // correctly rounded to single precision
    if (end == s.c_str() || *end != '\0') return false;
    *v = x;
    return true;
}

// Records of a text file (the last one may lack its newline).
bool read_records(const char* path, std::vector<std::string>* recs) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::string cur;
    int ch;
    bool any = false;
    while ((ch = std::fgetc(f)) != EOF) {
        any = true;
        if (ch == '\n') {
            if (!cur.empty() && cur.back() == '\r') cur.pop_back();
            recs->push_back(cur);
            cur.clear();
            any = false;
        } else {
            cur.push_back((char)ch);
        }
    }
    if (any) recs->push_back(cur);
    std::fclose(f);
    return true;
}

// y2 at x2 from (x1, y1) (linear_interpolation_1D, linear_interpolation.f90:
// 79-117): held constant outside [x1(1), x1(n1)]; inside, the first interval
// containing the point whose two end values are both non-zero, else 0.
void linear_1d(const float* x1, const float* y1, int n1, long s1, const float* x2, float* y2, int n2, long s2) {
    for (int j = 0; j < n2; ++j) {
        const float a3 = x2[j];
        float v = 0.f;
        if (a3 <= x1[0]) {
            v = y1[0];
        } else if (a3 >= x1[n1 - 1]) {
            v = y1[(long)(n1 - 1) * s1];
        } else {
            for (int i = 0; i < n1 - 1; ++i) {
                const float a1 = x1[i + 1], a2 = x1[i];
                const float b1 = y1[(long)(i + 1) * s1], b2 = y1[(long)i * s1];
                if (a3 >= a2 && a3 <= a1 && std::fabs(b1) > 0.f && std::fabs(b2) > 0.f) {
                    const float m = (b1 - b2) / (a1 - a2);
                    v = b2 + (a3 - a2) * m;
                    break;
                }
            }
        }
        y2[(long)j * s2] = v;
    }
}

}  // namespace

extern "C" {

int psdm_nav_read(const char* path, int32_t cols, int32_t dir_boat, float d_shot_model, int32_t shot_i,
                  int32_t shot_f, int32_t max_lines, int32_t* shotID, float* pos_shot, float* pos_bat,
                  int32_t* out) {
    if (!path || !out) return fail_arg("psdm_nav_read: null argument");
    if (cols != 11 && cols != 111 && cols != 1111)
        return fail_arg("psdm_nav_read: cols must be 11 (shot x), 111 (shot x y) or 1111 (shot x y depth)");
    if (dir_boat != 1 && dir_boat != -1) return fail_arg("psdm_nav_read: dir_boat must be 1 or -1");
    std::vector<std::string> recs;
    if (!read_records(path, &recs)) return fail_arg(std::string("psdm_nav_read: cannot open ") + path);
    const int nlines = (int)recs.size();
    out[0] = nlines;
    out[1] = out[2] = 0;
    if (nlines == 0) return fail_arg("psdm_nav_read: empty navigation file");
    if (nlines > max_lines || !shotID || !pos_shot || !pos_bat)
        return fail_arg("psdm_nav_read: output arrays hold fewer entries than the file's " + std::to_string(nlines) +
                        " records (out[0])");
    const int nval = cols == 11 ? 2 : (cols == 111 ? 3 : 4);
    std::vector<int> id(nlines);
    std::vector<float> xs(nlines, 0.f), ys(nlines, 0.f), bat(nlines, 0.f);
    for (int k = 0; k < nlines; ++k) {
        const std::vector<std::string> f = fields(recs[k]);
        bool ok = (int)f.size() >= nval && to_int(f[0], &id[k]) && to_real(f[1], &xs[k]);
        if (ok && nval >= 3) ok = to_real(f[2], &ys[k]);
        if (ok && nval >= 4) ok = to_real(f[3], &bat[k]);
        if (!ok)
            return fail_arg("psdm_nav_read: record " + std::to_string(k + 1) + " does not hold " +
                            std::to_string(nval) + " values (shot number, then reals)");
    }
    // Origin of the line: the first shot when the boat moves to +x, the last
    // otherwise (get_mcs_data.f90:68-78).
    const int o = dir_boat == 1 ? 0 : nlines - 1;
    const float x1 = xs[o], y1 = ys[o];
    if (shot_i == 0) shot_i = id[0];
    if (shot_f == 0) shot_f = id[nlines - 1];
    int line_i = 0, line_f = 0;
    for (int k = 0; k < nlines; ++k) {  // the last record with the number wins
        if (shot_i > 0 && id[k] == shot_i) line_i = k + 1;
        if (shot_f > 0 && id[k] == shot_f) line_f = k + 1;
    }
    for (int k = 0; k < nlines; ++k) {
        shotID[k] = id[k];
        const float dx = xs[k] - x1, dy = ys[k] - y1;
        pos_shot[k] = d_shot_model + std::sqrt(dx * dx + dy * dy);
        pos_bat[k] = std::fabs(bat[k]);
    }
    out[1] = line_i;
    out[2] = line_f;
    if (line_i == 0) return fail_arg("psdm_nav_read: first shot " + std::to_string(shot_i) + " not found");
    if (line_f == 0) return fail_arg("psdm_nav_read: last shot " + std::to_string(shot_f) + " not found");
    return PSDM_OK;
}

int psdm_channel_positions(float pos_shot, int32_t NumRec, int32_t dir_boat, int32_t offset_header,
                           float offset_unit, const int32_t* offsets, float near_offset, float drec,
                           float* pos_rec) {
    if (NumRec < 0 || !pos_rec) return fail_arg("psdm_channel_positions: null output or negative NumRec");
    const float dir = (float)dir_boat;
    if (offset_header == 1) {
        if (!offsets) return fail_arg("psdm_channel_positions: offset_header = 1 needs the header offsets");
        if (!(offset_unit != 0.f))
            return fail_arg("psdm_channel_positions: offset_unit must be > 0 (multiply) or < 0 (divide)");
        for (int i = 0; i < NumRec; ++i) {
            const float a = (float)std::abs((long)offsets[i]);
            const float off = offset_unit > 0.f ? a * offset_unit : a / std::fabs(offset_unit);
            pos_rec[i] = pos_shot - dir * off;
        }
        return PSDM_OK;
    }
    if (offset_header != 0) return fail_arg("psdm_channel_positions: offset_header must be 0 or 1");
    for (int i = 0; i < NumRec; ++i) pos_rec[i] = pos_shot - dir * (near_offset + (float)i * drec);
    return PSDM_OK;
}

int psdm_geometry_mcs(float pos_shot, int32_t NumRec, const float* pos_rec, float shot_depth, float streamer_depth,
                      float dd, int32_t* nxSou, int32_t* nySou, int32_t* nxRec, int32_t* nyRec) {
    if (!nxSou || !nySou || NumRec < 0 || (NumRec > 0 && (!pos_rec || !nxRec || !nyRec)) || !(dd > 0.f))
        return fail_arg("psdm_geometry_mcs: null argument, negative NumRec or dd <= 0");
    *nxSou = 1 + (int)std::floor(pos_shot / dd);
    *nySou = 1 + (int)std::floor(shot_depth / dd);
    const int ny = 1 + (int)std::floor(streamer_depth / dd);
    for (int i = 0; i < NumRec; ++i) {
        nxRec[i] = 1 + (int)std::floor(pos_rec[i] / dd);
        nyRec[i] = ny;
    }
    return PSDM_OK;
}

int psdm_linear_2d(int32_t nxmodel, int32_t nymodel, float dmodel, const float* vel, int32_t nx_prop,
                   int32_t ny_prop, float dmodel_prop, float* Vpmodel) {
    if (!vel || !Vpmodel || nxmodel < 1 || nymodel < 1 || nx_prop < 1 || ny_prop < 1)
        return fail_arg("psdm_linear_2d: null argument or empty grid");
    std::vector<float> xm(nxmodel), ym(nymodel), xp(nx_prop), yp(ny_prop);
    for (int i = 0; i < nxmodel; ++i) xm[i] = (float)i * dmodel;
    for (int i = 0; i < nymodel; ++i) ym[i] = (float)i * dmodel;
    for (int i = 0; i < nx_prop; ++i) xp[i] = (float)i * dmodel_prop;
    for (int i = 0; i < ny_prop; ++i) yp[i] = (float)i * dmodel_prop;
    // depth first, column by column, then along x row by row (linear_2D)
    std::vector<float> tmp((size_t)ny_prop * nxmodel);
    for (int i = 0; i < nxmodel; ++i)
        linear_1d(ym.data(), vel + (size_t)i * nymodel, nymodel, 1, yp.data(), tmp.data() + (size_t)i * ny_prop,
                  ny_prop, 1);
    for (int j = 0; j < ny_prop; ++j)
        linear_1d(xm.data(), tmp.data() + j, nxmodel, ny_prop, xp.data(), Vpmodel + j, nx_prop, ny_prop);
    return PSDM_OK;
}

int psdm_batmodel_from_velocity(int32_t nx_prop, int32_t ny_prop, float dmodel_prop, float water_velocity,
                                const float* Vpmodel, float* Batmodel) {
    if (!Vpmodel || !Batmodel || nx_prop < 1 || ny_prop < 1)
        return fail_arg("psdm_batmodel_from_velocity: null argument or empty grid");
    for (int i = 0; i < nx_prop; ++i) {
        Batmodel[i] = 0.f;
        const float* col = Vpmodel + (size_t)i * ny_prop;
        for (int j = 0; j < ny_prop; ++j)
            if (col[j] > water_velocity) {
                Batmodel[i] = (float)(j - 1) * dmodel_prop;  // (j-1-1)*dmodel_prop with 1-based j
                break;
            }
    }
    return PSDM_OK;
}

}  // extern "C"
