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
// and for wide-angle (OBS) data, where by reciprocity the OBSs act as sources
// and the shots as receivers:
//   psdm_nav_read_was        read_nav_shot_was   src/get_was_data.f90:70-125
//   psdm_nav_read_obs        read_nav_obs        src/get_was_data.f90:127-160
//   psdm_geometry_was        get_geometry_WAS    src/get_was_data.f90:162-189
//   psdm_bathymetry_nav      get_bathymetry_model_was / _mcs
//                                                src/get_was_data.f90:500-549
//   psdm_relocate_obs        relocation_zOBS     src/get_was_data.f90:30-68
// The navigation files are read as Fortran list-directed input: one record
// per line, values separated by blanks or commas, reals in any Fortran form
// (including a D exponent).  The bathymetry along the line is Akima's local
// cubic through the shots (Akima, J. ACM 17 (1970) 589-602), written here
// from the paper; the reference calls a vendored TOMS-433 routine (INTRPL).

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

// Parse the first `nrec` records with nval values each (an integer, then
// reals) into id / v[0..nval-2].
int parse_records(const char* path, const char* who, int nrec, int nval, std::vector<int>* id,
                  std::vector<std::vector<float>>* v) {
    std::vector<std::string> recs;
    if (!read_records(path, &recs)) return fail_arg(std::string(who) + ": cannot open " + path);
    if ((int)recs.size() < nrec)
        return fail_arg(std::string(who) + ": the file holds " + std::to_string(recs.size()) + " records, " +
                        std::to_string(nrec) + " expected");
    id->assign(nrec, 0);
    v->assign(nval - 1, std::vector<float>(nrec, 0.f));
    for (int k = 0; k < nrec; ++k) {
        const std::vector<std::string> f = fields(recs[k]);
        bool ok = (int)f.size() >= nval && to_int(f[0], &(*id)[k]);
        for (int q = 1; ok && q < nval; ++q) ok = to_real(f[q], &(*v)[q - 1][k]);
        if (!ok)
            return fail_arg(std::string(who) + ": record " + std::to_string(k + 1) + " does not hold " +
                            std::to_string(nval) + " values (a number, then reals)");
    }
    return PSDM_OK;
}

// Akima's interpolant through (x[i], y[i]), x strictly increasing, n >= 2.
// Segment slopes m_i are extended by two on each side (m_{-1} = 2 m_0 - m_1,
// ...), node slopes t_i weight m_{i-1} and m_i by |m_{i+1} - m_i| and
// |m_{i-1} - m_{i-2}| (their mean where both weights vanish), and each
// interval is the cubic with the end values and slopes; outside [x_0,
// x_{n-1}] the end intervals' cubics continue.
struct Akima {
    const float *x, *y;
    int n;
    std::vector<float> M, t;  // M[k + 2] = m_k, k = -2 .. n
    Akima(const float* x_, const float* y_, int n_) : x(x_), y(y_), n(n_), M(n_ + 3), t(n_) {
        for (int i = 0; i + 1 < n; ++i) M[i + 2] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]);
        if (n == 2) {
            M[0] = M[1] = M[3] = M[4] = M[2];
        } else {
            M[1] = 2.f * M[2] - M[3];
            M[0] = 2.f * M[1] - M[2];
            M[n + 1] = 2.f * M[n] - M[n - 1];
            M[n + 2] = 2.f * M[n + 1] - M[n];
        }
        for (int i = 0; i < n; ++i) {
            const float w1 = std::fabs(M[i + 3] - M[i + 2]), w2 = std::fabs(M[i + 1] - M[i]);
            const float w = w1 + w2;
            t[i] = w == 0.f ? (M[i + 1] + M[i + 2]) * 0.5f : (w1 * M[i + 1] + w2 * M[i + 2]) / w;
        }
    }
    float operator()(float u) const {
        if (u == x[n - 1]) return y[n - 1];
        int i = 0;
        if (u >= x[n - 1]) {
            i = n - 2;
        } else if (u > x[0]) {
            int lo = 0, hi = n - 1;  // x[lo] <= u < x[hi]
            while (hi - lo > 1) {
                const int mid = (lo + hi) / 2;
                if (x[mid] <= u) lo = mid; else hi = mid;
            }
            i = lo;
        }
        const float h = x[i + 1] - x[i], d = u - x[i], m = M[i + 2], t0 = t[i], t1 = t[i + 1];
        const float c2 = (3.f * m - 2.f * t0 - t1) / h;
        const float c3 = (t0 + t1 - 2.f * m) / (h * h);
        return y[i] + d * (t0 + d * (c2 + d * c3));
    }
};

}  // namespace

extern "C" {

int psdm_nav_read_was(const char* path, int32_t cols, int32_t NumShots, float d_shot_model, float added_space,
                      float dmodel, int32_t shot_i, int32_t shot_f, int32_t* shotID, float* pos_shot, float* pos_bat,
                      int32_t* out_i, float* out_f) {
    if (!path || !shotID || !pos_shot || !pos_bat || !out_i || !out_f || NumShots < 1 || !(dmodel > 0.f))
        return fail_arg("psdm_nav_read_was: null argument, NumShots < 1 or dmodel <= 0");
    if (cols != 11 && cols != 111 && cols != 1111)
        return fail_arg("psdm_nav_read_was: cols must be 11 (shot x), 111 (shot x y) or 1111 (shot x y depth)");
    const int nval = cols == 11 ? 2 : (cols == 111 ? 3 : 4);
    std::vector<int> id;
    std::vector<std::vector<float>> v;
    const int rc = parse_records(path, "psdm_nav_read_was", NumShots, nval, &id, &v);
    if (rc) return rc;
    const std::vector<float> zero(NumShots, 0.f);
    const std::vector<float>& xs = v[0];
    const std::vector<float>& ys = nval >= 3 ? v[1] : zero;
    const std::vector<float>& bat = nval >= 4 ? v[2] : zero;
    const float x1 = xs[0], y1 = ys[0];  // the first shot is the origin
    int line_i = 0, line_f = 0;
    for (int k = 0; k < NumShots; ++k) {
        shotID[k] = id[k];
        const float dx = xs[k] - x1, dy = ys[k] - y1;
        pos_shot[k] = d_shot_model + std::sqrt(dx * dx + dy * dy);
        pos_bat[k] = std::fabs(bat[k]);
        if (shot_i == id[k]) line_i = k + 1;
        if (shot_f == id[k]) line_f = k + 1;
    }
    const float xn = xs[NumShots - 1];
    const float length = xn + 2.f * added_space;  // from the last shot's coordinate
    out_f[0] = std::fabs(xn - x1) / (float)(NumShots - 1);
    out_f[1] = length;
    out_i[0] = line_i;
    out_i[1] = line_f;
    out_i[2] = 1 + (int)std::ceil(length / dmodel);
    return PSDM_OK;
}

int psdm_nav_read_obs(const char* path, int32_t NumOBS, float dmodel, int32_t* obsID, float* pos_xobs,
                      float* pos_zobs, int32_t* xgrid, int32_t* zgrid) {
    if (!path || !obsID || !pos_xobs || !pos_zobs || !xgrid || !zgrid || NumOBS < 1 || !(dmodel > 0.f))
        return fail_arg("psdm_nav_read_obs: null argument, NumOBS < 1 or dmodel <= 0");
    std::vector<int> id;
    std::vector<std::vector<float>> v;
    const int rc = parse_records(path, "psdm_nav_read_obs", NumOBS, 3, &id, &v);
    if (rc) return rc;
    for (int i = 0; i < NumOBS; ++i) {
        obsID[i] = id[i];
        pos_xobs[i] = std::fabs(v[0][i]);
        xgrid[i] = 1 + (int)std::ceil(pos_xobs[i] / dmodel);
        pos_zobs[i] = std::fabs(v[1][i]);
        zgrid[i] = 1 + (int)std::ceil(pos_zobs[i] / dmodel);
    }
    return PSDM_OK;
}

int psdm_geometry_was(int32_t xobs_grid, int32_t zobs_grid, int32_t NumRec, const float* pos_shot, float shot_depth,
                      float dd, int32_t* nxSou, int32_t* nySou, int32_t* nxRec, int32_t* nyRec) {
    if (!nxSou || !nySou || NumRec < 0 || (NumRec > 0 && (!pos_shot || !nxRec || !nyRec)) || !(dd > 0.f))
        return fail_arg("psdm_geometry_was: null argument, negative NumRec or dd <= 0");
    *nxSou = xobs_grid;  // the OBS is the source
    *nySou = zobs_grid;
    const int ny = 1 + (int)std::ceil(shot_depth / dd);
    for (int i = 0; i < NumRec; ++i) {  // the shots are the receivers
        nxRec[i] = 1 + (int)std::ceil(pos_shot[i] / dd);
        nyRec[i] = ny;
    }
    return PSDM_OK;
}

int psdm_bathymetry_nav(int32_t NumShots, const float* pos_shot, const float* pos_bat, float length_model,
                        int32_t nxmodel, float dmodel, float* bat_model) {
    if (!pos_shot || !pos_bat || !bat_model || NumShots < 1 || nxmodel < 1)
        return fail_arg("psdm_bathymetry_nav: null argument or empty input");
    // nodes: x = 0 and length_model hold the first and last shots' depths
    const int n = NumShots + 2;
    std::vector<float> x(n), y(n);
    x[0] = 0.f;
    y[0] = pos_bat[0];
    for (int i = 0; i < NumShots; ++i) {
        x[i + 1] = pos_shot[i];
        y[i + 1] = pos_bat[i];
    }
    x[n - 1] = length_model;
    y[n - 1] = pos_bat[NumShots - 1];
    for (int i = 1; i < n; ++i)
        if (!(x[i] > x[i - 1]))
            return fail_arg("psdm_bathymetry_nav: shot positions must increase strictly within (0, length_model)");
    const Akima ak(x.data(), y.data(), n);
    for (int i = 0; i < nxmodel; ++i) bat_model[i] = ak((float)i * dmodel);
    return PSDM_OK;
}

int psdm_relocate_obs(int32_t NumOBS, const int32_t* xgrid, const float* bat_model, int32_t nxmodel, float dmodel,
                      float* pos_zobs, int32_t* zgrid) {
    if (!xgrid || !bat_model || !pos_zobs || !zgrid || NumOBS < 0 || !(dmodel > 0.f))
        return fail_arg("psdm_relocate_obs: null argument, negative NumOBS or dmodel <= 0");
    for (int i = 0; i < NumOBS; ++i)
        if (xgrid[i] < 1 || xgrid[i] > nxmodel)
            return fail_arg("psdm_relocate_obs: OBS " + std::to_string(i + 1) + " lies outside the model");
    for (int i = 0; i < NumOBS; ++i) {
        pos_zobs[i] = bat_model[xgrid[i] - 1];  // the sea floor under the OBS
        zgrid[i] = 1 + (int)std::ceil(pos_zobs[i] / dmodel);
    }
    return PSDM_OK;
}


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
