// SU (Seismic Unix) trace files without the SU tools.
//
// The reference writes its images (PSDM_RTM.su, Velocity.su) by piping an
// ASCII dump through a2b | suaddhead | sushw | suchw (src/auxiliar.f90:
// 275-353, write_psdm; :180-221, write_vel), tools that are not installed
// here, and reads shot gathers as fixed-length traces with direct access
// (src/get_mcs_data.f90:150-214, get_shot_data; :440-500 for the header
// words).  This file does both natively.
//
// Trace layout (the SEG-Y/SU trace header, 240 bytes, then ns samples of
// 4-byte floats); the fields written here and their byte offsets:
//   tracl int32 @0, tracr int32 @4, cdp int32 @20, trid int16 @28,
//   ns uint16 @114, d1 float @180, f1 float @184, d2 float @188, f2 float @192.
// Byte order: the machine's (little-endian here) or big-endian on request,
// as the reference's endianness_data switch (get_mcs_data.f90:304-311).

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/psdm_rtm.h"
#include "rtm_internal.h"

namespace {

constexpr int kHeaderBytes = 240;

uint32_t bswap32(uint32_t v) { return (v >> 24) | ((v >> 8) & 0xff00u) | ((v << 8) & 0xff0000u) | (v << 24); }
uint16_t bswap16(uint16_t v) { return (uint16_t)((v >> 8) | (v << 8)); }

void put32(unsigned char* h, int off, uint32_t v, bool big) {
    if (big) v = bswap32(v);
    std::memcpy(h + off, &v, 4);
}
void put16(unsigned char* h, int off, uint16_t v, bool big) {
    if (big) v = bswap16(v);
    std::memcpy(h + off, &v, 2);
}
uint32_t fbits(float f) {
    uint32_t b;
    std::memcpy(&b, &f, 4);
    return b;
}

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

}  // namespace

extern "C" {

int psdm_su_write_image(const char* path, int32_t ni, int32_t nj, float di, float dj, int32_t trid,
                        const float* model, int32_t big_endian) {
    if (!path || !model || ni < 1 || nj < 1 || nj > 65535) {
        psdm::set_last_error("psdm_su_write_image: null argument or size outside 1..65535 samples");
        return PSDM_ERR_ARG;
    }
    File fh;
    fh.f = std::fopen(path, "wb");
    if (!fh.f) {
        psdm::set_last_error("psdm_su_write_image: cannot open the output file");
        return PSDM_ERR_ARG;
    }
    const bool big = big_endian != 0;
    std::vector<unsigned char> rec(kHeaderBytes + (size_t)nj * 4);
    for (int i = 0; i < ni; ++i) {
        std::memset(rec.data(), 0, kHeaderBytes);
        unsigned char* h = rec.data();
        const int tracl = i + 1;
        put32(h, 0, (uint32_t)tracl, big);                     // tracl (suaddhead)
        put32(h, 4, (uint32_t)tracl, big);                     // tracr (suaddhead)
        put32(h, 20, (uint32_t)(int32_t)(-di + di * tracl), big);  // cdp = -di + di*tracl (suchw)
        put16(h, 28, (uint16_t)(int16_t)trid, big);            // trid (sushw)
        put16(h, 114, (uint16_t)nj, big);                      // ns (suaddhead)
        put32(h, 180, fbits(dj), big);                         // d1
        put32(h, 184, fbits(0.f), big);                        // f1
        put32(h, 188, fbits(di), big);                         // d2
        put32(h, 192, fbits(0.f), big);                        // f2
        const float* col = model + (size_t)i * nj;             // model(:, i)
        for (int j = 0; j < nj; ++j) put32(rec.data() + kHeaderBytes, 4 * j, fbits(col[j]), big);
        if (std::fwrite(rec.data(), 1, rec.size(), fh.f) != rec.size()) {
            psdm::set_last_error("psdm_su_write_image: write failed");
            return PSDM_ERR_ARG;
        }
    }
    return PSDM_OK;
}

int psdm_su_read_shot(const char* path, int32_t NumRec, int32_t ns_max, int32_t nt, int32_t big_endian,
                      int32_t delay_samples, float* raw, float* delayed) {
    if (!path || !raw || NumRec < 1 || ns_max < 1 || nt < 1 || nt > ns_max) {
        psdm::set_last_error("psdm_su_read_shot: null argument or nt outside 1..ns_max");
        return PSDM_ERR_ARG;
    }
    File fh;
    fh.f = std::fopen(path, "rb");
    if (!fh.f) {
        psdm::set_last_error("psdm_su_read_shot: cannot open the input file");
        return PSDM_ERR_ARG;
    }
    const size_t rec = (size_t)kHeaderBytes + (size_t)ns_max * 4;
    std::vector<unsigned char> buf(rec);
    for (int j = 0; j < NumRec; ++j) {
        if (std::fseek(fh.f, (long)(j * rec), SEEK_SET) != 0 || std::fread(buf.data(), 1, rec, fh.f) != rec) {
            psdm::set_last_error("psdm_su_read_shot: file shorter than NumRec fixed-length traces");
            return PSDM_ERR_ARG;
        }
        float* tr = raw + (size_t)j * nt;
        for (int i = 0; i < nt; ++i) {
            uint32_t b;
            std::memcpy(&b, buf.data() + kHeaderBytes + 4 * i, 4);
            if (big_endian) b = bswap32(b);
            std::memcpy(tr + i, &b, 4);
        }
        if (delayed) {  // get_shot_data's time shift by delay_samples
            float* d = delayed + (size_t)j * nt;
            for (int i = 0; i < nt; ++i) d[i] = 0.f;
            if (delay_samples >= 0) {
                for (int i = 0; i + delay_samples < nt; ++i) d[i + delay_samples] = tr[i];
            } else {
                const int s = -delay_samples;
                for (int i = s; i < nt; ++i) d[i - s] = tr[i];
            }
        }
    }
    return PSDM_OK;
}

int psdm_su_read_header_i32(const char* path, int32_t NumRec, int32_t ns_max, int32_t byte_pos, int32_t big_endian,
                            int32_t* out) {
    if (!path || !out || NumRec < 1 || ns_max < 1 || byte_pos < 1 || byte_pos > kHeaderBytes - 3) {
        psdm::set_last_error("psdm_su_read_header_i32: null argument or byte position outside the header");
        return PSDM_ERR_ARG;
    }
    File fh;
    fh.f = std::fopen(path, "rb");
    if (!fh.f) {
        psdm::set_last_error("psdm_su_read_header_i32: cannot open the input file");
        return PSDM_ERR_ARG;
    }
    const size_t rec = (size_t)kHeaderBytes + (size_t)ns_max * 4;
    for (int j = 0; j < NumRec; ++j) {
        uint32_t b;
        if (std::fseek(fh.f, (long)(j * rec + (byte_pos - 1)), SEEK_SET) != 0 || std::fread(&b, 1, 4, fh.f) != 4) {
            psdm::set_last_error("psdm_su_read_header_i32: file shorter than NumRec fixed-length traces");
            return PSDM_ERR_ARG;
        }
        if (big_endian) b = bswap32(b);
        std::memcpy(out + j, &b, 4);
    }
    return PSDM_OK;
}

}  // extern "C"
