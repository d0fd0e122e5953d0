// Dispersion sets on the host: the text dispersion file of ModBB --dispersion
// read the way ModalBroadbandPropagator::read_dispersion_file does
// (ModalBroadbandPropagator.cpp:98-138), and a binary cache of the parsed
// arrays so repeated propagation runs skip the text parsing.
//
// Cache layout (native byte order), stamped with the text file it was made
// from (size, modification time, FNV-1a 64 hash of its bytes):
//   char magic[8] = "NCPADSP1"
//   uint64 text_size; int64 text_mtime_ns; uint64 text_hash
//   int32 n_freq (DC slot included); int32 n_modes; int32 text_rows; int32 0
//   double rho_src, rho_rcv
//   double f[n_freq]; int32 mode_off[n_freq + 1] (+ 4 bytes when n_freq is even)
//   double re_k[n_modes], im_k[n_modes], v_src[n_modes], v_rcv[n_modes]
#include <sys/stat.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "ncpa_gpu.h"

struct ncpa_dispersion {
    std::vector<double> f{0.0};  // DC slot first
    std::vector<int> off{0, 0};
    std::vector<double> kr, ki, vs, vr;
    double rho_src = 1.0, rho_rcv = 1.0;
    int text_rows = 0;  // newline characters of the text file
    int from_cache = 0;
};

namespace {

constexpr char kMagic[8] = {'N', 'C', 'P', 'A', 'D', 'S', 'P', '1'};
constexpr int kMaxModes = 4000;  // the reference's mode arrays (ModalBroadbandPropagator.cpp:33-36)

struct Stamp {
    uint64_t size = 0;
    int64_t mtime_ns = 0;
    uint64_t hash = 0;
};

// size, modification time and FNV-1a 64 hash of a file; newline count too
bool stamp_file(const char* path, Stamp& s, int& newlines) {
    struct stat st;
    if (stat(path, &st) != 0) return false;
    s.size = (uint64_t)st.st_size;
    s.mtime_ns = (int64_t)st.st_mtim.tv_sec * 1000000000LL + (int64_t)st.st_mtim.tv_nsec;
    std::FILE* fp = std::fopen(path, "rb");
    if (!fp) return false;
    uint64_t h = 1469598103934665603ull;
    newlines = 0;
    unsigned char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, fp)) > 0) {
        for (size_t i = 0; i < n; ++i) {
            h = (h ^ buf[i]) * 1099511628211ull;
            newlines += buf[i] == '\n';
        }
    }
    std::fclose(fp);
    s.hash = h;
    return true;
}

// text parse: lines "f M rho_src rho_rcv" followed by M quadruples
// (Re k, Im k, V_src, V_rcv); the densities of the last line are kept
bool parse_text(const char* path, ncpa_dispersion& d) {
    std::FILE* fp = std::fopen(path, "r");
    if (!fp) return false;
    double fr;
    while (std::fscanf(fp, "%lf", &fr) == 1) {
        int m = 0;
        if (std::fscanf(fp, "%d", &m) != 1 || std::fscanf(fp, "%lf", &d.rho_src) != 1 ||
            std::fscanf(fp, "%lf", &d.rho_rcv) != 1 || m < 0 || m > kMaxModes) {
            std::fclose(fp);
            return false;
        }
        for (int j = 0; j < m; ++j) {
            double x1, x2, y1, y2;
            if (std::fscanf(fp, "%lf %lf %lf %lf", &x1, &x2, &y1, &y2) != 4) {
                std::fclose(fp);
                return false;
            }
            d.kr.push_back(x1);
            d.ki.push_back(x2);
            d.vs.push_back(y1);
            d.vr.push_back(y2);
        }
        d.f.push_back(fr);
        d.off.push_back((int)d.kr.size());
    }
    std::fclose(fp);  // like the reference, reading stops at the first token that is not a number
    return true;
}

template <class T>
bool rd(std::FILE* fp, T* p, size_t n) {
    return n == 0 || std::fread(p, sizeof(T), n, fp) == n;
}
template <class T>
bool wr(std::FILE* fp, const T* p, size_t n) {
    return n == 0 || std::fwrite(p, sizeof(T), n, fp) == n;
}

// reads a cache whose stamp equals s; false (and no change to d) otherwise
bool read_cache(const char* path, const Stamp& s, ncpa_dispersion& d) {
    std::FILE* fp = std::fopen(path, "rb");
    if (!fp) return false;
    char magic[8];
    Stamp c;
    int32_t hdr[4];
    double rho[2];
    bool ok = rd(fp, magic, 8) && std::memcmp(magic, kMagic, 8) == 0 && rd(fp, &c.size, 1) &&
              rd(fp, &c.mtime_ns, 1) && rd(fp, &c.hash, 1) && c.size == s.size && c.mtime_ns == s.mtime_ns &&
              c.hash == s.hash && rd(fp, hdr, 4) && rd(fp, rho, 2);
    const int nf = ok ? hdr[0] : 0, nm = ok ? hdr[1] : 0;
    ok = ok && nf >= 1 && nm >= 0 && nm <= kMaxModes * nf;
    ncpa_dispersion t;
    if (ok) {
        t.f.resize(nf);
        t.off.resize(nf + 1);
        t.kr.resize(nm);
        t.ki.resize(nm);
        t.vs.resize(nm);
        t.vr.resize(nm);
        int32_t pad = 0;
        ok = rd(fp, t.f.data(), nf) && rd(fp, t.off.data(), nf + 1) && ((nf + 1) % 2 == 0 || rd(fp, &pad, 1)) &&
             rd(fp, t.kr.data(), nm) && rd(fp, t.ki.data(), nm) && rd(fp, t.vs.data(), nm) &&
             rd(fp, t.vr.data(), nm);
        char extra;
        ok = ok && std::fread(&extra, 1, 1, fp) == 0;  // nothing after the arrays
    }
    std::fclose(fp);
    if (!ok) return false;
    if (t.off[0] != 0 || t.off[nf] != nm) return false;
    for (int i = 0; i < nf; ++i)
        if (t.off[i + 1] < t.off[i] || t.off[i + 1] - t.off[i] > kMaxModes) return false;
    t.rho_src = rho[0];
    t.rho_rcv = rho[1];
    t.text_rows = hdr[2];
    t.from_cache = 1;
    d = std::move(t);
    return true;
}

bool write_cache(const char* path, const Stamp& s, const ncpa_dispersion& d) {
    const std::string tmp = std::string(path) + ".tmp";
    std::FILE* fp = std::fopen(tmp.c_str(), "wb");
    if (!fp) return false;
    const int32_t nf = (int32_t)d.f.size(), nm = (int32_t)d.kr.size();
    const int32_t hdr[4] = {nf, nm, d.text_rows, 0};
    const double rho[2] = {d.rho_src, d.rho_rcv};
    const int32_t pad = 0;
    bool ok = wr(fp, kMagic, 8) && wr(fp, &s.size, 1) && wr(fp, &s.mtime_ns, 1) && wr(fp, &s.hash, 1) &&
              wr(fp, hdr, 4) && wr(fp, rho, 2) && wr(fp, d.f.data(), nf) && wr(fp, d.off.data(), nf + 1) &&
              ((nf + 1) % 2 == 0 || wr(fp, &pad, 1)) && wr(fp, d.kr.data(), nm) && wr(fp, d.ki.data(), nm) &&
              wr(fp, d.vs.data(), nm) && wr(fp, d.vr.data(), nm);
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok || std::rename(tmp.c_str(), path) != 0) {
        std::remove(tmp.c_str());
        return false;
    }
    return true;
}

}  // namespace

extern "C" {

ncpa_status ncpa_dispersion_read(const char* text_path, const char* cache_path, ncpa_dispersion** out) {
    if (!text_path || !out) return NCPA_EINVAL;
    *out = nullptr;
    try {
        auto d = std::make_unique<ncpa_dispersion>();
        Stamp s;
        int rows = 0;
        if (!stamp_file(text_path, s, rows)) return NCPA_EPARSE;
        if (cache_path && read_cache(cache_path, s, *d)) {
            *out = d.release();
            return NCPA_OK;
        }
        if (!parse_text(text_path, *d)) return NCPA_EPARSE;
        d->text_rows = rows;
        if (cache_path && !write_cache(cache_path, s, *d)) return NCPA_EINVAL;
        *out = d.release();
        return NCPA_OK;
    } catch (const std::bad_alloc&) {
        return NCPA_ENOMEM;
    }
}

ncpa_status ncpa_dispersion_desc_get(const ncpa_dispersion* d, ncpa_dispersion_desc* desc, int* text_rows,
                                     int* from_cache) {
    if (!d) return NCPA_EINVAL;
    if (desc) {
        desc->n_freq = (int)d->f.size();
        desc->f = d->f.data();
        desc->mode_off = d->off.data();
        desc->re_k = d->kr.data();
        desc->im_k = d->ki.data();
        desc->v_src = d->vs.data();
        desc->v_rcv = d->vr.data();
        desc->rho_src = d->rho_src;
        desc->rho_rcv = d->rho_rcv;
    }
    if (text_rows) *text_rows = d->text_rows;
    if (from_cache) *from_cache = d->from_cache;
    return NCPA_OK;
}

ncpa_status ncpa_dispersion_destroy(ncpa_dispersion* d) {
    if (!d) return NCPA_EINVAL;
    delete d;
    return NCPA_OK;
}

}  // extern "C"
