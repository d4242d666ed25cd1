// readers.cpp -- the model's input files read on the host: bathymetry
// (.md and XBeach .dep grids), sea-level and wind series, wave-boundary
// parameter series (constant and JONSWAP records) and XBeach "reuse"
// boundary files (a list of binary q / E record files), with the reference's
// file formats and tokenisation (read_input.cpp:25-593, 1476-1635).
//
// Line tokens: split on tabs (empty tokens skipped); when a line has fewer
// tokens than the format needs, on spaces; then on commas; still fewer is a
// format error (the reference exits there).  Numbers are parsed like
// std::stod / std::stoi (leading blanks, longest valid prefix).  Values the
// reference stores in float (grids, the binary boundary records) are rounded
// to float as it does.  Errors return a status; nothing exits.
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cctype>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/xbg_io.h"

namespace {

const double PI_REF = 3.14159265;   // the reference's pi macro

std::vector<std::string> split_skip(const std::string& s, char d) {
    std::vector<std::string> out;
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, d))
        if (!item.empty()) out.push_back(item);
    return out;
}

bool tokens(const std::string& line, size_t need, std::vector<std::string>& t) {
    t = split_skip(line, '\t');
    if (t.size() < need) t = split_skip(line, ' ');
    if (t.size() < need) t = split_skip(line, ',');
    return t.size() >= need;
}

bool num(const std::string& s, double& v) {
    const char* p = s.c_str();
    char* end = nullptr;
    errno = 0;
    v = std::strtod(p, &end);
    return end != p && errno != ERANGE;
}

bool inum(const std::string& s, int& v) {
    const char* p = s.c_str();
    char* end = nullptr;
    errno = 0;
    long x = std::strtol(p, &end, 10);
    if (end == p || errno == ERANGE || x < INT32_MIN || x > INT32_MAX) return false;
    v = (int)x;
    return true;
}

// whitespace-separated tokens of a whole file (the fscanf-based readers)
struct Scan {
    FILE* fp = nullptr;
    explicit Scan(const char* path) { fp = std::fopen(path, "r"); }
    ~Scan() { if (fp) std::fclose(fp); }
    bool word(std::string& w) {
        w.clear();
        int c;
        while ((c = std::fgetc(fp)) != EOF && std::isspace(c)) {}
        if (c == EOF) return false;
        do { w.push_back((char)c); } while ((c = std::fgetc(fp)) != EOF && !std::isspace(c));
        return true;
    }
    bool f32(float& v) {
        std::string w;
        if (!word(w)) return false;
        const char* p = w.c_str();
        char* end = nullptr;
        v = std::strtof(p, &end);
        return end != p;
    }
    bool d64(double& v) {
        std::string w;
        return word(w) && num(w, v);
    }
    bool u32(long& v) {
        std::string w;
        if (!word(w)) return false;
        const char* p = w.c_str();
        char* end = nullptr;
        v = std::strtol(p, &end, 10);
        return end != p;
    }
};

int read_lines(const char* path, std::vector<std::string>& lines) {
    std::ifstream fs(path);
    if (fs.fail()) return XBG_ERR_IO;
    std::string line;
    while (std::getline(fs, line)) lines.push_back(line);
    return XBG_OK;
}

}  // namespace

extern "C" int xbg_read_table(const char* path, int kind, double grdalpha, double rtlength, double* out, int cap,
                              int* nrec, int* ncol) {
    if (!path || !nrec || kind < XBG_TAB_SEALEVEL || kind > XBG_TAB_JONSWAP) return XBG_ERR_ARG;
    static const int need[4] = {2, 3, 5, 6};     // tokens a line must have
    static const int cols[4] = {3, 6, 5, 6};     // values returned per record
    const bool comments = kind == XBG_TAB_SEALEVEL || kind == XBG_TAB_WIND;   // '#' lines skipped
    std::vector<std::string> lines;
    int rc = read_lines(path, lines);
    if (rc) return rc;
    std::vector<double> rows;
    std::vector<std::string> t;
    double last[6] = {0, 0, 0, 0, 0, 3.3};
    for (const std::string& line : lines) {
        if (line.empty() || (comments && line[0] == '#')) continue;
        if (!tokens(line, need[kind], t)) return XBG_ERR_FORMAT;
        double v[6] = {0, 0, 0, 0, 0, 3.3};
        for (int k = 0; k < need[kind]; k++)
            if (!num(t[k], v[k])) return XBG_ERR_FORMAT;
        double r[6];
        if (kind == XBG_TAB_SEALEVEL) {               // readWLfile: wlev1 = wlev0 without a third column
            r[0] = v[0]; r[1] = v[1]; r[2] = v[1];
            double w1;
            if (t.size() > 2) { if (!num(t[2], w1)) return XBG_ERR_FORMAT; r[2] = w1; }
        } else if (kind == XBG_TAB_WIND) {            // readWNDfile: direction to the grid x axis
            r[0] = v[0]; r[1] = v[1]; r[2] = v[2];
            r[3] = (1.5 * PI_REF - grdalpha) - v[2] * PI_REF / 180;
            r[4] = v[1] * std::cos(r[3]);
            r[5] = v[1] * std::sin(r[3]);
        } else {                                       // ReadCstBnd / ReadJSWPBnd
            r[0] = v[0]; r[1] = v[1]; r[2] = v[2];
            r[3] = (1.5 * PI_REF - grdalpha) - v[3] * PI_REF / 180;
            r[4] = v[4]; r[5] = v[5];
        }
        rows.insert(rows.end(), r, r + cols[kind]);
        std::memcpy(last, r, sizeof(double) * cols[kind]);
    }
    if (kind == XBG_TAB_JONSWAP) {                     // a closing record rtlength after the last
        if (rows.empty()) return XBG_ERR_FORMAT;
        last[0] += rtlength;
        rows.insert(rows.end(), last, last + cols[kind]);
    }
    *nrec = (int)(rows.size() / cols[kind]);
    if (ncol) *ncol = cols[kind];
    if (!out) return XBG_OK;
    if (cap < *nrec) return XBG_ERR_ARG;
    std::memcpy(out, rows.data(), rows.size() * sizeof(double));
    return XBG_OK;
}

extern "C" int xbg_read_md_head(const char* path, int* nx, int* ny, double* dx, double* grdalpha_deg) {
    if (!path || !nx || !ny || !dx || !grdalpha_deg) return XBG_ERR_ARG;
    std::ifstream fs(path);
    if (fs.fail()) return XBG_ERR_IO;
    std::string line;
    std::getline(fs, line);
    std::vector<std::string> t;
    if (line.empty() || !tokens(line, 5, t)) return XBG_ERR_FORMAT;
    if (!inum(t[0], *nx) || !inum(t[1], *ny) || !num(t[2], *dx) || !num(t[4], *grdalpha_deg)) return XBG_ERR_FORMAT;
    return XBG_OK;
}

extern "C" int xbg_read_md(const char* path, int nx, int ny, float* zb) {
    if (!path || nx < 1 || ny < 1 || !zb) return XBG_ERR_ARG;
    Scan s(path);
    if (!s.fp) return XBG_ERR_IO;
    long a, b;
    double c, d, e;
    if (!s.u32(a) || !s.u32(b) || !s.d64(c) || !s.d64(d) || !s.d64(e)) return XBG_ERR_FORMAT;
    if (a != nx || b != ny) return XBG_ERR_ARG;      // the grid the caller sized zb for
    for (int row = 0; row < ny; row++) {             // each row starts with its 1-based row number
        long j;
        if (!s.u32(j) || j < 1 || j > ny) return XBG_ERR_FORMAT;
        for (int i = 0; i < nx; i++)
            if (!s.f32(zb[i + (size_t)(j - 1) * nx])) return XBG_ERR_FORMAT;
    }
    return XBG_OK;
}

extern "C" int xbg_read_dep(const char* path, int nx, int ny, float* zb) {
    if (!path || nx < 1 || ny < 1 || !zb) return XBG_ERR_ARG;
    Scan s(path);
    if (!s.fp) return XBG_ERR_IO;
    for (size_t k = 0; k < (size_t)nx * ny; k++)
        if (!s.f32(zb[k])) return XBG_ERR_FORMAT;
    return XBG_OK;
}

extern "C" int xbg_read_xbbnd_head(const char* path, double* hdr) {
    if (!path || !hdr) return XBG_ERR_ARG;
    std::ifstream fs(path);
    if (fs.fail()) return XBG_ERR_IO;
    std::string line;
    std::getline(fs, line);
    std::vector<std::string> t;
    if (!tokens(line, 5, t)) return XBG_ERR_FORMAT;
    double v[5];
    for (int k = 0; k < 5; k++)
        if (!num(t[k], v[k])) return XBG_ERR_FORMAT;
    hdr[0] = v[0] * PI_REF / 180.0;    // thetamin, thetamax, dtheta in radians
    hdr[1] = v[1] * PI_REF / 180.0;
    hdr[2] = v[2] * PI_REF / 180.0;
    hdr[3] = v[3];                     // dtbc
    hdr[4] = v[4];                     // rtlength
    return XBG_OK;
}

// the entries below the header: time, Trep, q file, E file
static int xb_entries(const char* path, std::vector<double>& time, std::vector<double>& trep,
                      std::vector<std::string>& qf, std::vector<std::string>& ef) {
    std::vector<std::string> lines;
    int rc = read_lines(path, lines);
    if (rc) return rc;
    std::vector<std::string> t;
    for (size_t n = 1; n < lines.size(); n++) {
        if (lines[n].empty()) continue;
        if (!tokens(lines[n], 4, t)) return XBG_ERR_FORMAT;
        double a, b;
        if (!num(t[0], a) || !num(t[1], b)) return XBG_ERR_FORMAT;
        time.push_back(a); trep.push_back(b); qf.push_back(t[2]); ef.push_back(t[3]);
    }
    return time.empty() ? XBG_ERR_FORMAT : XBG_OK;
}

extern "C" int xbg_read_xbbnd_list(const char* path, double rtlength, double* time, double* Trep, int cap,
                                   int* nrec) {
    if (!path || !nrec) return XBG_ERR_ARG;
    std::vector<double> tm, tr;
    std::vector<std::string> qf, ef;
    int rc = xb_entries(path, tm, tr, qf, ef);
    if (rc) return rc;
    tm.push_back(tm.back() + rtlength);   // the closing entry (same Trep and files)
    tr.push_back(tr.back());
    *nrec = (int)tm.size();
    if (!time && !Trep) return XBG_OK;
    if (cap < *nrec || !time || !Trep) return XBG_ERR_ARG;
    for (int k = 0; k < *nrec; k++) { time[k] = tm[k]; Trep[k] = tr[k]; }
    return XBG_OK;
}

extern "C" int xbg_read_xbbnd_step(const char* path, int step, int ny, int ntheta, int nrec, double* q,
                                   double* St, double* Trep) {
    if (!path || ny < 1 || ntheta < 1 || nrec < 1 || !q || !St || !Trep) return XBG_ERR_ARG;
    std::vector<double> tm, tr;
    std::vector<std::string> qf, ef;
    int rc = xb_entries(path, tm, tr, qf, ef);
    if (rc) return rc;
    if (step < 0 || step >= (int)tm.size()) return XBG_ERR_ARG;
    // file names are as written in the list (relative names resolve against
    // the working directory, as in the reference)
    auto load = [&](const std::string& f, size_t n, double* dst) -> int {
        FILE* fp = std::fopen(f.c_str(), "rb");
        if (!fp) return XBG_ERR_IO;
        std::vector<double> buf(n);
        size_t got = std::fread(buf.data(), sizeof(double), n, fp);
        std::fclose(fp);
        if (got != n) return XBG_ERR_FORMAT;
        for (size_t k = 0; k < n; k++) dst[k] = (double)(float)buf[k];   // DECNUM rounding
        return XBG_OK;
    };
    if ((rc = load(qf[step], (size_t)4 * ny * nrec, q))) return rc;
    if ((rc = load(ef[step], (size_t)ntheta * ny * nrec, St))) return rc;
    *Trep = (double)(float)tr[step];
    return XBG_OK;
}

// ReadSPECBnd (read_input.cpp:534-593): a list of (time, SWAN spectrum file)
// records, tab / space / comma separated, blank lines skipped, and the
// closing record rtlength after the last (same file).  Names are copied
// NUL-terminated into rows of name_len bytes; a name that does not fit is a
// format error.
extern "C" int xbg_read_spec_list(const char* path, double rtlength, double* time, char* names, int name_len,
                                  int cap, int* nrec) {
    if (!path || !nrec) return XBG_ERR_ARG;
    std::ifstream fs(path);
    if (fs.fail()) return XBG_ERR_IO;
    std::vector<double> tm;
    std::vector<std::string> nm;
    std::string line;
    std::vector<std::string> t;
    while (std::getline(fs, line)) {
        if (line.empty()) continue;
        if (!tokens(line, 2, t)) return XBG_ERR_FORMAT;
        double v;
        if (!num(t[0], v)) return XBG_ERR_FORMAT;
        tm.push_back(v);
        nm.push_back(t[1]);
    }
    if (tm.empty()) return XBG_ERR_FORMAT;
    tm.push_back(tm.back() + rtlength);   // the closing record
    nm.push_back(nm.back());
    *nrec = (int)tm.size();
    if (!time && !names) return XBG_OK;
    if (cap < *nrec || !time || !names || name_len < 2) return XBG_ERR_ARG;
    for (int k = 0; k < *nrec; k++) {
        if ((int)nm[k].size() >= name_len) return XBG_ERR_FORMAT;
        time[k] = tm[k];
        std::memset(names + (size_t)k * name_len, 0, name_len);
        std::memcpy(names + (size_t)k * name_len, nm[k].data(), nm[k].size());
    }
    return XBG_OK;
}
