// ncwrite.cpp -- the map-output file of the model in the netCDF classic
// format (64-bit offset variant), written without libnetcdf.
//
// Layout of a classic netCDF file (the published format specification):
//   header = magic numrecs dim_list gatt_list var_list
//     magic    'C' 'D' 'F' 2           (2: 64-bit offsets)
//     numrecs  number of records (4-byte big-endian)
//     dim_list NC_DIMENSION n [name length]...     (length 0: the record dim)
//     gatt_list ABSENT
//     var_list NC_VARIABLE n [name ndims dimids... vatt_list type vsize begin]...
//   data   = the non-record variables, each at its begin offset, then the
//            records: record r of variable v at begin_v + r * recsize, recsize
//            the sum of the record variables' vsize.
// Integers are big-endian; names are padded with zero bytes to 4; floats are
// big-endian IEEE single precision.
//
// The dimensions and variables are the reference's (writenetcdf.cpp:32-240):
// dims xx, yy, theta, time (unlimited); variables time(time), xx(xx), yy(yy),
// theta(theta) and one float per output name over (time, yy, xx) or
// (time, theta, yy, xx), in the order they are given.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/xbg_io.h"

namespace {

const uint32_t NC_DIMENSION = 0x0A, NC_VARIABLE = 0x0B, NC_FLOAT = 5;

struct Var {
    std::string name;
    std::vector<int> dims;   // dimension ids
    bool record = false;
    uint64_t vsize = 0, begin = 0;
};

void put32(std::vector<uint8_t>& b, uint32_t v) {
    for (int s = 24; s >= 0; s -= 8) b.push_back((uint8_t)(v >> s));
}
void put64(std::vector<uint8_t>& b, uint64_t v) {
    for (int s = 56; s >= 0; s -= 8) b.push_back((uint8_t)(v >> s));
}
void put_name(std::vector<uint8_t>& b, const std::string& s) {
    put32(b, (uint32_t)s.size());
    b.insert(b.end(), s.begin(), s.end());
    while (b.size() % 4) b.push_back(0);
}
// big-endian copy of n floats
void to_be(const float* src, size_t n, std::vector<uint8_t>& dst) {
    dst.resize(n * 4);
    for (size_t k = 0; k < n; k++) {
        uint32_t u;
        std::memcpy(&u, src + k, 4);
        dst[4 * k] = (uint8_t)(u >> 24);
        dst[4 * k + 1] = (uint8_t)(u >> 16);
        dst[4 * k + 2] = (uint8_t)(u >> 8);
        dst[4 * k + 3] = (uint8_t)u;
    }
}

}  // namespace

struct xbg_nc {
    FILE* fp = nullptr;
    int nx = 0, ny = 0, nt = 0;
    std::vector<Var> vars;       // time, xx, yy, theta, then the outputs
    uint64_t recsize = 0, rec0 = 0;
    int64_t nrec = 0;
    std::vector<uint8_t> buf;

    int write_at(uint64_t off, const void* p, size_t n) {
        if (fseeko(fp, (off_t)off, SEEK_SET) != 0) return XBG_ERR_IO;
        if (n && fwrite(p, 1, n, fp) != n) return XBG_ERR_IO;
        return XBG_OK;
    }
    int write_floats(uint64_t off, const float* p, size_t n) {
        to_be(p, n, buf);
        return write_at(off, buf.data(), buf.size());
    }
};

extern "C" int xbg_nc_create(const char* path, int clobber, int nx, int ny, double dx, int ntheta, double dtheta,
                             double thetamin, int nvars, const char* const* names, const int* ndims, xbg_nc** out) {
    if (!path || !out || nx < 1 || ny < 1 || ntheta < 1 || nvars < 0 || (nvars && (!names || !ndims)))
        return XBG_ERR_ARG;
    *out = nullptr;
    // dimension ids: 0 xx, 1 yy, 2 theta, 3 time
    const uint32_t dimlen[4] = {(uint32_t)nx, (uint32_t)ny, (uint32_t)ntheta, 0};
    const char* dimname[4] = {"xx", "yy", "theta", "time"};
    std::vector<Var> vars(4);
    vars[0].name = "time"; vars[0].dims = {3}; vars[0].record = true;
    vars[1].name = "xx"; vars[1].dims = {0};
    vars[2].name = "yy"; vars[2].dims = {1};
    vars[3].name = "theta"; vars[3].dims = {2};
    for (int k = 0; k < nvars; k++) {
        if (!names[k] || !names[k][0] || (ndims[k] != 3 && ndims[k] != 4)) return XBG_ERR_ARG;
        Var v;
        v.name = names[k];
        for (const Var& w : vars)
            if (w.name == v.name) return XBG_ERR_ARG;
        v.dims = ndims[k] == 3 ? std::vector<int>{3, 1, 0} : std::vector<int>{3, 2, 1, 0};
        v.record = true;
        vars.push_back(v);
    }
    for (Var& v : vars) {   // vsize: one record's (or the whole variable's) bytes
        uint64_t n = 4;
        for (int d : v.dims)
            if (dimlen[d]) n *= dimlen[d];
        v.vsize = n;
    }
    // header with placeholder offsets, to learn its size
    auto header = [&](std::vector<uint8_t>& b, int64_t numrecs) {
        b.clear();
        b.push_back('C'); b.push_back('D'); b.push_back('F'); b.push_back(2);
        put32(b, (uint32_t)numrecs);
        put32(b, NC_DIMENSION);
        put32(b, 4);
        for (int d = 0; d < 4; d++) { put_name(b, dimname[d]); put32(b, dimlen[d]); }
        put32(b, 0); put32(b, 0);            // no global attributes
        put32(b, NC_VARIABLE);
        put32(b, (uint32_t)vars.size());
        for (const Var& v : vars) {
            put_name(b, v.name);
            put32(b, (uint32_t)v.dims.size());
            for (int d : v.dims) put32(b, (uint32_t)d);
            put32(b, 0); put32(b, 0);        // no variable attributes
            put32(b, NC_FLOAT);
            put32(b, (uint32_t)(v.vsize > 0xFFFFFFFFull ? 0xFFFFFFFFull : v.vsize));
            put64(b, v.begin);
        }
    };
    std::vector<uint8_t> hb;
    header(hb, 0);
    uint64_t off = hb.size();
    for (Var& v : vars)
        if (!v.record) { v.begin = off; off += v.vsize; }
    const uint64_t rec0 = off;
    uint64_t recsize = 0;
    for (Var& v : vars)
        if (v.record) { v.begin = rec0 + recsize; recsize += v.vsize; }
    header(hb, 0);

    struct stat st;
    if (!clobber && stat(path, &st) == 0) return XBG_ERR_ARG;
    FILE* fp = fopen(path, "wb");
    if (!fp) return XBG_ERR_IO;
    xbg_nc* f = new xbg_nc();
    f->fp = fp; f->nx = nx; f->ny = ny; f->nt = ntheta;
    f->vars = vars; f->recsize = recsize; f->rec0 = rec0;
    int rc = f->write_at(0, hb.data(), hb.size());
    // coordinate values as the reference computes them (float arithmetic for theta)
    std::vector<float> xs(nx), ys(ny), th(ntheta);
    for (int i = 0; i < nx; i++) xs[i] = (float)(i * dx);
    for (int j = 0; j < ny; j++) ys[j] = (float)(j * dx);
    const float dth = (float)dtheta, tmin = (float)thetamin;
    for (int t = 0; t < ntheta; t++) th[t] = t * dth + tmin + 0.5f * dth;
    if (!rc) rc = f->write_floats(vars[1].begin, xs.data(), xs.size());
    if (!rc) rc = f->write_floats(vars[2].begin, ys.data(), ys.size());
    if (!rc) rc = f->write_floats(vars[3].begin, th.data(), th.size());
    if (!rc && fflush(fp) != 0) rc = XBG_ERR_IO;
    if (rc) { fclose(fp); delete f; return rc; }
    *out = f;
    return XBG_OK;
}

extern "C" int xbg_nc_write_record(xbg_nc* f, double time, const float* const* data) {
    if (!f || (f->vars.size() > 4 && !data)) return XBG_ERR_ARG;
    const uint64_t base = f->rec0 + (uint64_t)f->nrec * f->recsize;
    const float t = (float)time;
    int rc = f->write_floats(base + (f->vars[0].begin - f->rec0), &t, 1);
    for (size_t k = 4; k < f->vars.size() && !rc; k++) {
        const Var& v = f->vars[k];
        if (!data[k - 4]) return XBG_ERR_ARG;
        rc = f->write_floats(base + (v.begin - f->rec0), data[k - 4], v.vsize / 4);
    }
    if (rc) return rc;
    f->nrec++;
    uint8_t nr[4] = {(uint8_t)(f->nrec >> 24), (uint8_t)(f->nrec >> 16), (uint8_t)(f->nrec >> 8), (uint8_t)f->nrec};
    rc = f->write_at(4, nr, 4);
    if (!rc && fflush(f->fp) != 0) rc = XBG_ERR_IO;
    return rc;
}

extern "C" int xbg_nc_records(const xbg_nc* f, int64_t* nrec) {
    if (!f || !nrec) return XBG_ERR_ARG;
    *nrec = f->nrec;
    return XBG_OK;
}

extern "C" int xbg_nc_close(xbg_nc* f) {
    if (!f) return XBG_ERR_ARG;
    int rc = fclose(f->fp) == 0 ? XBG_OK : XBG_ERR_IO;
    delete f;
    return rc;
}
