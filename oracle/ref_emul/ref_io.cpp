// TEST INFRASTRUCTURE ONLY: plain-C entry points onto the reference's own
// input readers (read_input.cpp, compiled in place from the reference
// checkout), so the tests can compare the library's readers with them on
// the same files.  Every function here calls the reference function and
// copies its result out; nothing is restated.  The reference readers call
// exit() on malformed files, so the tests only hand them valid ones.
#include <cstring>
#include <string>
#include <vector>

#include "XBeachGPU.h"

// declared in XBeachGPU.h:342-343 and defined in a reference file not built here
template <class T> const T& min(const T& a, const T& b) { return !(b < a) ? a : b; }
template <class T> const T& max(const T& a, const T& b) { return (a < b) ? b : a; }
template const double& min<double>(const double&, const double&);
template const double& max<double>(const double&, const double&);

std::vector<SLBnd> readWLfile(std::string WLfilename);
std::vector<WindBnd> readWNDfile(std::string WNDfilename, double grdalpha);
std::vector<Wavebndparam> ReadCstBnd(XBGPUParam XParam);
std::vector<Wavebndparam> ReadJSWPBnd(XBGPUParam XParam);
XBGPUParam readXbbndhead(XBGPUParam Param);
std::vector<Wavebndparam> readXbbndfile(XBGPUParam Param);
std::vector<Wavebndparam> ReadSPECBnd(XBGPUParam XParam);
void readbathyHead(std::string filename, int& nx, int& ny, double& dx, double& grdalpha);
extern "C" void readbathy(std::string filename, float*& zb);
extern "C" void readXBbathy(std::string filename, int nx, int ny, float*& zb);
extern "C" void readXbbndstep(XBGPUParam Param, std::vector<Wavebndparam> wavebnd, int step, float& Trep,
                              double*& qfile, double*& Stfile);

extern "C" {

int ref_io_sealevel(const char* path, double* out, int cap) {
    std::vector<SLBnd> v = readWLfile(path);
    for (int k = 0; k < (int)v.size() && k < cap; k++) {
        out[3 * k] = v[k].time; out[3 * k + 1] = v[k].wlev0; out[3 * k + 2] = v[k].wlev1;
    }
    return (int)v.size();
}

int ref_io_wind(const char* path, double grdalpha, double* out, int cap) {
    std::vector<WindBnd> v = readWNDfile(path, grdalpha);
    for (int k = 0; k < (int)v.size() && k < cap; k++) {
        double r[6] = {v[k].time, v[k].spd, v[k].dir, v[k].theta, v[k].U, v[k].V};
        std::memcpy(out + 6 * k, r, sizeof(r));
    }
    return (int)v.size();
}

int ref_io_wave(const char* path, int jonswap, double grdalpha, double rtlength, double* out, int cap) {
    XBGPUParam P;
    P.wavebndfile = path;
    P.grdalpha = grdalpha;
    P.rtlength = rtlength;
    std::vector<Wavebndparam> v = jonswap ? ReadJSWPBnd(P) : ReadCstBnd(P);
    const int nc = jonswap ? 6 : 5;
    for (int k = 0; k < (int)v.size() && k < cap; k++) {
        double r[6] = {v[k].time, v[k].Hs, v[k].Tp, v[k].Dp, v[k].s, v[k].gamma};
        std::memcpy(out + nc * k, r, nc * sizeof(double));
    }
    return (int)v.size();
}

void ref_io_md_head(const char* path, int* nx, int* ny, double* dx, double* grdalpha) {
    readbathyHead(path, *nx, *ny, *dx, *grdalpha);
}

void ref_io_md(const char* path, float* zb) { readbathy(path, zb); }

void ref_io_dep(const char* path, int nx, int ny, float* zb) { readXBbathy(path, nx, ny, zb); }

void ref_io_xbhead(const char* path, double* hdr) {
    XBGPUParam P;
    P.wavebndfile = path;
    P = readXbbndhead(P);
    hdr[0] = P.thetamin; hdr[1] = P.thetamax; hdr[2] = P.dtheta; hdr[3] = P.dtbc; hdr[4] = P.rtlength;
}

int ref_io_xblist(const char* path, double rtlength, double* time, double* Trep, int cap) {
    XBGPUParam P;
    P.wavebndfile = path;
    P.rtlength = rtlength;
    std::vector<Wavebndparam> v = readXbbndfile(P);
    for (int k = 0; k < (int)v.size() && k < cap; k++) { time[k] = v[k].time; Trep[k] = v[k].Trep; }
    return (int)v.size();
}

void ref_io_xbstep(const char* path, double rtlength, double dtbc, int nx, int ny, int ntheta, int step,
                   double* q, double* St, double* Trep) {
    XBGPUParam P;
    P.wavebndfile = path;
    P.rtlength = rtlength;
    P.dtbc = dtbc;
    P.nx = nx; P.ny = ny; P.ntheta = ntheta;
    std::vector<Wavebndparam> v = readXbbndfile(P);
    float tr = 0.0f;
    readXbbndstep(P, v, step, tr, q, St);
    *Trep = tr;
}

// ReadSPECBnd's records: times and file names (rows of name_len bytes)
int ref_io_speclist(const char* path, double rtlength, double* time, char* names, int name_len, int cap) {
    XBGPUParam P;
    P.wavebndfile = path;
    P.rtlength = rtlength;
    std::vector<Wavebndparam> v = ReadSPECBnd(P);
    for (int k = 0; k < (int)v.size() && k < cap; k++) {
        time[k] = v[k].time;
        std::memset(names + (size_t)k * name_len, 0, name_len);
        std::strncpy(names + (size_t)k * name_len, v[k].Swanfile.c_str(), name_len - 1);
    }
    return (int)v.size();
}

}  // extern "C"
