// Readers of the reference's input files (host code, no device work): the run parameters of
// InputFile.txt, the source and receiver lines of SrcRcv.txt and the raw model files, so that a
// workflow built around the reference's executables can drive this library with its own files.
// The writers of the reference's output files need the solver's records and live in solver.cu.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <strings.h>
#include <vector>

#include "../../include/twave.h"

namespace {

// the reference splits every line at "_": the first token names the entry (input_processing.cpp:22-28)
std::vector<std::string> tokens(const std::string &line)
{
    std::vector<std::string> t;
    size_t b = 0;
    while (true) {
        const size_t e = line.find('_', b);
        t.push_back(line.substr(b, e == std::string::npos ? std::string::npos : e - b));
        if (e == std::string::npos) break;
        b = e + 1;
    }
    return t;
}

bool to_long(const std::string &s, long *v)
{
    char *end = nullptr;
    *v = strtol(s.c_str(), &end, 10);
    return end != s.c_str();
}

bool to_double(const std::string &s, double *v)
{
    char *end = nullptr;
    *v = strtod(s.c_str(), &end);
    return end != s.c_str();
}

// 'X' is data y, 'Y' is data x (namespace_forward.hpp:56-61): an "XY" pair of letters or
// numbers arrives as (data y, data x)
}  // namespace

extern "C" {

// file_input_processing (input_processing.cpp:11-137): entries model, grids (X then Y), dxM, dxS
// (num, den), bdry (x left, x right, y left, y right), Nt, MAXdt, CFL, frequency, delay, device;
// dt = MAXdt * CFL (main_host_FDM_2D.tpp:57). Unknown lines are ignored, as there.
int tw_io_read_input(const char *path, tw_io_input *out)
{
    if (!path || !out) return TW_ERR_INVALID;
    std::ifstream f(path);
    if (!f.is_open()) return TW_ERR_IO;
    tw_io_input r{};
    r.cfl = 0.625;              // the reference's defaults (namespace_input.hpp:53-58)
    r.dt_max = (double)(1L << 30);
    r.central_f = 5.0;
    r.time_delay = 0.25;
    std::string line;
    bool ok = true;
    while (std::getline(f, line)) {
        const std::vector<std::string> t = tokens(line);
        const std::string &k = t[0];
        auto num = [&](size_t i, long *v) { ok = ok && i < t.size() && to_long(t[i], v); };
        auto real = [&](size_t i, double *v) { ok = ok && i < t.size() && to_double(t[i], v); };
        if (k == "model") { num(1, &r.My_prmt); num(2, &r.Mx_prmt); }
        else if (k == "grids") { num(1, &r.My); num(2, &r.Mx); }
        else if (k == "dxM") { long a = 0, b = 0; num(1, &a); num(2, &b); r.num_dxM = (int)a; r.den_dxM = (int)b; }
        else if (k == "dxS") { long a = 0, b = 0; num(1, &a); num(2, &b); r.num_dx = (int)a; r.den_dx = (int)b; }
        else if (k == "bdry") {
            if (t.size() < 2 || t[1].size() < 4) ok = false;
            else for (int q = 0; q < 4; q++) r.bdry[q] = (char)toupper(t[1][q]);
        }
        else if (k == "Nt") num(1, &r.Nt);
        else if (k == "MAXdt") real(1, &r.dt_max);
        else if (k == "CFL") real(1, &r.cfl);
        else if (k == "frequency") real(1, &r.central_f);
        else if (k == "delay") real(1, &r.time_delay);
        else if (k == "device") { long d = 0; num(1, &d); r.device = (int)d; }
    }
    if (!ok) return TW_ERR_IO;
    r.dt = r.dt_max * r.cfl;
    *out = r;
    return TW_OK;
}

// input_SrcRcv_locations (inverse.cpp:133-322): "Src_<index>_<XY types>_<X num>_<X den>_<Y num>_<Y den>"
// and "Rcv_<src index>_<index>_<XY types>_..." (receivers after their source), in file order.
// Writes up to cap points; *n is the number in the file; TW_ERR_INVALID when cap is too small.
int tw_io_read_srcrcv(const char *path, tw_io_point *pts, int cap, int *n)
{
    if (!path || !n || cap < 0 || (cap > 0 && !pts)) return TW_ERR_INVALID;
    std::ifstream f(path);
    if (!f.is_open()) return TW_ERR_IO;
    std::vector<tw_io_point> v;
    std::map<long, bool> sources;
    std::string line;
    while (std::getline(f, line)) {
        const std::vector<std::string> t = tokens(line);
        const bool src = strcasecmp(t[0].c_str(), "Src") == 0, rcv = strcasecmp(t[0].c_str(), "Rcv") == 0;
        if (!src && !rcv) continue;
        const size_t base = src ? 2 : 3;   // position of the grid-type token
        if (t.size() < base + 5 || t[base].size() < 2) return TW_ERR_IO;
        tw_io_point p{};
        long a = 0, b = 0;
        if (!to_long(t[1], &a)) return TW_ERR_IO;
        p.src_index = a;
        p.rcv_index = -1;
        if (rcv) {
            if (!to_long(t[2], &b)) return TW_ERR_IO;
            p.rcv_index = b;
            if (!sources.count(p.src_index)) return TW_ERR_IO;   // a receiver before its source
        } else {
            sources[p.src_index] = true;
        }
        p.type_y = (char)toupper(t[base][0]);   // X letter: data y
        p.type_x = (char)toupper(t[base][1]);   // Y letter: data x
        long q[4];
        for (int i = 0; i < 4; i++)
            if (!to_long(t[base + 1 + i], &q[i])) return TW_ERR_IO;
        p.num_y = q[0];
        p.den_y = q[1];
        p.num_x = q[2];
        p.den_x = q[3];
        v.push_back(p);
    }
    *n = (int)v.size();
    if ((int)v.size() > cap) return pts ? TW_ERR_INVALID : TW_OK;
    for (size_t i = 0; i < v.size(); i++) pts[i] = v[i];
    return TW_OK;
}

// input_inverse_parameter (inverse.cpp:6-130): raw native doubles of the (Mx_prmt+1) x (My_prmt+1)
// node model, x outer; out: the padded (Mx_prmt+2) x (My_prmt+2) layout tw_set_material_model
// takes (row stride My_prmt+2), zero in the padding.
int tw_io_read_model(const char *path, long Mx_prmt, long My_prmt, double *padded)
{
    if (!path || !padded || Mx_prmt < 1 || My_prmt < 1) return TW_ERR_INVALID;
    const long Nx = Mx_prmt + 1, Ny = My_prmt + 1;
    FILE *fp = fopen(path, "rb");
    if (!fp) return TW_ERR_IO;
    fseek(fp, 0, SEEK_END);
    const long bytes = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    if (bytes != Nx * Ny * (long)sizeof(double)) {   // the reference stops on a size mismatch (inverse.cpp:48-53)
        fclose(fp);
        return TW_ERR_IO;
    }
    std::vector<double> raw((size_t)Nx * Ny);
    const size_t got = fread(raw.data(), sizeof(double), raw.size(), fp);
    fclose(fp);
    if (got != raw.size()) return TW_ERR_IO;
    memset(padded, 0, sizeof(double) * (size_t)(Nx + 1) * (Ny + 1));
    for (long ix = 0; ix < Nx; ix++)
        for (long iy = 0; iy < Ny; iy++) padded[ix * (Ny + 1) + iy] = raw[(size_t)ix * Ny + iy];
    return TW_OK;
}

}  // extern "C"
