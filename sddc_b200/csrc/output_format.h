// File formats of the reference's output, shared by the host library
// (synchronous writers, host_setup.cpp) and the drop-in's background writer
// (output.cu):
//   restart  WRITE_ALL_DATA_PARALLEL (write_data.f90:1-83), read back by
//            READ_ALL_DATA_BINARY (read_data_restart.f90:36-70): int32 iter,
//            float64 ctime, then per cell an int32 global cell number and
//            the cell's Q(9,N,N) as float64, native byte order
//   Tecplot  tecpost_parallel (tecplotter.f90:99-415): binary .plt of
//            version #!TDV111, one FE-quadrilateral zone, block packing,
//            13 float32 variables X Y RHO U V W P Bx By Bz Az muAV etaAV on
//            the plot nodes, then the 0-based connectivity of the plot cells
// One rank writes the whole file, so the offsets the reference computes per
// rank collapse to one sequential write.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace sddc {
namespace fmt {

// 'restart.', I8.8, '.dat' (write_data.f90:45)
inline std::string restart_name(int iter)
{
    char b[32];
    if (iter < 0 || iter > 99999999) return "restart.********.dat";  // Fortran's overflow field
    std::snprintf(b, sizeof b, "restart.%08d.dat", iter);
    return b;
}

// 'TEC', I7.7 of int(ctime), characters 3..6 of F6.3 of the fraction,
// '.plt' (tecplotter.f90:176-177).  The fraction is rounded to three
// decimals from its exact binary value; an exact tie rounds away from zero
// (Fortran's compatible rounding).  A fraction that rounds up to 1 gives
// ".000" with the integer part unchanged, as the reference's name does.
inline std::string tecplot_name(double ctime)
{
    const double ip = std::trunc(ctime);
    std::string head;
    if (!(ip >= 0.0) || ip > 9999999.0) head = "TEC*******";
    else {
        char b[16];
        std::snprintf(b, sizeof b, "TEC%07d", (int)ip);
        head = b;
    }
    const double frac = ctime - ip;
    // frac (53 bits) * 1000 (10 bits) is exact in the 64-bit mantissa of
    // long double; fall back to the nearest integer where that is narrower
    long double t = (long double)frac * 1000.0L;
    long double fl = std::floor(t);
    long double r = t - fl;
    long long d = (long long)fl + ((r > 0.5L || r == 0.5L) ? 1 : 0);
    if (d < 0) d = -d;  // negative times do not occur in a run
    char tail[16];
    std::snprintf(tail, sizeof tail, ".%03lld", d % 1000);
    return head + tail + ".plt";
}

struct Writer {
    std::FILE *f = nullptr;
    std::string err;
    std::vector<char> buf;
    explicit Writer(const char *path)
    {
        f = std::fopen(path, "wb");
        if (!f) err = std::string("cannot open ") + path + " for writing";
        else {
            buf.resize(8u << 20);
            std::setvbuf(f, buf.data(), _IOFBF, buf.size());
        }
    }
    bool put(const void *p, size_t bytes)
    {
        if (!f || !err.empty()) return false;
        if (bytes && std::fwrite(p, 1, bytes, f) != bytes) err = "short write";
        return err.empty();
    }
    template <class T> bool put1(T v) { return put(&v, sizeof v); }
    bool close()
    {
        if (f) {
            if (std::fclose(f) != 0 && err.empty()) err = "close failed";
            f = nullptr;
        }
        return err.empty();
    }
    ~Writer()
    {
        if (f) std::fclose(f);
    }
};

// WRITE_ALL_DATA_PARALLEL: icg NULL writes cell numbers 1..ncell
inline int write_restart(const char *path, int iter, double ctime, int N, int ncell, const int *icg,
                         const double *Q, std::string &err)
{
    Writer w(path);
    const size_t cell = (size_t)9 * N * N;
    bool ok = w.put1<int32_t>(iter) && w.put1<double>(ctime);
    for (int c = 0; ok && c < ncell; c++) {
        const int32_t g = icg ? icg[c] : c + 1;
        ok = w.put1<int32_t>(g) && w.put(Q + cell * c, cell * sizeof(double));
    }
    ok = w.close() && ok;
    if (!ok) err = "restart " + std::string(path) + ": " + w.err;
    return ok ? 0 : -1;
}

// READ_ALL_DATA_BINARY: nrec records (NCELLGLOB); a record whose global
// number maps to no local cell (icg2ic 0, or outside 1..ncell without a map)
// is skipped, as IC = 0 is there.  icg2ic (nglob entries) may be NULL for
// the identity.
inline int read_restart(const char *path, int N, int ncell, int nrec, const int *icg2ic, int nglob, double *Q,
                        int *iter, double *ctime, std::string &err)
{
    std::FILE *f = std::fopen(path, "rb");
    if (!f) {
        err = std::string("cannot open ") + path;
        return -1;
    }
    const size_t cell = (size_t)9 * N * N;
    std::vector<double> tmp(cell);
    int32_t it = 0;
    double ct = 0.0;
    bool ok = std::fread(&it, 4, 1, f) == 1 && std::fread(&ct, 8, 1, f) == 1;
    for (int i = 0; ok && i < nrec; i++) {
        int32_t g = 0;
        ok = std::fread(&g, 4, 1, f) == 1 && std::fread(tmp.data(), sizeof(double), cell, f) == cell;
        if (!ok) break;
        int ic = 0;
        if (icg2ic) ic = (g >= 1 && g <= nglob) ? icg2ic[g - 1] : 0;
        else ic = (g >= 1 && g <= ncell) ? g : 0;
        if (ic >= 1 && ic <= ncell) std::memcpy(Q + cell * (ic - 1), tmp.data(), cell * sizeof(double));
    }
    std::fclose(f);
    if (!ok) {
        err = std::string("restart ") + path + ": file ends before " + std::to_string(nrec) + " records";
        return -1;
    }
    if (iter) *iter = it;
    if (ctime) *ctime = ct;
    return 0;
}

// one plotted variable: value i is p[i * stride]
struct PlotVar {
    const double *p;
    size_t stride;
};

constexpr int kPlotVars = 13;

inline bool put_string(Writer &w, const char *s)
{
    // write_tecplot_string: one int32 per character, then 0
    for (const char *c = s; *c; c++)
        if (!w.put1<int32_t>((int32_t)(unsigned char)*c)) return false;
    return w.put1<int32_t>(0);
}

// tecpost_parallel for one rank: vars in the order X Y RHO U V W P Bx By Bz
// Az muAV etaAV, connec (4,plotcells) 1-based as connec_c2n holds it.
inline int write_tecplot(const char *path, double ctime, int plotnodes, int plotcells, const PlotVar *vars,
                         const int *connec, std::string &err)
{
    static const char *names[kPlotVars] = {"X", "Y", "RHO", "U", "V", "W", "P",
                                           "Bx", "By", "Bz", "Az", "muAV", "etaAV"};
    // minval / maxval of each variable in double (minmax(2,nvar))
    double minmax[2 * kPlotVars];
    for (int v = 0; v < kPlotVars; v++) {
        double lo = vars[v].p[0], hi = lo;
        for (int i = 1; i < plotnodes; i++) {
            const double x = vars[v].p[(size_t)i * vars[v].stride];
            if (x < lo) lo = x;
            if (x > hi) hi = x;
        }
        minmax[2 * v] = lo;
        minmax[2 * v + 1] = hi;
    }
    Writer w(path);
    bool ok = w.put("#!TDV111", 8) && w.put1<int32_t>(1) && w.put1<int32_t>(0) && put_string(w, "step data") &&
              w.put1<int32_t>(kPlotVars);
    for (int v = 0; ok && v < kPlotVars; v++) ok = put_string(w, names[v]);
    const int32_t zone[12] = {-1, 3, 0, 0, 0, 0, plotnodes, plotcells, 0, 0, 0, 0};
    ok = ok && w.put1<float>(299.0f) && put_string(w, "ZONE 001") && w.put1<int32_t>(-1) && w.put1<int32_t>(0) &&
         w.put1<double>(ctime) && w.put(zone, sizeof zone) && w.put1<float>(357.0f) && w.put1<float>(299.0f);
    int32_t fmt[kPlotVars + 3];
    for (int v = 0; v < kPlotVars; v++) fmt[v] = 1;  // float
    fmt[kPlotVars] = 0;
    fmt[kPlotVars + 1] = 0;
    fmt[kPlotVars + 2] = -1;
    ok = ok && w.put(fmt, sizeof fmt) && w.put(minmax, sizeof minmax);
    std::vector<float> blk(plotnodes > 0 ? plotnodes : 1);
    for (int v = 0; ok && v < kPlotVars; v++) {
        for (int i = 0; i < plotnodes; i++) blk[i] = (float)vars[v].p[(size_t)i * vars[v].stride];
        ok = w.put(blk.data(), sizeof(float) * (size_t)plotnodes);
    }
    std::vector<int32_t> cn(4 * (size_t)(plotcells > 0 ? plotcells : 1));
    for (size_t i = 0; i < 4 * (size_t)plotcells; i++) cn[i] = connec[i] - 1;
    ok = ok && w.put(cn.data(), sizeof(int32_t) * 4 * (size_t)plotcells);
    ok = w.close() && ok;
    if (!ok) err = "tecplot " + std::string(path) + ": " + w.err;
    return ok ? 0 : -1;
}

}  // namespace fmt
}  // namespace sddc
