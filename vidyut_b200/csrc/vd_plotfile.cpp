// vd_plotfile.cpp -- plotfile output of one box (vd_write_plotfile in vidyut_b200.h).
//
// The reference writes its state with amrex::WriteMultiLevelPlotfile
// (Vidyut::WritePlotFile, Source/Plot.cpp:29-39) under the names of
// Source/Vidyut.cpp:32-52.  This library has no AMReX, so it writes the same
// published single-level plotfile layout itself, from host memory:
//   <dir>/Header               text: "HyperCLaw-V1.1", the variable names, the
//                              dimension, time, level count, problem extent,
//                              domain box, step, cell size, coordinate system,
//                              and the level's grid with its physical extent
//   <dir>/Level_0/Cell_H       text: the multi-fab header (component count, the
//                              box array, where each FAB starts, per-component
//                              minima and maxima)
//   <dir>/Level_0/Cell_D_00000 the FAB: a one-line descriptor of the number format
//                              (IEEE double, little-endian) and the box, then the
//                              values, component by component, x fastest.
#include <sys/stat.h>
#include <sys/types.h>

#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "vd_host.h"

namespace {

int perr(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int perr(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return vd_host::set_error(code, buf);
}

bool make_dir(const std::string& d)
{
    if (mkdir(d.c_str(), 0755) == 0) return true;
    struct stat sb;
    return errno == EEXIST && stat(d.c_str(), &sb) == 0 && S_ISDIR(sb.st_mode);
}

// an integer vector of the box's dimension, "(a,b,c)"
std::string ivec(const int* v, int dim)
{
    std::ostringstream o;
    o << '(';
    for (int d = 0; d < dim; d++) o << (d ? "," : "") << v[d];
    o << ')';
    return o.str();
}

// a cell-centred box, "((lo) (hi) (0,..))"
std::string box_text(const vd_box* bx, int dim)
{
    const int z[3] = {0, 0, 0};
    return "(" + ivec(bx->lo, dim) + " " + ivec(bx->hi, dim) + " " + ivec(z, dim) + ")";
}

bool little_endian()
{
    const uint16_t one = 1;
    unsigned char c;
    memcpy(&c, &one, 1);
    return c == 1;
}

}  // namespace

extern "C" int vd_write_plotfile(const char* dir, const vd_box* bx, const double* data, int ncomp,
                                 const char* const* names, const double prob_lo[3], const double dx[3], double time,
                                 int step)
{
    if (!dir || !bx || !data || !names || !prob_lo || !dx) return perr(VD_ERR_ARG, "null argument");
    const int dim = bx->dim;
    if (dim < 1 || dim > 3) return perr(VD_ERR_DIM, "dimension %d", dim);
    if (ncomp < 1) return perr(VD_ERR_ARG, "ncomp %d", ncomp);
    int64_t ncell = 1;
    int n[3];
    for (int d = 0; d < 3; d++) {
        n[d] = bx->hi[d] - bx->lo[d] + 1;
        if (n[d] < 1 || (d >= dim && n[d] != 1)) return perr(VD_ERR_ARG, "box extent %d along %d", n[d], d);
        ncell *= n[d];
    }
    for (int c = 0; c < ncomp; c++)
        if (!names[c] || !names[c][0] || strchr(names[c], '\n'))
            return perr(VD_ERR_ARG, "variable name %d is empty or spans lines", c);
    const std::string root(dir), lev = root + "/Level_0";
    if (!make_dir(root) || !make_dir(lev)) return perr(VD_ERR_ARG, "cannot create %s: %s", lev.c_str(), strerror(errno));

    // Header
    {
        std::ofstream h(root + "/Header", std::ios::out | std::ios::trunc);
        if (!h) return perr(VD_ERR_ARG, "cannot write %s/Header", dir);
        h << std::setprecision(17);
        h << "HyperCLaw-V1.1\n" << ncomp << '\n';
        for (int c = 0; c < ncomp; c++) h << names[c] << '\n';
        h << dim << '\n' << time << '\n' << 0 << '\n';
        for (int d = 0; d < dim; d++) h << prob_lo[d] << ' ';
        h << '\n';
        for (int d = 0; d < dim; d++) h << prob_lo[d] + dx[d] * n[d] << ' ';
        h << '\n';
        h << '\n';  // refinement ratios: none below one level
        h << box_text(bx, dim) << " \n";
        h << step << " \n";
        for (int d = 0; d < dim; d++) h << dx[d] << ' ';
        h << '\n';
        h << 0 << '\n' << 0 << '\n';  // Cartesian coordinates, no boundary width
        h << 0 << ' ' << 1 << ' ' << time << '\n' << step << '\n';
        for (int d = 0; d < dim; d++)
            h << prob_lo[d] + dx[d] * bx->lo[d] << ' ' << prob_lo[d] + dx[d] * (bx->hi[d] + 1) << '\n';
        h << "Level_0/Cell\n";
        if (!h) return perr(VD_ERR_ARG, "writing %s/Header failed", dir);
    }
    // the FAB
    std::string fab_head;
    {
        std::ostringstream f;
        f << "FAB ((8, (64 11 52 0 1 12 0 1023)),(8, " << (little_endian() ? "(8 7 6 5 4 3 2 1)" : "(1 2 3 4 5 6 7 8)")
          << "))" << box_text(bx, dim) << ' ' << ncomp << '\n';
        fab_head = f.str();
        std::ofstream d(lev + "/Cell_D_00000", std::ios::out | std::ios::trunc | std::ios::binary);
        if (!d) return perr(VD_ERR_ARG, "cannot write %s/Cell_D_00000", lev.c_str());
        d << fab_head;
        d.write(reinterpret_cast<const char*>(data), (std::streamsize)(sizeof(double) * ncell * ncomp));
        if (!d) return perr(VD_ERR_ARG, "writing %s/Cell_D_00000 failed", lev.c_str());
    }
    // Cell_H: the multi-fab header with the per-component extrema
    {
        std::ofstream h(lev + "/Cell_H", std::ios::out | std::ios::trunc);
        if (!h) return perr(VD_ERR_ARG, "cannot write %s/Cell_H", lev.c_str());
        h << std::setprecision(17);
        h << 1 << '\n' << 1 << '\n' << ncomp << '\n' << 0 << '\n';
        h << "(1 0\n" << box_text(bx, dim) << "\n)\n";
        h << 1 << '\n' << "FabOnDisk: Cell_D_00000 0\n\n";
        std::vector<double> mn(ncomp), mx(ncomp);
        for (int c = 0; c < ncomp; c++) {
            const double* p = data + (int64_t)c * ncell;
            double a = p[0], b = p[0];
            for (int64_t q = 1; q < ncell; q++) {
                a = std::fmin(a, p[q]);
                b = std::fmax(b, p[q]);
            }
            mn[c] = a;
            mx[c] = b;
        }
        h << 1 << ',' << ncomp << '\n';
        for (int c = 0; c < ncomp; c++) h << mn[c] << ',';
        h << "\n\n" << 1 << ',' << ncomp << '\n';
        for (int c = 0; c < ncomp; c++) h << mx[c] << ',';
        h << '\n';
        if (!h) return perr(VD_ERR_ARG, "writing %s/Cell_H failed", lev.c_str());
    }
    return VD_OK;
}
