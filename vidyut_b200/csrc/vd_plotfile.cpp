// vd_plotfile.cpp -- plotfile and checkpoint files of one box (vd_write_plotfile,
// vd_write_checkpoint, vd_read_checkpoint in vidyut_b200.h).
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
// Checkpoints follow Vidyut::WriteCheckpointFile / ReadCheckpointFile
// (Source/Plot.cpp:41-178): a text Header ("Checkpoint file for Vidyut", the
// finest level, then lines of istep, dt and t_new per level, then the box array)
// and the state as a multi-fab Level_0/phi (phi_H, phi_D_00000) in the same
// layout as the plotfile's.
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

const char* kFabFormat = "FAB ((8, (64 11 52 0 1 12 0 1023)),(8, ";

// Level directory lev holding one FAB of the box: <lev>/<prefix>_D_00000 and the
// multi-fab header <lev>/<prefix>_H with the per-component extrema.
int write_multifab(const std::string& lev, const char* prefix, const vd_box* bx, int dim, const double* data,
                   int ncomp, int64_t ncell)
{
    const std::string dname = std::string(prefix) + "_D_00000";
    {
        std::ofstream d(lev + "/" + dname, std::ios::out | std::ios::trunc | std::ios::binary);
        if (!d) return perr(VD_ERR_ARG, "cannot write %s/%s", lev.c_str(), dname.c_str());
        d << kFabFormat << (little_endian() ? "(8 7 6 5 4 3 2 1)" : "(1 2 3 4 5 6 7 8)") << "))" << box_text(bx, dim)
          << ' ' << ncomp << '\n';
        d.write(reinterpret_cast<const char*>(data), (std::streamsize)(sizeof(double) * ncell * ncomp));
        if (!d) return perr(VD_ERR_ARG, "writing %s/%s failed", lev.c_str(), dname.c_str());
    }
    std::ofstream h(lev + "/" + prefix + "_H", std::ios::out | std::ios::trunc);
    if (!h) return perr(VD_ERR_ARG, "cannot write %s/%s_H", lev.c_str(), prefix);
    h << std::setprecision(17);
    h << 1 << '\n' << 1 << '\n' << ncomp << '\n' << 0 << '\n';
    h << "(1 0\n" << box_text(bx, dim) << "\n)\n";
    h << 1 << '\n' << "FabOnDisk: " << dname << " 0\n\n";
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
    if (!h) return perr(VD_ERR_ARG, "writing %s/%s_H failed", lev.c_str(), prefix);
    return VD_OK;
}

// box extent checks shared by the writers; n[] and ncell out
int check_box(const vd_box* bx, int n[3], int64_t* ncell)
{
    const int dim = bx->dim;
    if (dim < 1 || dim > 3) return perr(VD_ERR_DIM, "dimension %d", dim);
    *ncell = 1;
    for (int d = 0; d < 3; d++) {
        n[d] = bx->hi[d] - bx->lo[d] + 1;
        if (n[d] < 1 || (d >= dim && n[d] != 1)) return perr(VD_ERR_ARG, "box extent %d along %d", n[d], d);
        *ncell *= n[d];
    }
    return VD_OK;
}

}  // namespace

extern "C" int vd_write_plotfile(const char* dir, const vd_box* bx, const double* data, int ncomp,
                                 const char* const* names, const double prob_lo[3], const double dx[3], double time,
                                 int step)
{
    if (!dir || !bx || !data || !names || !prob_lo || !dx) return perr(VD_ERR_ARG, "null argument");
    const int dim = bx->dim;
    if (ncomp < 1) return perr(VD_ERR_ARG, "ncomp %d", ncomp);
    int64_t ncell = 1;
    int n[3];
    int rc = check_box(bx, n, &ncell);
    if (rc) return rc;
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
    return write_multifab(lev, "Cell", bx, dim, data, ncomp, ncell);
}

extern "C" int vd_write_checkpoint(const char* dir, const vd_box* bx, const double* data, int ncomp, int istep,
                                   double dt, double time)
{
    if (!dir || !bx || !data) return perr(VD_ERR_ARG, "null argument");
    if (ncomp < 1) return perr(VD_ERR_ARG, "ncomp %d", ncomp);
    int n[3];
    int64_t ncell = 1;
    int rc = check_box(bx, n, &ncell);
    if (rc) return rc;
    const std::string root(dir), lev = root + "/Level_0";
    if (!make_dir(root) || !make_dir(lev)) return perr(VD_ERR_ARG, "cannot create %s: %s", lev.c_str(), strerror(errno));
    {
        std::ofstream h(root + "/Header", std::ios::out | std::ios::trunc);
        if (!h) return perr(VD_ERR_ARG, "cannot write %s/Header", dir);
        h << std::setprecision(17);
        h << "Checkpoint file for Vidyut\n" << 0 << '\n';
        h << istep << " \n" << dt << " \n" << time << " \n";
        h << "(1 0\n" << box_text(bx, bx->dim) << "\n)\n";
        if (!h) return perr(VD_ERR_ARG, "writing %s/Header failed", dir);
    }
    return write_multifab(lev, "phi", bx, bx->dim, data, ncomp, ncell);
}

namespace {

// "((a,b,c) (d,e,f) (0,0,0))" -> lo, hi; the dimension from the comma count
bool parse_box(const std::string& t, vd_box* bx)
{
    int v[6] = {0, 0, 0, 0, 0, 0};
    const size_t a = t.find("(("), b = t.find(") (", a == std::string::npos ? 0 : a);
    if (a == std::string::npos || b == std::string::npos) return false;
    const std::string lo = t.substr(a + 2, b - a - 2);
    const size_t c = t.find(')', b + 3);
    if (c == std::string::npos) return false;
    const std::string hi = t.substr(b + 3, c - b - 3);
    int dim = 1;
    for (char ch : lo) dim += ch == ',';
    if (dim < 1 || dim > 3) return false;
    std::string l = lo, h = hi;
    for (char& ch : l) ch = ch == ',' ? ' ' : ch;
    for (char& ch : h) ch = ch == ',' ? ' ' : ch;
    std::istringstream il(l), ih(h);
    for (int d = 0; d < dim; d++)
        if (!(il >> v[d]) || !(ih >> v[3 + d])) return false;
    memset(bx, 0, sizeof(*bx));
    bx->dim = dim;
    for (int d = 0; d < 3; d++) {
        bx->lo[d] = d < dim ? v[d] : 0;
        bx->hi[d] = d < dim ? v[3 + d] : 0;
    }
    return true;
}

}  // namespace

extern "C" int vd_read_checkpoint(const char* dir, vd_box* bx, double* data, int64_t capacity, int* ncomp,
                                  int* istep, double* dt, double* time)
{
    if (!dir || !bx || !ncomp || !istep || !dt || !time) return perr(VD_ERR_ARG, "null argument");
    const std::string root(dir);
    std::ifstream h(root + "/Header");
    if (!h) return perr(VD_ERR_ARG, "cannot read %s/Header", dir);
    std::string title, line;
    std::getline(h, title);
    if (title != "Checkpoint file for Vidyut") return perr(VD_ERR_ARG, "%s/Header is not a Vidyut checkpoint", dir);
    int finest = -1;
    h >> finest;
    std::getline(h, line);
    if (finest != 0) return perr(VD_ERR_ARG, "checkpoint has %d refinement levels; one is supported", finest);
    std::getline(h, line);
    *istep = std::stoi(line);
    std::getline(h, line);
    *dt = std::stod(line);
    std::getline(h, line);
    *time = std::stod(line);
    std::getline(h, line);  // "(1 0"
    if (line.rfind("(1 ", 0) != 0) return perr(VD_ERR_ARG, "checkpoint box array must hold one box");
    std::getline(h, line);
    if (!parse_box(line, bx)) return perr(VD_ERR_ARG, "unreadable box in %s/Header", dir);
    int n[3];
    int64_t ncell = 1;
    int rc = check_box(bx, n, &ncell);
    if (rc) return rc;
    std::ifstream d(root + "/Level_0/phi_D_00000", std::ios::binary);
    if (!d) return perr(VD_ERR_ARG, "cannot read %s/Level_0/phi_D_00000", dir);
    std::string head;
    std::getline(d, head);
    const std::string want = std::string(kFabFormat) + (little_endian() ? "(8 7 6 5 4 3 2 1)" : "(1 2 3 4 5 6 7 8)") + "))";
    if (head.rfind(want, 0) != 0) return perr(VD_ERR_ARG, "FAB data not in this machine's IEEE double format");
    const int nc = std::atoi(head.substr(head.rfind(' ') + 1).c_str());
    if (nc < 1) return perr(VD_ERR_ARG, "FAB component count unreadable");
    *ncomp = nc;
    if (!data) return VD_OK;  // size query
    if (capacity < ncell * nc) return perr(VD_ERR_ARG, "buffer of %lld doubles for %lld values", (long long)capacity, (long long)(ncell * nc));
    d.read(reinterpret_cast<char*>(data), (std::streamsize)(sizeof(double) * ncell * nc));
    if (!d) return perr(VD_ERR_ARG, "%s/Level_0/phi_D_00000 is truncated", dir);
    return VD_OK;
}
