// writers.cu -- the line-out and plane files of the reference's test program
// (write_lines / write_plane, code/test_opensc.f90:237-295), filled by one batched
// interpolation each instead of one interpolate_field call per point.
//
// Files (in `dir`, or the working directory when dir is NULL or empty):
//   x_lineout.dat, y_lineout.dat, z_lineout.dat: x y z Ex Ey Ez per row, Fortran format
//     '(6(1pe14.7,1x))', points (i-1)*delta + min for i = nlo .. nhi-1 along one axis
//     through (xcent, ycent, zcent);
//   x_z_Ex_Ez_By.dat: x z Ex Ez By per row (list-directed), the plane y = 0, x fastest.
#include <cstdio>
#include <string>
#include <vector>

#include "abi_util.cuh"

using namespace osc;
using namespace osc_abi;

namespace {

// Fortran 1PE14.7: one digit before the point, seven after, exponent E+dd, or +ddd
// without the E when |exponent| > 99; right-justified in 14 columns.
void fmt_1pe14_7(double v, char out[15]) {
    char buf[64];
    if (v != v) {
        std::snprintf(out, 15, "%14s", "NaN");
        return;
    }
    if (v == 1.0 / 0.0 || v == -1.0 / 0.0) {
        std::snprintf(out, 15, "%14s", v > 0 ? "Infinity" : "-Infinity");
        return;
    }
    std::snprintf(buf, sizeof buf, "%.7E", v);  // d.dddddddE+xx or E+xxx
    std::string s(buf);
    const size_t e = s.find('E');
    std::string mant = s.substr(0, e), ex = s.substr(e + 1);
    const char sign = ex[0];
    std::string digits = ex.substr(1);
    while (digits.size() > 2 && digits[0] == '0') digits.erase(0, 1);
    std::string r = digits.size() <= 2 ? mant + "E" + sign + digits : mant + sign + digits;
    std::snprintf(out, 15, "%14s", r.c_str());
}

// List-directed REAL(8) output: 17 significant digits.
void fmt_list(double v, char *out, size_t n) { std::snprintf(out, n, " %24.16E", v); }

std::string join(const char *dir, const char *name) {
    std::string d = dir ? dir : "";
    if (d.empty()) return name;
    if (d.back() != '/') d += '/';
    return d + name;
}

}  // namespace

extern "C" {

int osc_format_1pe14_7(double v, char *out15) {
    if (!out15) return OSC_E_INVALID;
    fmt_1pe14_7(v, out15);
    return OSC_OK;
}

int osc_write_lines(osc_ctx *ctx, const osc_mesh3d *mesh, const double *efield, double xcent, double ycent,
                    double zcent, const char *dir) {
    if (!ctx) return OSC_E_INVALID;
    int n[3];
    TRY(mesh_dims(ctx, mesh, n));
    if (!efield) return bad(ctx, "efield");
    const char *names[3] = {"x_lineout.dat", "y_lineout.dat", "z_lineout.dat"};
    for (int ax = 0; ax < 3; ++ax) {
        const int64_t np = mesh->nhi[ax] - mesh->nlo[ax];  // i = nlo .. nhi-1 (last point skipped)
        std::vector<double> x(np), y(np), z(np), E(3 * (size_t)np);
        for (int64_t t = 0; t < np; ++t) {
            const int i = mesh->nlo[ax] + (int)t;
            double p[3] = {xcent, ycent, zcent};
            p[ax] = (i - 1) * mesh->delta[ax] + mesh->min[ax];
            x[t] = p[0];
            y[t] = p[1];
            z[t] = p[2];
        }
        int64_t ncl = 0;
        if (np > 0)
            TRY(osc_interpolate_field(ctx, mesh, efield, nullptr, np, x.data(), y.data(), z.data(), E.data(), nullptr,
                                      &ncl));
        const std::string path = join(dir, names[ax]);
        FILE *f = std::fopen(path.c_str(), "w");
        if (!f) return set_err(ctx, OSC_E_INVALID, "cannot open %s", path.c_str());
        for (int64_t t = 0; t < np; ++t) {
            const double row[6] = {x[t], y[t], z[t], E[3 * t], E[3 * t + 1], E[3 * t + 2]};
            for (int c = 0; c < 6; ++c) {
                char s[15];
                fmt_1pe14_7(row[c], s);
                std::fputs(s, f);
                std::fputc(' ', f);
            }
            std::fputc('\n', f);
        }
        std::fclose(f);
    }
    return OSC_OK;
}

int osc_write_plane(osc_ctx *ctx, const osc_mesh3d *mesh, const double *efield, const double *bfield,
                    const char *dir) {
    if (!ctx) return OSC_E_INVALID;
    int n[3];
    TRY(mesh_dims(ctx, mesh, n));
    if (!efield || !bfield) return bad(ctx, "efield and bfield");
    const int64_t nxp = mesh->nhi[0] - mesh->nlo[0], nzp = mesh->nhi[2] - mesh->nlo[2];
    const int64_t np = nxp * nzp;
    std::vector<double> x(np), y(np, 0.0), z(np), E(3 * (size_t)np), B(3 * (size_t)np);
    for (int64_t k = 0; k < nzp; ++k)
        for (int64_t i = 0; i < nxp; ++i) {
            const int64_t t = k * nxp + i;
            x[t] = (mesh->nlo[0] + i - 1) * mesh->delta[0] + mesh->min[0];
            z[t] = (mesh->nlo[2] + k - 1) * mesh->delta[2] + mesh->min[2];
        }
    int64_t ncl = 0;
    if (np > 0)
        TRY(osc_interpolate_field(ctx, mesh, efield, bfield, np, x.data(), y.data(), z.data(), E.data(), B.data(),
                                  &ncl));
    const std::string path = join(dir, "x_z_Ex_Ez_By.dat");
    FILE *f = std::fopen(path.c_str(), "w");
    if (!f) return set_err(ctx, OSC_E_INVALID, "cannot open %s", path.c_str());
    for (int64_t t = 0; t < np; ++t) {
        const double row[5] = {x[t], z[t], E[3 * t], E[3 * t + 2], B[3 * t + 1]};
        for (int c = 0; c < 5; ++c) {
            char s[40];
            fmt_list(row[c], s, sizeof s);
            std::fputs(s, f);
        }
        std::fputc('\n', f);
    }
    std::fclose(f);
    return OSC_OK;
}

}  // extern "C"
