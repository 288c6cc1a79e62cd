// osc_igf.cuh -- FP64 integrated-Green-function primitives, evaluated on the GPU.
//
// These are the indefinite integrals of OpenSpaceCharge's IGF method; the 8-corner
// difference of a primitive over a cell is the cell integral.  The log/atan terms cancel
// catastrophically at large offsets, so they stay in FP64 on every path.
#pragma once

#include <math.h>

namespace osc {

// \int 1/r dx dy dz  (code/open_spacecharge_mod.f90:741-747, lafun2)
__device__ __forceinline__ double igf_lafun2(double x, double y, double z) {
    const double r = sqrt(x * x + y * y + z * z);
    double t = -((z * z) * atan(x * y / (z * r))) / 2;
    t = t - ((y * y) * atan(x * z / (y * r))) / 2;
    t = t - ((x * x) * atan(y * z / (x * r))) / 2;
    t = t + y * z * log(x + r);
    t = t + x * z * log(y + r);
    t = t + x * y * log(z + r);
    return t;
}

// \int x/r^3 dx dy dz  (code/open_spacecharge_mod.f90:721-726, xlafun2)
__device__ __forceinline__ double igf_xlafun2(double x, double y, double z) {
    const double r = sqrt(x * x + y * y + z * z);
    return x * atan((y * z) / (r * x)) - z * log(r + y) + y * log((r - z) / (r + z)) / 2;
}

// Primitive of component icomp at (u,v,w): 0 phi, 1 Ex, 2 Ey, 3 Ez -- the argument
// permutations of osc_get_cgrn_freespace (code/open_spacecharge_mod.f90:683-686).
__device__ __forceinline__ double igf_primitive(int icomp, double u, double v, double w) {
    switch (icomp) {
    case 0: return igf_lafun2(u, v, w);
    case 1: return igf_xlafun2(u, v, w);
    case 2: return igf_xlafun2(v, w, u);
    default: return igf_xlafun2(w, u, v);
    }
}

// ---- legacy point-evaluated IGFs (code/open_spacecharge_core_mod.f90:189-428) ----------
__device__ __forceinline__ double igf_coulombfun(double u, double v, double w, double gam) {
    if (u == 0.0 && v == 0.0 && w == 0.0) return 0.0;
    return 1.0 / sqrt(u * u + v * v + (gam * w) * (gam * w));
}
__device__ __forceinline__ double igf_lafun(double x, double y, double z) {
    const double r = sqrt(x * x + y * y + z * z);
    double res = -0.5 * (z * z) * atan(x * y / (z * r));
    res = res - 0.5 * (y * y) * atan(x * z / (y * r));
    res = res - 0.5 * (x * x) * atan(y * z / (x * r));
    res = res + y * z * log(x + r);
    res = res + x * z * log(y + r);
    res = res + x * y * log(z + r);
    return res;
}
__device__ __forceinline__ double igf_xlafun(double x, double y, double z) {
    const double r = sqrt(x * x + y * y + z * z);
    double res = z - x * atan(z / x) + x * atan(y * z / (x * r));
    if (y + r != 0) res = res - z * log(y + r);
    if (z + r != 0) res = res - y * log(z + r);
    return res;
}
__device__ __forceinline__ double igf_ylafun(double x, double y, double z) {
    const double r = sqrt(x * x + y * y + z * z);
    double res = x - y * atan(x / y) + y * atan(z * x / (y * r));
    if (z + r != 0) res = res - x * log(z + r);
    if (x + r != 0) res = res - z * log(x + r);
    return res;
}
__device__ __forceinline__ double igf_zlafun(double x, double y, double z) {
    const double r = sqrt(x * x + y * y + z * z);
    double res = y - z * atan(y / z) + z * atan(x * y / (z * r));
    if (x + r != 0) res = res - y * log(x + r);
    if (y + r != 0) res = res - x * log(y + r);
    return res;
}
__device__ __forceinline__ double igf_legacy_prim(int icomp, double x, double y, double z) {
    switch (icomp) {
    case 0: return igf_lafun(x, y, z);
    case 1: return igf_xlafun(x, y, z);
    case 2: return igf_ylafun(x, y, z);
    default: return igf_zlafun(x, y, z);
    }
}
// igfcoulombfun / igfexfun / igfeyfun / igfezfun / coulombfun (core:205-372)
__device__ __forceinline__ double igf_point(int icomp, int igfflag, double u, double v, double w,
                                            double gam, double dx, double dy, double dz) {
    if (igfflag == 0) return icomp == 0 ? igf_coulombfun(u, v, w, gam) : 0.0;
    const double x1 = u - 0.5 * dx, x2 = u + 0.5 * dx;
    const double y1 = v - 0.5 * dy, y2 = v + 0.5 * dy;
    const double z1 = (w - 0.5 * dz) * gam, z2 = (w + 0.5 * dz) * gam;
    if (icomp != 0 && x1 < 0.0 && x2 > 0.0 && y1 < 0.0 && y2 > 0.0 && z1 < 0.0 && z2 > 0.0)
        return 0.0;
    double res = igf_legacy_prim(icomp, x2, y2, z2);
    res = res - igf_legacy_prim(icomp, x1, y2, z2);
    res = res - igf_legacy_prim(icomp, x2, y1, z2);
    res = res - igf_legacy_prim(icomp, x2, y2, z1);
    res = res - igf_legacy_prim(icomp, x1, y1, z1);
    res = res + igf_legacy_prim(icomp, x1, y1, z2);
    res = res + igf_legacy_prim(icomp, x1, y2, z1);
    res = res + igf_legacy_prim(icomp, x2, y1, z1);
    if (icomp == 0 || icomp == 3) return res / (dx * dy * dz * gam);
    return res / (dx * dy * dz);
}

}  // namespace osc
