// Host-side set-up of the sponge boundary: the strength field sigma of
// SpongeBC (src/SpongeBC.cpp:3-360), computed once from the mesh coordinates.
#include <cmath>
#include <string>

#include "mc3d_internal.h"

using namespace mc3d;

namespace {

// 0.068 s^2 + 0.845 s^8 ramp scaled by the strength (src/SpongeBC.cpp:105)
inline double ramp(double strength, double s) {
    return strength * (0.068 * std::pow(s, 2.0) + 0.845 * std::pow(s, 8.0));
}

}  // namespace

extern "C" int mc3d_sponge_sigma(const mc3d_config *cfg, const double *x, const double *y, const double *z,
                                 double *sigma) {
    if (!cfg || !x || !y || !z || !sigma) return fail(MC3D_ERR_ARG, "null argument");
    const long long n = (long long)cfg->Nx * cfg->Ny * cfg->Nz;
    if (n <= 0) return fail(MC3D_ERR_ARG, "empty grid");
    const double *X[3] = {x, y, z};
    double mn[3], mx[3];
    for (int d = 0; d < 3; d++) {
        mn[d] = 1e300;
        mx[d] = -1e300;
        for (long long i = 0; i < n; i++) {
            mn[d] = std::fmin(mn[d], X[d][i]);
            mx[d] = std::fmax(mx[d], X[d][i]);
        }
    }
    for (long long i = 0; i < n; i++) sigma[i] = 0.0;
    const double st = cfg->sponge_strength;
    const int *k = cfg->bc_kind;
    if (cfg->sponge_kind == MC3D_SPONGE_RECTILINEAR) {
        // initRectSpongeBC (src/SpongeBC.cpp:65-188), faces X0, X1, Y0, Y1, Z0, Z1
        for (int d = 0; d < 3; d++) {
            const double L0 = cfg->sponge_rect_perc[2 * d] * (mx[d] - mn[d]);
            const double L1 = cfg->sponge_rect_perc[2 * d + 1] * (mx[d] - mn[d]);
            if (k[2 * d] == MC3D_BC_SPONGE)
                for (long long i = 0; i < n; i++) {
                    double dd = X[d][i] - mn[d];
                    if (dd < L0) sigma[i] = std::fmax(ramp(st, (L0 - dd) / L0), sigma[i]);
                }
            if (k[2 * d + 1] == MC3D_BC_SPONGE)
                for (long long i = 0; i < n; i++) {
                    double dd = mx[d] - X[d][i];
                    if (dd < L1) sigma[i] = std::fmax(ramp(st, (X[d][i] - (mx[d] - L1)) / L1), sigma[i]);
                }
        }
        return MC3D_OK;
    }
    if (cfg->sponge_kind == MC3D_SPONGE_CYLINDRICAL) {
        // initCylSpongeBC (src/SpongeBC.cpp:190-262): axis along z, sponge on the Y1 face
        if (cfg->sponge_cyl_orient != 2)
            return fail(MC3D_ERR_CONFIG, "SPONGECYLINDRICAL SHAPE NEEDS TO BE IMPLEMENTED FOR ORIENT = " +
                                             std::to_string(cfg->sponge_cyl_orient));
        const double *ax = cfg->sponge_cyl_axis;
        const double rx = std::fmax(std::fabs(mn[0] - ax[0]), std::fabs(mx[0] - ax[0]));
        const double ry = std::fmax(std::fabs(mn[1] - ax[1]), std::fabs(mx[1] - ax[1]));
        const double rmax = std::fmax(rx, ry), rmin = cfg->sponge_rmin;
        if (k[3] == MC3D_BC_SPONGE)
            for (long long i = 0; i < n; i++) {
                double r = std::sqrt(std::pow(x[i] - ax[0], 2.0) + std::pow(y[i] - ax[1], 2.0));
                if (r > rmin) sigma[i] = std::fmax(ramp(st, (r - rmin) / (rmax - rmin)), sigma[i]);
            }
        return MC3D_OK;
    }
    return fail(MC3D_ERR_CONFIG, "unknown SPONGE.KIND");
}
