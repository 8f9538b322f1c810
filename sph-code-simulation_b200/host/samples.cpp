// samples.cpp — deterministic initial conditions for the benchmark workloads.
//
// These are the inputs of the hot path, not part of it.  Each generator
// writes SoA arrays in the field order of include/sphgpu.h and returns the
// particle count; call once with fields == NULL to size the buffers.
//
//   sphgpu_sample_evrard       Evrard sphere, Solver::make_evrard
//                              (src/sample/evrard.cpp:13-87): N^3 lattice in
//                              [-1,1]^3 cut to the unit sphere, radius
//                              remapped r -> r^1.5, equal masses 1/Np,
//                              rho = 1/(2 pi r), u = 0.05 G, v = 0.
//   sphgpu_sample_shear_layer  3-D periodic shear layer in [0,1]x[0,1]x[0,Lz],
//                              the 2-D Kelvin-Helmholtz set-up of
//                              Solver::make_khi (src/sample/khi.cpp:12-73)
//                              extruded to 3-D with equal-mass lattices.
//   sphgpu_sample_shock_tube   3-D shock tube along x in [-0.5,0.5] x [0,Ly]^2,
//                              uniform lattice, left/right pressure states.
//   sphgpu_sample_sr_shock_tube  special-relativistic Sod tube of
//                              Solver::make_sr_sod (src/sample/sr_sod.cpp:15-
//                              199; Kitajima et al. 2025, sec. 3.1.1) in 3-D:
//                              left n = 1, P = 1 on a lattice of spacing dx,
//                              right n = 0.125, P = 0.1 on spacing 2 dx, so
//                              every particle carries the same baryon number
//                              nu = dx^3; v = 0, conserved S = 0 and
//                              e = gamma_lor H - P / (N c^2).
#include <cmath>
#include <cstdint>
#include <vector>

#include "sphgpu.h"

namespace {

void put(double* const* f, int k, int64_t i, double v)
{
    if(f && f[k]) f[k][i] = v;
}

}  // namespace

extern "C" {

int64_t sphgpu_sample_evrard(int N, double G, double gamma, double* const* f)
{
    const double dx = 2.0 / N;
    std::vector<double> px, py, pz;
    for(int i = 0; i < N; ++i) {
        for(int j = 0; j < N; ++j) {
            for(int k = 0; k < N; ++k) {
                double r[3] = {(i + 0.5) * dx - 1.0, (j + 0.5) * dx - 1.0, (k + 0.5) * dx - 1.0};
                const double r0 = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                if(r0 > 1.0) continue;
                if(r0 > 0.0) {
                    const double s = std::pow(r0, 1.5) / r0;
                    r[0] *= s;
                    r[1] *= s;
                    r[2] *= s;
                }
                px.push_back(r[0]);
                py.push_back(r[1]);
                pz.push_back(r[2]);
            }
        }
    }
    const int64_t n = (int64_t)px.size();
    if(!f) return n;
    const double mass = 1.0 / n;
    const double u = 0.05 * G;
    for(int64_t i = 0; i < n; ++i) {
        put(f, SPHGPU_F_POS_X, i, px[i]);
        put(f, SPHGPU_F_POS_Y, i, py[i]);
        put(f, SPHGPU_F_POS_Z, i, pz[i]);
        put(f, SPHGPU_F_MASS, i, mass);
        const double r = std::sqrt(px[i] * px[i] + py[i] * py[i] + pz[i] * pz[i]);
        const double dens = 1.0 / (2.0 * M_PI * r);
        put(f, SPHGPU_F_DENS, i, dens);
        put(f, SPHGPU_F_ENE, i, u);
        put(f, SPHGPU_F_PRES, i, (gamma - 1.0) * dens * u);
    }
    return n;
}

// Dense band 0.25 < y < 0.75: rho = 2, vx = -0.5 on a lattice of spacing
// dx * 2^(-1/3); outside: rho = 1, vx = +0.5 at spacing dx.  Lattice counts
// are rounded so both lattices tile the periodic box exactly; every particle
// has mass (total mass) / N.  P = 2.5 everywhere,
// vy = 0.025 sin(4 pi x) [exp(-(y-.25)^2 / 2 s^2) + exp(-(y-.75)^2 / 2 s^2)],
// s = 0.05.
int64_t sphgpu_sample_shear_layer(double dx, double lz, double gamma, double* const* f)
{
    struct Lat {
        int nx, ny, nz;
        double y0, ly, rho, vx;
    };
    const double dx2 = dx * std::pow(2.0, -1.0 / 3.0);
    Lat lats[3] = {
        {(int)std::lround(1.0 / dx), (int)std::lround(0.25 / dx), (int)std::lround(lz / dx), 0.0, 0.25, 1.0, 0.5},
        {(int)std::lround(1.0 / dx2), (int)std::lround(0.5 / dx2), (int)std::lround(lz / dx2), 0.25, 0.5, 2.0, -0.5},
        {(int)std::lround(1.0 / dx), (int)std::lround(0.25 / dx), (int)std::lround(lz / dx), 0.75, 0.25, 1.0, 0.5},
    };
    int64_t n = 0;
    for(auto& l : lats) n += (int64_t)l.nx * l.ny * l.nz;
    if(!f) return n;
    const double mass = (1.0 * 0.5 * lz + 2.0 * 0.5 * lz) / n;
    const double s2 = 0.05 * 0.05;
    int64_t i = 0;
    for(auto& l : lats) {
        const double hx = 1.0 / l.nx, hy = l.ly / l.ny, hz = lz / l.nz;
        for(int a = 0; a < l.nx; ++a) {
            for(int b = 0; b < l.ny; ++b) {
                for(int c = 0; c < l.nz; ++c, ++i) {
                    const double x = (a + 0.5) * hx, y = l.y0 + (b + 0.5) * hy, z = (c + 0.5) * hz;
                    put(f, SPHGPU_F_POS_X, i, x);
                    put(f, SPHGPU_F_POS_Y, i, y);
                    put(f, SPHGPU_F_POS_Z, i, z);
                    put(f, SPHGPU_F_VEL_X, i, l.vx);
                    put(f, SPHGPU_F_VEL_Y, i,
                        0.025 * std::sin(4.0 * M_PI * x)
                            * (std::exp(-(y - 0.25) * (y - 0.25) / (2 * s2)) + std::exp(-(y - 0.75) * (y - 0.75) / (2 * s2))));
                    put(f, SPHGPU_F_MASS, i, mass);
                    put(f, SPHGPU_F_DENS, i, l.rho);
                    put(f, SPHGPU_F_PRES, i, 2.5);
                    put(f, SPHGPU_F_ENE, i, 2.5 / ((gamma - 1.0) * l.rho));
                }
            }
        }
    }
    return n;
}

// Tube x in [-0.5, 0.5], y, z in [0, ly]; lattice spacing dx (rounded to tile
// the box); rho = 1 on both sides, p = p_left for x < 0 and p_right otherwise.
int64_t sphgpu_sample_shock_tube(double dx, double ly, double p_left, double p_right,
                                 double gamma, double* const* f)
{
    const int nx = (int)std::lround(1.0 / dx), ny = (int)std::lround(ly / dx);
    const int64_t n = (int64_t)nx * ny * ny;
    if(!f) return n;
    const double hx = 1.0 / nx, hy = ly / ny;
    const double mass = 1.0 * ly * ly / n;
    int64_t i = 0;
    for(int a = 0; a < nx; ++a) {
        for(int b = 0; b < ny; ++b) {
            for(int c = 0; c < ny; ++c, ++i) {
                const double x = -0.5 + (a + 0.5) * hx;
                const double p = x < 0.0 ? p_left : p_right;
                put(f, SPHGPU_F_POS_X, i, x);
                put(f, SPHGPU_F_POS_Y, i, (b + 0.5) * hy);
                put(f, SPHGPU_F_POS_Z, i, (c + 0.5) * hy);
                put(f, SPHGPU_F_MASS, i, mass);
                put(f, SPHGPU_F_DENS, i, 1.0);
                put(f, SPHGPU_F_PRES, i, p);
                put(f, SPHGPU_F_ENE, i, p / ((gamma - 1.0) * 1.0));
            }
        }
    }
    return n;
}

// Special-relativistic Sod tube, x in [-0.5, 0.5], y, z in [0, ly]; ly / (2 dx)
// must be a whole number for the right lattice to tile the box.
int64_t sphgpu_sample_sr_shock_tube(double dx, double ly, double gamma, double c_speed, double* const* f)
{
    const int nxl = (int)std::lround(0.5 / dx), nyl = (int)std::lround(ly / dx);
    const int nxr = nxl / 2, nyr = nyl / 2;
    const int64_t nl = (int64_t)nxl * nyl * nyl, nr = (int64_t)nxr * nyr * nyr;
    if(!f) return nl + nr;
    const double c2 = c_speed * c_speed;
    int64_t i = 0;
    for(int side = 0; side < 2; ++side) {
        const int nx = side ? nxr : nxl, ny = side ? nyr : nyl;
        const double hx = 0.5 / nx, hy = ly / ny;
        const double n = side ? 0.125 : 1.0, P = side ? 0.1 : 1.0;
        // one baryon number for both sides: nu = n x (volume per particle)
        const double nu = 1.0 * (0.5 / nxl) * (ly / nyl) * (ly / nyl);
        const double u = P / ((gamma - 1.0) * n);
        const double H = 1.0 + u / c2 + P / (n * c2);
        const double N = 1.0 * n;
        const double e = 1.0 * H - P / (N * c2);
        for(int a = 0; a < nx; ++a) {
            for(int b = 0; b < ny; ++b) {
                for(int c = 0; c < ny; ++c, ++i) {
                    put(f, SPHGPU_F_POS_X, i, (side ? 0.0 : -0.5) + (a + 0.5) * hx);
                    put(f, SPHGPU_F_POS_Y, i, (b + 0.5) * hy);
                    put(f, SPHGPU_F_POS_Z, i, (c + 0.5) * hy);
                    put(f, SPHGPU_F_MASS, i, nu);
                    put(f, SPHGPU_F_DENS, i, n);
                    put(f, SPHGPU_F_PRES, i, P);
                    put(f, SPHGPU_F_ENE, i, u);
                    put(f, SPHGPU_F_SR_E, i, e);
                    put(f, SPHGPU_F_SR_N, i, N);
                    put(f, SPHGPU_F_SR_NU, i, nu);
                    put(f, SPHGPU_F_SR_GAMMA_LOR, i, 1.0);
                }
            }
        }
    }
    return nl + nr;
}

}  // extern "C"
