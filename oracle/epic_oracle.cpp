// ORACLE -- test infrastructure only (see oracle_core.hpp for the pinning
// statement).  CPU FP64 restatement of the reference EPIC 3-D parcel step on a
// single MPI rank, exported through the same C ABI as the product
// (include/epic_gpu.h) with the prefix epic_oracle_ instead of epic_gpu_.
//
// Single-rank semantics of the reference's MPI calls:
//   * field halo accumulate / fill (field_mpi.f90) = periodic index wrap in x, y
//   * parcel_communicate (parcel_mpi.f90:101-126) = apply_periodic_bc
//   * reverse_x/y (mpi_reverse.f90:332-398) = local index map kx -> nx-1-kx
//   * nearest-search neighbour exchange (parcel_nearest.f90:1466-1621) =
//     periodic copies of boundary small parcels appended in receive order
//   * MPI_Allreduce / mpi_blocking_reduce = plain sums / max
#include "oracle_core.hpp"
#include "../include/epic_gpu.h"

#include <algorithm>
#include <memory>
#include <numeric>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace oracle;

namespace {

// Indices of the velocity gradient tensor (fields.f90:52-60), 0-based.
enum { I_DUDX = 0, I_DUDY, I_DUDZ, I_DVDX, I_DVDY, I_DVDZ, I_DWDX, I_DWDY };

struct Ctx {
    epic_cfg cfg;
    std::string err;
    int nx, ny, nz;
    // parameters.f90:93-165
    double lower[3], extent[3], upper[3], extenti[3], dx[3], dxi[3];
    double vdomain, vdomaini, vcell, vcelli, ncelli, ngridi, center[3], hl[3], hli[3];
    double vmin, amax;
    long ncell, ngrid;
    // physics.f90:170-185
    double glat, lambda_c, q_0, f_cor[3];
    bool bndry_zeta_zero[2];
    // ls_rk.f90:32-54
    std::vector<double> ca, cb;
    int n_stages;
    // parcels (parcel_container.f90:18-106, parcel_ellipsoid.f90:36-134)
    long n = 0;
    std::vector<double> pos, vor, B, vol, buoy, hum;     // (3,n) (3,n) (5,n) (n) (n) (n)
    std::vector<double> dpos, dvor, strain, dB;          // (3,n) (3,n) (8,n) (5,n)
    std::vector<double> Vetas, Vtaus;                    // (3,n) (3,n)
    // labels (ENABLE_LABELS, parcel_container.f90:41-57): cfg.labels = 1
    std::vector<int64_t> label;
    std::vector<double> dil;
    long merge_calls = 0;
    // fields (fields.f90:21-51): (nz+3) x ny x nx, z fastest, x slowest
    long nzh, fsz;
    std::vector<double> velog[3], vortg[3], vtend[3], velgradg[8];
    std::vector<double> tbuoyg, dbuoyg, humg, volg;
    std::vector<int> nparg, nsparg;
    // spectral tables (sta3dfft.f90:52-109, inversion_utils.f90:79-253)
    std::vector<double> rkx, hrkx, rky, hrky, rkz, rkzi;
    std::vector<double> k2l2, k2l2i;                     // (ny, nx) : ky + ny*kx
    std::vector<double> filt, green, phim, phip, dphim, dphip, thetam, thetap, dthetam, dthetap;
    std::vector<double> etdv, htdv;                      // (0:nz, ny, nx)
    std::vector<double> gamtop, gambot;
    double dz, dzi, hdzi, dzisq, ap;
    RealFFT fx, fy;
    TrigTransform tz;
    // parcel_correction.f90:29
    double vor_bar[3] = {0, 0, 0};
    // last merge pairs (1-based)
    std::vector<int> last_isma, last_iclo;
    // counters for diagnostics
    long n_parcel_splits = 0, n_parcel_merges = 0, n_big_close = 0;
    double t = 0.0;
    // surface fluxes (bndry_fluxes.f90:25-36): (ny, nx), y fastest, scaled by 2/dz
    bool l_enable_flux = false;
    std::vector<double> binc, hinc;
    double zdepth = 0.0;
    // strain magnitude of parcel_damp (fields.f90 strain_mag)
    std::vector<double> strain_mag;

    long fi(int iz, int iy, int ix) const { return ((long)ix * ny + iy) * nzh + (iz + 1); }
    long si(int iz, int ky, int kx) const { return ((long)kx * ny + ky) * (nz + 1) + iz; }
    long hi2(int ky, int kx) const { return (long)kx * ny + ky; }
    int wrapx(int i) const { i %= nx; return i < 0 ? i + nx : i; }
    int wrapy(int j) const { j %= ny; return j < 0 ? j + ny : j; }
};

// ---------------------------------------------------------------------------
// parameters.f90:93-165, physics.f90:170-185
void update_parameters(Ctx& c) {
    const epic_cfg& g = c.cfg;
    c.nx = g.nx; c.ny = g.ny; c.nz = g.nz;
    int nn[3] = {g.nx, g.ny, g.nz};
    for (int k = 0; k < 3; ++k) {
        c.lower[k] = g.lower[k];
        c.extent[k] = g.extent[k];
        c.upper[k] = c.lower[k] + c.extent[k];
        c.extenti[k] = one / c.extent[k];
        c.dx[k] = c.extent[k] / (double)nn[k];
        c.dxi[k] = one / c.dx[k];
    }
    c.vdomain = c.extent[0] * c.extent[1] * c.extent[2];
    c.vdomaini = one / c.vdomain;
    c.vcell = c.dx[0] * c.dx[1] * c.dx[2];
    c.vcelli = one / c.vcell;
    c.ncell = (long)g.nx * g.ny * g.nz;
    c.ncelli = one / (double)c.ncell;
    c.ngrid = (long)g.nx * g.ny * (g.nz + 1);
    c.ngridi = one / (double)c.ngrid;
    for (int k = 0; k < 3; ++k) {
        c.center[k] = f12 * (c.lower[k] + c.upper[k]);
        c.hl[k] = c.extent[k] / two;
        c.hli[k] = one / c.hl[k];
    }
    c.vmin = c.vcell / g.min_vratio;
    c.amax = std::pow(f34 * fpi, f13) * std::min(c.dx[0], std::min(c.dx[1], c.dx[2]));
    c.glat = g.gravity * g.L_v / (g.c_p * g.theta_0);
    c.lambda_c = one / g.height_c;
    c.q_0 = g.q_0;
    if (g.l_planetary_vorticity) {
        double lat_ref = g.lat_degrees * (one / (180.0 * fpi));
        c.f_cor[0] = zero;
        c.f_cor[1] = two * g.ang_vel * std::cos(lat_ref);
        c.f_cor[2] = two * g.ang_vel * std::sin(lat_ref);
    } else {
        c.f_cor[0] = c.f_cor[1] = c.f_cor[2] = zero;
    }
    c.bndry_zeta_zero[0] = g.bndry_zeta_zero[0] != 0;
    c.bndry_zeta_zero[1] = g.bndry_zeta_zero[1] != 0;
    // ls_rk.f90:32-54, 64-84
    if (g.rk_order == 4) {
        c.ca = {-567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0, 0.0};
        c.cb = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                2277821191437.0 / 14882151754819.0};
        c.n_stages = 5;
    } else if (g.rk_order == 3) {
        c.ca = {-5.0 / 9.0, -153.0 / 128.0, 0.0};
        c.cb = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
        c.n_stages = 3;
    } else {
        throw OracleError(EPIC_ERR_CONFIG, "Only third and fourth order RK supported.");
    }
}

// sta3dfft.f90:52-109 + inversion_utils.f90:79-253 (init_inversion)
void set_hyperbolic_functions(Ctx& c, int kx, int ky, const std::vector<double>& zm,
                              const std::vector<double>& zp) {
    int nz = c.nz;
    double kl = std::sqrt(c.k2l2[c.hi2(ky, kx)]);
    double fac = kl * c.extent[2];
    double ef = std::exp(-fac);
    double div = one / (one - ef * ef);
    double k2ifac = f12 * c.k2l2i[c.hi2(ky, kx)];
    for (int iz = 0; iz <= nz; ++iz) {
        double Lm = kl * zm[iz], Lp = kl * zp[iz];
        double ep = std::exp(-Lp), em = std::exp(-Lm);
        long s = c.si(iz, ky, kx);
        c.phim[s] = div * (ep - ef * em);
        c.phip[s] = div * (em - ef * ep);
        c.dphim[s] = -kl * div * (ep + ef * em);
        c.dphip[s] = kl * div * (em + ef * ep);
        double Q = div * (one + ef * ef);
        double R = div * two * ef;
        c.thetam[s] = k2ifac * (R * Lm * c.phip[s] - Q * Lp * c.phim[s]);
        c.thetap[s] = k2ifac * (R * Lp * c.phim[s] - Q * Lm * c.phip[s]);
        c.dthetam[s] = -k2ifac * ((Q * Lp - one) * c.dphim[s] - R * Lm * c.dphip[s]);
        c.dthetap[s] = -k2ifac * ((Q * Lm - one) * c.dphip[s] - R * Lp * c.dphim[s]);
    }
}

void init_inversion(Ctx& c) {
    int nx = c.nx, ny = c.ny, nz = c.nz;
    c.fx.init(nx); c.fy.init(ny); c.tz.init(nz);
    int nwx = nx / 2, nwy = ny / 2;
    c.hrkx.assign(nx + 1, 0.0); c.hrky.assign(ny + 1, 0.0);
    for (int k = 1; k <= nx; ++k) c.hrkx[k] = (pi / c.extent[0]) * (double)k;   // sta2dfft.f90:63-67
    for (int k = 1; k <= ny; ++k) c.hrky[k] = (pi / c.extent[1]) * (double)k;
    c.rkx.assign(nx, 0.0); c.rky.assign(ny, 0.0);
    for (int kx = 1; kx <= nwx - 1; ++kx) { c.rkx[kx] = c.hrkx[2 * kx]; c.rkx[nx - kx] = c.hrkx[2 * kx]; }
    c.rkx[nwx] = c.hrkx[nx];
    for (int ky = 1; ky <= nwy - 1; ++ky) { c.rky[ky] = c.hrky[2 * ky]; c.rky[ny - ky] = c.hrky[2 * ky]; }
    c.rky[nwy] = c.hrky[ny];
    c.rkz.assign(nz + 1, 0.0); c.rkzi.assign(nz + 1, 0.0);
    for (int i = 1; i <= nz; ++i) c.rkz[i] = (pi / c.extent[2]) * (double)i;      // deriv1d.f90:12-33
    for (int i = 1; i <= nz - 1; ++i) c.rkzi[i] = one / c.rkz[i];

    c.dz = c.dx[2]; c.dzi = c.dxi[2]; c.dzisq = c.dxi[2] * c.dxi[2]; c.hdzi = f12 * c.dxi[2];
    long hs = (long)nx * ny, ss = hs * (nz + 1);
    c.k2l2.assign(hs, 0.0); c.k2l2i.assign(hs, 0.0);
    for (int kx = 0; kx < nx; ++kx)
        for (int ky = 0; ky < ny; ++ky) c.k2l2[c.hi2(ky, kx)] = c.rkx[kx] * c.rkx[kx] + c.rky[ky] * c.rky[ky];
    c.k2l2[c.hi2(0, 0)] = one;
    for (long h = 0; h < hs; ++h) c.k2l2i[h] = one / c.k2l2[h];
    c.k2l2[c.hi2(0, 0)] = zero; c.k2l2i[c.hi2(0, 0)] = zero;

    // Hou and Li filter (inversion_utils.f90:129-150)
    double kxmaxi = one / *std::max_element(c.rkx.begin(), c.rkx.end());
    double kymaxi = one / *std::max_element(c.rky.begin(), c.rky.end());
    double kzmaxi = one / *std::max_element(c.rkz.begin(), c.rkz.end());
    std::vector<double> skx(nx), sky(ny), skz(nz + 1);
    for (int k = 0; k < nx; ++k) skx[k] = -36.0 * powi(kxmaxi * c.rkx[k], 36);
    for (int k = 0; k < ny; ++k) sky[k] = -36.0 * powi(kymaxi * c.rky[k], 36);
    for (int k = 0; k <= nz; ++k) skz[k] = -36.0 * powi(kzmaxi * c.rkz[k], 36);
    c.filt.assign(ss, 0.0);
    for (int kx = 0; kx < nx; ++kx)
        for (int ky = 0; ky < ny; ++ky) {
            double f0 = std::exp(skx[kx] + sky[ky]);
            c.filt[c.si(0, ky, kx)] = f0;
            c.filt[c.si(nz, ky, kx)] = f0;
            for (int kz = 1; kz <= nz - 1; ++kz) c.filt[c.si(kz, ky, kx)] = f0 * std::exp(skz[kz]);
        }
    for (int kz = 0; kz <= nz; ++kz) c.filt[c.si(kz, 0, 0)] = one;

    // Green function (inversion_utils.f90:168-175)
    c.green.assign(ss, 0.0);
    for (int kx = 0; kx < nx; ++kx)
        for (int ky = 0; ky < ny; ++ky) {
            long h = c.hi2(ky, kx);
            for (int kz = 1; kz <= nz; ++kz) c.green[c.si(kz, ky, kx)] = -one / (c.k2l2[h] + c.rkz[kz] * c.rkz[kz]);
            c.green[c.si(0, ky, kx)] = -c.k2l2i[h];
        }

    std::vector<double> zm(nz + 1), zp(nz + 1);
    for (int iz = 0; iz <= nz; ++iz) {
        double z = c.lower[2] + c.dx[2] * (double)iz;
        zm[iz] = c.upper[2] - z;
        zp[iz] = z - c.lower[2];
    }
    for (auto* v : {&c.phim, &c.phip, &c.dphim, &c.dphip, &c.thetam, &c.thetap, &c.dthetam, &c.dthetap})
        v->assign(ss, 0.0);
    for (int kx = 0; kx < nx; ++kx)
        for (int ky = 1; ky < ny; ++ky) set_hyperbolic_functions(c, kx, ky, zm, zp);
    for (int kx = 1; kx < nx; ++kx) set_hyperbolic_functions(c, kx, 0, zm, zp);
    std::vector<double> phip00(nz + 1);
    for (int iz = 0; iz <= nz; ++iz) {
        long s = c.si(iz, 0, 0);
        c.phim[s] = zm[iz] / c.extent[2];
        c.phip[s] = zp[iz] / c.extent[2];
        c.dphim[s] = -one / c.extent[2];
        c.dphip[s] = one / c.extent[2];
        c.thetam[s] = c.thetap[s] = c.dthetam[s] = c.dthetap[s] = zero;
        phip00[iz] = c.phip[s];
    }
    c.gamtop.assign(nz + 1, 0.0); c.gambot.assign(nz + 1, 0.0);
    for (int iz = 0; iz <= nz; ++iz) c.gamtop[iz] = f12 * c.extent[2] * (phip00[iz] * phip00[iz] - f13);
    for (int iz = 0; iz <= nz; ++iz) c.gambot[iz] = c.gamtop[nz - iz];

    // tridiagonal coefficients (inversion_utils.f90:230-250)
    c.ap = c.dzisq;
    c.etdv.assign(ss, 0.0); c.htdv.assign(ss, 0.0);
    for (int kx = 0; kx < nx; ++kx)
        for (int ky = 0; ky < ny; ++ky) {
            double a0 = -two * c.dzisq - c.k2l2[c.hi2(ky, kx)];
            c.htdv[c.si(0, ky, kx)] = one / a0;
            c.etdv[c.si(0, ky, kx)] = -two * c.ap * c.htdv[c.si(0, ky, kx)];
            for (int iz = 1; iz <= nz - 1; ++iz) {
                c.htdv[c.si(iz, ky, kx)] = one / (a0 + c.ap * c.etdv[c.si(iz - 1, ky, kx)]);
                c.etdv[c.si(iz, ky, kx)] = -c.ap * c.htdv[c.si(iz, ky, kx)];
            }
            if (kx == 0 && ky == 0) c.etdv[c.si(nz - 1, 0, 0)] = zero;
            c.htdv[c.si(nz, ky, kx)] = one / (a0 + two * c.ap * c.etdv[c.si(nz - 1, ky, kx)]);
        }
    for (int iz = 0; iz <= nz; ++iz) { c.htdv[c.si(iz, 0, 0)] = zero; c.etdv[c.si(iz, 0, 0)] = zero; }
}

// ---------------------------------------------------------------------------
// Semi-spectral helpers.  sp arrays are (0:nz, ny, nx) z fastest.
typedef std::vector<double> Arr;

// fftxyp2s (sta3dfft.f90:134-191): y transform then x transform of fp(0:nz).
void fftxyp2s(Ctx& c, const Arr& fp, Arr& fs) {
    int nx = c.nx, ny = c.ny, nz = c.nz;
    fs.assign((size_t)nx * ny * (nz + 1), 0.0);
#pragma omp parallel for schedule(static)
    for (int iz = 0; iz <= nz; ++iz) {
        std::vector<double> line(std::max(nx, ny));
        for (int ix = 0; ix < nx; ++ix) {
            for (int iy = 0; iy < ny; ++iy) line[iy] = fp[c.fi(iz, iy, ix)];
            c.fy.forfft(line.data());
            for (int iy = 0; iy < ny; ++iy) fs[c.si(iz, iy, ix)] = line[iy];
        }
        for (int ky = 0; ky < ny; ++ky) {
            for (int ix = 0; ix < nx; ++ix) line[ix] = fs[c.si(iz, ky, ix)];
            c.fx.forfft(line.data());
            for (int ix = 0; ix < nx; ++ix) fs[c.si(iz, ky, ix)] = line[ix];
        }
    }
}

// fftxys2p (sta3dfft.f90:196-257): writes fp(0:nz) only.
void fftxys2p(Ctx& c, const Arr& fs, Arr& fp) {
    int nx = c.nx, ny = c.ny, nz = c.nz;
    Arr tmp((size_t)nx * ny * (nz + 1));
#pragma omp parallel for schedule(static)
    for (int iz = 0; iz <= nz; ++iz) {
        std::vector<double> line(std::max(nx, ny));
        for (int ky = 0; ky < ny; ++ky) {
            for (int kx = 0; kx < nx; ++kx) line[kx] = fs[c.si(iz, ky, kx)];
            c.fx.revfft(line.data());
            for (int ix = 0; ix < nx; ++ix) tmp[c.si(iz, ky, ix)] = line[ix];
        }
        for (int ix = 0; ix < nx; ++ix) {
            for (int ky = 0; ky < ny; ++ky) line[ky] = tmp[c.si(iz, ky, ix)];
            c.fy.revfft(line.data());
            for (int iy = 0; iy < ny; ++iy) fp[c.fi(iz, iy, ix)] = line[iy];
        }
    }
}

// diffx (sta3dfft.f90:301-337) with reverse_x (mpi_reverse.f90:332-363):
// ds(kx) = si * hrkx(min(2kx, 2(nx-kx))) * fs(nx-kx).
void diffx(Ctx& c, const Arr& fs, Arr& ds) {
    int nx = c.nx, ny = c.ny, nz = c.nz, nwx = nx / 2;
    ds.assign(fs.size(), 0.0);
    for (int kx = 1; kx < nx; ++kx) {
        int dkx = std::min(2 * kx, 2 * (nx - kx));
        double sgn = (kx >= nwx + 1) ? 1.0 : -1.0;
        double f = sgn * c.hrkx[dkx];
        for (int ky = 0; ky < ny; ++ky)
            for (int iz = 0; iz <= nz; ++iz) ds[c.si(iz, ky, kx)] = f * fs[c.si(iz, ky, nx - kx)];
    }
    if (nx % 2 == 0)
        for (int ky = 0; ky < ny; ++ky)
            for (int iz = 0; iz <= nz; ++iz) ds[c.si(iz, ky, nwx)] = zero;
}

// diffy (sta3dfft.f90:339-374)
void diffy(Ctx& c, const Arr& fs, Arr& ds) {
    int nx = c.nx, ny = c.ny, nz = c.nz, nwy = ny / 2;
    ds.assign(fs.size(), 0.0);
    for (int ky = 1; ky < ny; ++ky) {
        int dky = std::min(2 * ky, 2 * (ny - ky));
        double sgn = (ky >= nwy + 1) ? 1.0 : -1.0;
        double f = sgn * c.hrky[dky];
        for (int kx = 0; kx < nx; ++kx)
            for (int iz = 0; iz <= nz; ++iz) ds[c.si(iz, ky, kx)] = f * fs[c.si(iz, ny - ky, kx)];
    }
    if (ny % 2 == 0)
        for (int kx = 0; kx < nx; ++kx)
            for (int iz = 0; iz <= nz; ++iz) ds[c.si(iz, nwy, kx)] = zero;
}

// field_decompose_semi_spectral (inversion_utils.f90:370-401)
void field_decompose_semi_spectral(Ctx& c, Arr& s) {
    int nx = c.nx, ny = c.ny, nz = c.nz;
#pragma omp parallel for schedule(static)
    for (int kx = 0; kx < nx; ++kx)
        for (int ky = 0; ky < ny; ++ky) {
            double* p = &s[c.si(0, ky, kx)];
            long t = c.si(0, ky, kx);
            for (int iz = 1; iz <= nz - 1; ++iz)
                p[iz] = p[iz] - (p[0] * c.phim[t + iz] + p[nz] * c.phip[t + iz]);
            double top = p[nz];
            c.tz.dst(p + 1);
            p[nz] = top;
        }
}

// field_combine_semi_spectral (inversion_utils.f90:421-456)
void field_combine_semi_spectral(Ctx& c, Arr& s) {
    int nx = c.nx, ny = c.ny, nz = c.nz;
#pragma omp parallel for schedule(static)
    for (int kx = 0; kx < nx; ++kx)
        for (int ky = 0; ky < ny; ++ky) {
            double* p = &s[c.si(0, ky, kx)];
            long t = c.si(0, ky, kx);
            double top = p[nz];
            p[nz] = zero;
            c.tz.dst(p + 1);
            p[nz] = top;
            for (int iz = 1; iz <= nz - 1; ++iz)
                p[iz] = p[iz] + p[0] * c.phim[t + iz] + p[nz] * c.phip[t + iz];
        }
}

// field_decompose_physical (inversion_utils.f90:358-366)
void field_decompose_physical(Ctx& c, const Arr& fc, Arr& sf) {
    fftxyp2s(c, fc, sf);
    field_decompose_semi_spectral(c, sf);
}

// field_combine_physical (inversion_utils.f90:405-417)
void field_combine_physical(Ctx& c, const Arr& sf, Arr& fc) {
    Arr sfc = sf;
    field_combine_semi_spectral(c, sfc);
    fftxys2p(c, sfc, fc);
}

// central_diffz_semi_spectral (inversion_utils.f90:460-480)
void central_diffz_semi_spectral(Ctx& c, const Arr& fs, Arr& ds) {
    int nx = c.nx, ny = c.ny, nz = c.nz;
    ds.assign(fs.size(), 0.0);
    for (int kx = 0; kx < nx; ++kx)
        for (int ky = 0; ky < ny; ++ky) {
            long t = c.si(0, ky, kx);
            ds[t] = c.dzi * (fs[t + 1] - fs[t]);
            ds[t + nz] = c.dzi * (fs[t + nz] - fs[t + nz - 1]);
            for (int iz = 1; iz <= nz - 1; ++iz) ds[t + iz] = (fs[t + iz + 1] - fs[t + iz - 1]) * c.hdzi;
        }
}

// central_diffz (inversion_utils.f90:485-510), physical space incl. halo rows
void central_diffz(Ctx& c, const Arr& f, Arr& df) {
    int nx = c.nx, ny = c.ny, nz = c.nz;
    df.assign(f.size(), 0.0);
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy) {
            long t = c.fi(0, iy, ix);
            df[t] = c.dzi * (f[t + 1] - f[t]);
            df[t + nz] = c.dzi * (f[t + nz] - f[t + nz - 1]);
            for (int iz = 1; iz <= nz - 1; ++iz) df[t + iz] = (f[t + iz + 1] - f[t + iz - 1]) * c.hdzi;
            df[t - 1] = two * df[t] - df[t + 1];
            df[t + nz + 1] = two * df[t + nz] - df[t + nz - 1];
        }
}

// diffz (inversion_utils.f90:523-559): d/dz of a field in the decomposed
// semi-spectral form (linear part through dphim / dphip, the sine series
// through rkz and a cosine transform), returned decomposed.  Not called by
// the step; its unit tests (test_mpi_diffz0..5) pin the decomposition.
void diffz(Ctx& c, const Arr& fs, Arr& ds) {
    int nx = c.nx, ny = c.ny, nz = c.nz;
    ds.assign(fs.size(), 0.0);
    std::vector<double> as(nz + 1);
    for (int kx = 0; kx < nx; ++kx)
        for (int ky = 0; ky < ny; ++ky) {
            long t = c.si(0, ky, kx);
            for (int iz = 0; iz <= nz; ++iz) ds[t + iz] = fs[t] * c.dphim[t + iz] + fs[t + nz] * c.dphip[t + iz];
            as[0] = zero;
            for (int kz = 1; kz <= nz - 1; ++kz) as[kz] = c.rkz[kz] * fs[t + kz];
            as[nz] = zero;
            c.tz.dct(as.data());
            for (int iz = 0; iz <= nz; ++iz) ds[t + iz] = ds[t + iz] + as[iz];
        }
    field_decompose_semi_spectral(c, ds);
}

// lapinv1 (inversion_utils.f90:567-589)
void lapinv1(Ctx& c, Arr& fs) {
    int nx = c.nx, ny = c.ny, nz = c.nz;
#pragma omp parallel for schedule(static)
    for (int kx = 0; kx < nx; ++kx)
        for (int ky = 0; ky < ny; ++ky) {
            long t = c.si(0, ky, kx);
            double* f = &fs[t];
            const double* h = &c.htdv[t];
            const double* e = &c.etdv[t];
            std::vector<double> rs(f, f + nz + 1);
            f[0] = rs[0] * h[0];
            for (int iz = 1; iz <= nz - 1; ++iz) f[iz] = (rs[iz] - c.ap * f[iz - 1]) * h[iz];
            f[nz] = (rs[nz] - two * c.ap * f[nz - 1]) * h[nz];
            for (int iz = nz - 1; iz >= 0; --iz) f[iz] = e[iz] * f[iz + 1] + f[iz];
        }
    for (int iz = 0; iz <= nz; ++iz) fs[c.si(iz, 0, 0)] = zero;
}

// z halo helpers
void extrap_halo(Ctx& c, Arr& f) {
    for (int ix = 0; ix < c.nx; ++ix)
        for (int iy = 0; iy < c.ny; ++iy) {
            long t = c.fi(0, iy, ix);
            f[t - 1] = two * f[t] - f[t + 1];
            f[t + c.nz + 1] = two * f[t + c.nz] - f[t + c.nz - 1];
        }
}
void antisym_halo(Ctx& c, Arr& f) {
    for (int ix = 0; ix < c.nx; ++ix)
        for (int iy = 0; iy < c.ny; ++iy) {
            long t = c.fi(0, iy, ix);
            f[t - 1] = -f[t + 1];
            f[t + c.nz + 1] = -f[t + c.nz - 1];
        }
}

// vel2vgrad (inversion.f90:259-317)
void vel2vgrad(Ctx& c, Arr svel[3]) {
    Arr ds;
    diffx(c, svel[0], ds); fftxys2p(c, ds, c.velgradg[I_DUDX]);
    diffy(c, svel[0], ds); fftxys2p(c, ds, c.velgradg[I_DUDY]);
    diffx(c, svel[2], ds); fftxys2p(c, ds, c.velgradg[I_DWDX]);
    extrap_halo(c, c.velgradg[I_DUDX]);
    extrap_halo(c, c.velgradg[I_DUDY]);
    antisym_halo(c, c.velgradg[I_DWDX]);
    diffy(c, svel[1], ds); fftxys2p(c, ds, c.velgradg[I_DVDY]);
    diffy(c, svel[2], ds); fftxys2p(c, ds, c.velgradg[I_DWDY]);
    extrap_halo(c, c.velgradg[I_DVDY]);
    antisym_halo(c, c.velgradg[I_DWDY]);
    for (long i = 0; i < c.fsz; ++i) {
        c.velgradg[I_DUDZ][i] = c.velgradg[I_DWDX][i] + c.vortg[1][i];
        c.velgradg[I_DVDX][i] = c.velgradg[I_DUDY][i] + c.vortg[2][i];
        c.velgradg[I_DVDZ][i] = c.velgradg[I_DWDY][i] - c.vortg[0][i];
    }
}

// vor2vel (inversion.f90:25-254)
void vor2vel(Ctx& c) {
    int nx = c.nx, ny = c.ny, nz = c.nz;
    long ss = (long)nx * ny * (nz + 1);
    Arr as(ss), bs(ss), ds(ss), es(ss), cs(ss), svor[3], svel[3];
    std::vector<double> ubar(nz + 1), vbar(nz + 1);
    for (int nc = 0; nc < 3; ++nc) {
        field_decompose_physical(c, c.vortg[nc], svor[nc]);
        for (long i = 0; i < ss; ++i) svor[nc][i] = c.filt[i] * svor[nc][i];
    }
    // solenoidality (:43-87)
    diffx(c, svor[1], as);
    diffy(c, svor[0], bs);
    for (long i = 0; i < ss; ++i) ds[i] = as[i] - bs[i];
    cs = svor[2];
    field_combine_semi_spectral(c, cs);
    central_diffz_semi_spectral(c, cs, es);
    field_decompose_semi_spectral(c, es);
    for (int iz = 0; iz <= nz; ++iz) { ubar[iz] = svor[0][c.si(iz, 0, 0)]; vbar[iz] = svor[1][c.si(iz, 0, 0)]; }
    diffx(c, es, svor[0]);
    diffy(c, ds, cs);
    for (long h = 0; h < (long)nx * ny; ++h)
        for (int iz = 0; iz <= nz; ++iz) {
            long i = h * (nz + 1) + iz;
            svor[0][i] = c.k2l2i[h] * (svor[0][i] + cs[i]);
        }
    diffy(c, es, svor[1]);
    diffx(c, ds, cs);
    for (long h = 0; h < (long)nx * ny; ++h)
        for (int iz = 0; iz <= nz; ++iz) {
            long i = h * (nz + 1) + iz;
            svor[1][i] = c.k2l2i[h] * (svor[1][i] - cs[i]);
        }
    for (int iz = 0; iz <= nz; ++iz) { svor[0][c.si(iz, 0, 0)] = ubar[iz]; svor[1][c.si(iz, 0, 0)] = vbar[iz]; }
    // combine vorticity in physical space (:91-93)
    for (int nc = 0; nc < 3; ++nc) field_combine_physical(c, svor[nc], c.vortg[nc]);
    // source term for w (:97-150)
    diffy(c, svor[0], ds);
    diffx(c, svor[1], es);
    for (long i = 0; i < ss; ++i) ds[i] = ds[i] - es[i];
#pragma omp parallel for schedule(static)
    for (long h = 0; h < (long)nx * ny; ++h) {
        long t = h * (nz + 1);
        for (int iz = 1; iz <= nz - 1; ++iz)
            bs[t + iz] = ds[t] * c.thetam[t + iz] + ds[t + nz] * c.thetap[t + iz];
        for (int iz = 0; iz <= nz; ++iz)
            es[t + iz] = ds[t] * c.dthetam[t + iz] + ds[t + nz] * c.dthetap[t + iz];
        for (int iz = 1; iz <= nz - 1; ++iz) ds[t + iz] = c.green[t + iz] * ds[t + iz];
        as[t] = zero;
        for (int kz = 1; kz <= nz - 1; ++kz) as[t + kz] = c.rkz[kz] * ds[t + kz];
        as[t + nz] = zero;
        c.tz.dct(&as[t]);
        c.tz.dst(&ds[t + 1]);
        ds[t] = zero;
        for (int iz = 1; iz <= nz - 1; ++iz) ds[t + iz] = ds[t + iz] + bs[t + iz];
        ds[t + nz] = zero;
        for (int iz = 0; iz <= nz; ++iz) es[t + iz] = es[t + iz] + as[t + iz];
    }
    cs = svor[2];
    field_combine_semi_spectral(c, cs);
    // horizontally averaged flow (:158-176)
    ubar[0] = vbar[0] = zero;
    for (int iz = 1; iz <= nz - 1; ++iz) {
        ubar[iz] = -c.rkzi[iz] * svor[1][c.si(iz, 0, 0)];
        vbar[iz] = c.rkzi[iz] * svor[0][c.si(iz, 0, 0)];
    }
    ubar[nz] = vbar[nz] = zero;
    c.tz.dct(ubar.data());
    c.tz.dct(vbar.data());
    for (int iz = 0; iz <= nz; ++iz) {
        ubar[iz] = ubar[iz] + svor[1][c.si(nz, 0, 0)] * c.gamtop[iz] - svor[1][c.si(0, 0, 0)] * c.gambot[iz];
        vbar[iz] = vbar[iz] - svor[0][c.si(nz, 0, 0)] * c.gamtop[iz] + svor[0][c.si(0, 0, 0)] * c.gambot[iz];
    }
    // u (:180-201)
    diffx(c, es, as);
    diffy(c, cs, bs);
    for (long h = 0; h < (long)nx * ny; ++h)
        for (int iz = 0; iz <= nz; ++iz) {
            long i = h * (nz + 1) + iz;
            as[i] = c.k2l2i[h] * (as[i] + bs[i]);
        }
    for (int iz = 0; iz <= nz; ++iz) as[c.si(iz, 0, 0)] = ubar[iz];
    svel[0] = as;
    fftxys2p(c, as, c.velog[0]);
    // v (:205-226)
    diffy(c, es, as);
    diffx(c, cs, bs);
    for (long h = 0; h < (long)nx * ny; ++h)
        for (int iz = 0; iz <= nz; ++iz) {
            long i = h * (nz + 1) + iz;
            as[i] = c.k2l2i[h] * (as[i] - bs[i]);
        }
    for (int iz = 0; iz <= nz; ++iz) as[c.si(iz, 0, 0)] = vbar[iz];
    svel[1] = as;
    fftxys2p(c, as, c.velog[1]);
    // w (:230-233)
    svel[2] = ds;
    fftxys2p(c, ds, c.velog[2]);
    vel2vgrad(c, svel);
    // z halo (:239-246)
    extrap_halo(c, c.velog[0]);
    extrap_halo(c, c.velog[1]);
    antisym_halo(c, c.velog[2]);
}

// divergence (inversion.f90:409-445); f[3] overwritten
void divergence(Ctx& c, Arr f[3], Arr& div) {
    Arr fs, ds;
    fftxyp2s(c, f[0], fs); diffx(c, fs, ds); fftxys2p(c, ds, f[0]); extrap_halo(c, f[0]);
    fftxyp2s(c, f[1], fs); diffy(c, fs, ds); fftxys2p(c, ds, f[1]); extrap_halo(c, f[1]);
    central_diffz(c, f[2], div);
    for (long i = 0; i < c.fsz; ++i) div[i] = f[0][i] + f[1][i] + div[i];
}

// vorticity_tendency (inversion.f90:321-404)
void vorticity_tendency(Ctx& c) {
    Arr f[3];
    for (int k = 0; k < 3; ++k) f[k].assign(c.fsz, 0.0);
    const double* fc = c.f_cor;
    for (int comp = 0; comp < 3; ++comp) {
        const Arr& u = c.velog[comp];
        for (long i = 0; i < c.fsz; ++i) {
            f[0][i] = (c.vortg[0][i] + fc[0]) * u[i];
            f[1][i] = (c.vortg[1][i] + fc[1]) * u[i];
            f[2][i] = (c.vortg[2][i] + fc[2]) * u[i];
            if (comp == 0) f[1][i] = f[1][i] + c.tbuoyg[i];
            if (comp == 1) f[0][i] = f[0][i] - c.tbuoyg[i];
        }
        divergence(c, f, c.vtend[comp]);
    }
    for (int ix = 0; ix < c.nx; ++ix)
        for (int iy = 0; iy < c.ny; ++iy) {
            if (c.bndry_zeta_zero[0]) c.vtend[2][c.fi(0, iy, ix)] = zero;
            if (c.bndry_zeta_zero[1]) c.vtend[2][c.fi(c.nz, iy, ix)] = zero;
        }
    for (int k = 0; k < 3; ++k) extrap_halo(c, c.vtend[k]);
}

// diverge (inversion.f90:410-455)
void diverge(Ctx& c, const Arr& div, Arr grad[3]) {
    Arr ds, us, vs, ws;
    fftxyp2s(c, div, ds);
    for (int iz = 0; iz <= c.nz; ++iz) ds[c.si(iz, 0, 0)] = zero;
    lapinv1(c, ds);
    diffx(c, ds, us); grad[0].assign(c.fsz, 0.0); fftxys2p(c, us, grad[0]);
    diffy(c, ds, vs); grad[1].assign(c.fsz, 0.0); fftxys2p(c, vs, grad[1]);
    central_diffz_semi_spectral(c, ds, ws);
    for (int kx = 0; kx < c.nx; ++kx)
        for (int ky = 0; ky < c.ny; ++ky) { ws[c.si(0, ky, kx)] = zero; ws[c.si(c.nz, ky, kx)] = zero; }
    grad[2].assign(c.fsz, 0.0);
    fftxys2p(c, ws, grad[2]);
}

// ---------------------------------------------------------------------------
// Parcel ellipsoid maths (parcel_ellipsoid.f90)
static const double rho_e = std::sqrt(two / five);                         // :29
static const double costheta[4] = {std::cos(fpi4), std::cos(three * fpi4), std::cos(five * fpi4),
                                   std::cos(7.0 * fpi4)};                   // :33
static const double sintheta[4] = {std::sin(fpi4), std::sin(three * fpi4), std::sin(five * fpi4),
                                   std::sin(7.0 * fpi4)};

inline double get_abc(double volume) { return f34 * volume * fpi; }          // :409-415

// get_B33 (parcel_ellipsoid.f90:383-402)
double get_B33(Ctx& c, long n) {
    const double* b = &c.B[5 * n];
    double abc = get_abc(c.vol[n]);
    double den = b[0] * b[3] - b[1] * b[1];
    if (std::fabs(den) <= 2.220446049250313e-16)
        throw OracleError(EPIC_ERR_NUMERICAL, "in parcel_ellipsoid::get_B33: Division by small number!");
    // Fortran precedence: B11 * B23**2 = B11 * (B23 * B23)
    return (abc * abc - b[2] * (b[1] * b[4] - b[2] * b[3]) + b[0] * (b[4] * b[4]) - b[1] * b[2] * b[4]) / den;
}

// get_full_matrix (parcel_ellipsoid.f90:266-282), column-major
void get_full_matrix(Ctx& c, long n, double* U) {
    const double* b = &c.B[5 * n];
    U[0] = b[0]; U[3] = b[1]; U[6] = b[2];
    U[1] = b[1]; U[4] = b[3]; U[7] = b[4];
    U[2] = b[2]; U[5] = b[4]; U[8] = get_B33(c, n);
}

void get_eigenvalues(Ctx& c, long n, double* D) {                            // :288-305
    double U[9];
    get_full_matrix(c, n, U);
    scherzinger_eigenvalues(U, D);
}

void diagonalise(Ctx& c, long n, double* D, double* V) {                    // :359-376
    double U[9];
    get_full_matrix(c, n, U);
    scherzinger_diagonalise(U, D, V);
}

// get_points (parcel_ellipsoid.f90:216-260)
void get_points(Ctx& c, long n, bool reuse, double pts[4][3]) {
    double* Veta = &c.Vetas[3 * n];
    double* Vtau = &c.Vtaus[3 * n];
    if (!reuse) {
        double D[3], V[9];
        diagonalise(c, n, D, V);
        double se = std::sqrt(std::fabs(D[0] - D[2])) * rho_e;
        double st = std::sqrt(std::fabs(D[1] - D[2])) * rho_e;
        for (int k = 0; k < 3; ++k) { Veta[k] = se * V[k]; Vtau[k] = st * V[3 + k]; }
    }
    for (int j = 0; j < 4; ++j)
        for (int k = 0; k < 3; ++k)
            pts[j][k] = c.pos[3 * n + k] + Veta[k] * costheta[j] + Vtau[k] * sintheta[j];
}

// get_dBdt (parcel_ellipsoid.f90:466-507)
void get_dBdt(Ctx& c, long n, double* Bout) {
    const double* s = &c.strain[8 * n];
    const double* b = &c.B[5 * n];
    double dwdz = -(s[I_DUDX] + s[I_DVDY]);
    double B33 = get_B33(c, n);
    Bout[0] = two * (s[I_DUDX] * b[0] + s[I_DUDY] * b[1] + s[I_DUDZ] * b[2]);
    Bout[1] = s[I_DVDX] * b[0] - dwdz * b[1] + s[I_DVDZ] * b[2] + s[I_DUDY] * b[3] + s[I_DUDZ] * b[4];
    Bout[2] = s[I_DWDX] * b[0] + s[I_DWDY] * b[1] - s[I_DVDY] * b[2] + s[I_DUDY] * b[4] + s[I_DUDZ] * B33;
    Bout[3] = two * (s[I_DVDX] * b[1] + s[I_DVDY] * b[3] + s[I_DVDZ] * b[4]);
    Bout[4] = s[I_DWDX] * b[1] + s[I_DVDX] * b[2] + s[I_DWDY] * b[3] - s[I_DUDX] * b[4] + s[I_DVDZ] * B33;
}

// trilinear (interpl.f90:17-56); ww[k][j][i]
void trilinear(const Ctx& c, const double* p, int& ii, int& jj, int& kk, double ww[2][2][2]) {
    double xyz[3];
    for (int k = 0; k < 3; ++k) xyz[k] = (p[k] - c.lower[k]) * c.dxi[k];
    ii = ffloor(xyz[0]); jj = ffloor(xyz[1]); kk = ffloor(xyz[2]);
    double px = xyz[0] - (double)ii, pxc = one - px;
    double py = xyz[1] - (double)jj, pyc = one - py;
    double pz = xyz[2] - (double)kk, pzc = one - pz;
    double w00 = pyc * pxc, w10 = pyc * px, w01 = py * pxc, w11 = py * px;
    ww[0][0][0] = pzc * w00; ww[0][0][1] = pzc * w10; ww[0][1][0] = pzc * w01; ww[0][1][1] = pzc * w11;
    ww[1][0][0] = pz * w00;  ww[1][0][1] = pz * w10;  ww[1][1][0] = pz * w01;  ww[1][1][1] = pz * w11;
}

void check_k(const Ctx& c, int ks) {
    if (ks < -1 || ks > c.nz)
        throw OracleError(EPIC_ERR_NUMERICAL, "interpolation point outside the vertical halo");
}

// Sum over the 2x2x2 corners in Fortran column-major order (k fastest).
inline double corner_sum(const Ctx& c, const Arr& f, int is, int js, int ks, double ww[2][2][2]) {
    double s = 0.0;
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int k = 0; k < 2; ++k)
                s += ww[k][j][i] * f[c.fi(ks + k, c.wrapy(js + j), c.wrapx(is + i))];
    return s;
}

// apply_periodic_bc / apply_reflective_bc (parcel_bc.f90:17-42)
inline void apply_periodic_bc(const Ctx& c, double* p) {
    p[0] = p[0] - c.extent[0] * (double)fint((p[0] - c.center[0]) * c.hli[0]);
    p[1] = p[1] - c.extent[1] * (double)fint((p[1] - c.center[1]) * c.hli[1]);
}
inline void apply_reflective_bc(const Ctx& c, double* p, double* b) {
    if (p[2] > c.upper[2]) {
        p[2] = two * c.upper[2] - p[2];
        b[2] = -b[2]; b[4] = -b[4];
    } else if (p[2] < c.lower[2]) {
        p[2] = two * c.lower[2] - p[2];
        b[2] = -b[2]; b[4] = -b[4];
    }
}
void parcel_communicate(Ctx& c) {
    for (long n = 0; n < c.n; ++n) apply_periodic_bc(c, &c.pos[3 * n]);
}

// z fold of a scattered field (parcel_interpl.f90:256-275)
void free_slip_fold(Ctx& c, Arr& f) {
    for (int ix = 0; ix < c.nx; ++ix)
        for (int iy = 0; iy < c.ny; ++iy) {
            long t = c.fi(0, iy, ix);
            f[t] = two * f[t];
            f[t + c.nz] = two * f[t + c.nz];
            f[t + 1] = f[t + 1] + f[t - 1];
            f[t + c.nz - 1] = f[t + c.nz - 1] + f[t + c.nz + 1];
        }
}

// vol2grid (parcel_interpl.f90:92-135)
static void v2g_parcel(Ctx& c, long n, bool reuse, double* vg) {
    double pts[4][3], ww[2][2][2];
    int is, js, ks;
    double pvol = c.vol[n];
    get_points(c, n, reuse, pts);
    for (int p = 0; p < 4; ++p) {
        trilinear(c, pts[p], is, js, ks, ww);
        check_k(c, ks);
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j)
                for (int k = 0; k < 2; ++k)
                    vg[c.fi(ks + k, c.wrapy(js + j), c.wrapx(is + i))] += f14 * ww[k][j][i] * pvol;
    }
}

void vol2grid(Ctx& c, bool reuse) {
    std::fill(c.volg.begin(), c.volg.end(), 0.0);
#ifdef _OPENMP
    int nt = std::min(omp_get_max_threads(), 32);
    std::vector<std::vector<double>> priv(nt, std::vector<double>(c.fsz, 0.0));
#pragma omp parallel num_threads(nt)
    {
        double* vg = priv[omp_get_thread_num()].data();
#pragma omp for schedule(static)
        for (long n = 0; n < c.n; ++n) v2g_parcel(c, n, reuse, vg);
    }
#pragma omp parallel for schedule(static)
    for (long g = 0; g < c.fsz; ++g)
        for (int t = 0; t < nt; ++t) c.volg[g] += priv[t][g];
#else
    for (long n = 0; n < c.n; ++n) v2g_parcel(c, n, reuse, c.volg.data());
#endif
    free_slip_fold(c, c.volg);
}

// par2grid (parcel_interpl.f90:146-323)
// Scatter of parcel n into the 7 accumulation fields f[0..6] (vortg x,y,z,
// dbuoyg, humg, tbuoyg, volg).
static void p2g_parcel(Ctx& c, long n, bool reuse, double* const* f) {
    double pts[4][3], ww[2][2][2];
    int is, js, ks;
    double pvol = c.vol[n];
    double q_c = c.hum[n] - c.q_0 * std::exp(c.lambda_c * (c.lower[2] - c.pos[3 * n + 2]));
    q_c = std::max(zero, q_c);
    double btot = c.buoy[n] + c.glat * q_c;
    get_points(c, n, reuse, pts);
    double vals[6] = {c.vor[3 * n], c.vor[3 * n + 1], c.vor[3 * n + 2], c.buoy[n], c.hum[n], btot};
    for (int p = 0; p < 4; ++p) {
        trilinear(c, pts[p], is, js, ks, ww);
        check_k(c, ks);
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j)
                for (int k = 0; k < 2; ++k) {
                    long g = c.fi(ks + k, c.wrapy(js + j), c.wrapx(is + i));
                    double w = f14 * pvol * ww[k][j][i];
                    for (int l = 0; l < 6; ++l) f[l][g] += w * vals[l];
                    f[6][g] += w;
                }
    }
}

void par2grid(Ctx& c, bool reuse) {
    for (auto* f : {&c.vortg[0], &c.vortg[1], &c.vortg[2], &c.volg, &c.dbuoyg, &c.humg, &c.tbuoyg})
        std::fill(f->begin(), f->end(), 0.0);
    std::fill(c.nparg.begin(), c.nparg.end(), 0);
    std::fill(c.nsparg.begin(), c.nsparg.end(), 0);
    double* tgt[7] = {c.vortg[0].data(), c.vortg[1].data(), c.vortg[2].data(), c.dbuoyg.data(), c.humg.data(),
                      c.tbuoyg.data(), c.volg.data()};
    for (long n = 0; n < c.n; ++n) {
        int i0 = ffloor((c.pos[3 * n] - c.lower[0]) * c.dxi[0]);
        int j0 = ffloor((c.pos[3 * n + 1] - c.lower[1]) * c.dxi[1]);
        int k0 = ffloor((c.pos[3 * n + 2] - c.lower[2]) * c.dxi[2]);
        check_k(c, k0);
        long cidx = c.fi(k0, c.wrapy(j0), c.wrapx(i0));
        c.nparg[cidx] += 1;
        if (c.vol[n] <= c.vmin) c.nsparg[cidx] += 1;
    }
#ifdef _OPENMP
    // per-thread accumulation then a fixed-order sum (the reference uses an
    // OpenMP array reduction, parcel_interpl.f90:172-176)
    int nt = std::min(omp_get_max_threads(), 32);
    std::vector<std::vector<double>> priv(nt, std::vector<double>(7 * c.fsz, 0.0));
#pragma omp parallel num_threads(nt)
    {
        int tid = omp_get_thread_num();
        double* f[7];
        for (int l = 0; l < 7; ++l) f[l] = priv[tid].data() + (size_t)l * c.fsz;
#pragma omp for schedule(static)
        for (long n = 0; n < c.n; ++n) p2g_parcel(c, n, reuse, f);
    }
#pragma omp parallel for schedule(static)
    for (long g = 0; g < c.fsz; ++g)
        for (int t = 0; t < nt; ++t)
            for (int l = 0; l < 7; ++l) tgt[l][g] += priv[t][(size_t)l * c.fsz + g];
#else
    for (long n = 0; n < c.n; ++n) p2g_parcel(c, n, reuse, tgt);
#endif
    // parcel counts: fold z halo (:237-243) and check (:245-250)
    long total = 0;
    for (int ix = 0; ix < c.nx; ++ix)
        for (int iy = 0; iy < c.ny; ++iy) {
            long t = c.fi(0, iy, ix);
            c.nparg[t] += c.nparg[t - 1];
            c.nparg[t + c.nz - 1] += c.nparg[t + c.nz];
            c.nsparg[t] += c.nsparg[t - 1];
            c.nsparg[t + c.nz - 1] += c.nsparg[t + c.nz];
            for (int iz = 0; iz < c.nz; ++iz) total += c.nparg[t + iz];
        }
    if (total != c.n)
        throw OracleError(EPIC_ERR_PARCEL_COUNT, "par2grid: Wrong total number of parcels!");
    free_slip_fold(c, c.volg);
    for (int l = 0; l < 3; ++l) free_slip_fold(c, c.vortg[l]);
    free_slip_fold(c, c.tbuoyg);
    free_slip_fold(c, c.dbuoyg);
    free_slip_fold(c, c.humg);
    for (int ix = 0; ix < c.nx; ++ix)
        for (int iy = 0; iy < c.ny; ++iy) {
            long t = c.fi(0, iy, ix);
            for (int iz = 0; iz <= c.nz; ++iz)
                for (int l = 0; l < 3; ++l) c.vortg[l][t + iz] = c.vortg[l][t + iz] / c.volg[t + iz];
            if (c.bndry_zeta_zero[0]) c.vortg[2][t] = zero;
            if (c.bndry_zeta_zero[1]) c.vortg[2][t + c.nz] = zero;
            for (int l = 0; l < 3; ++l) {
                c.vortg[l][t - 1] = two * c.vortg[l][t] - c.vortg[l][t + 1];
                c.vortg[l][t + c.nz + 1] = two * c.vortg[l][t + c.nz] - c.vortg[l][t + c.nz - 1];
            }
            for (int iz = 0; iz <= c.nz; ++iz) {
                c.dbuoyg[t + iz] = c.dbuoyg[t + iz] / c.volg[t + iz];
                c.humg[t + iz] = c.humg[t + iz] / c.volg[t + iz];
                c.tbuoyg[t + iz] = c.tbuoyg[t + iz] / c.volg[t + iz];
            }
            c.tbuoyg[t - 1] = two * c.tbuoyg[t] - c.tbuoyg[t + 1];
            c.tbuoyg[t + c.nz + 1] = two * c.tbuoyg[t + c.nz] - c.tbuoyg[t + c.nz - 1];
        }
}

// grid2par (parcel_interpl.f90:405-470)
void grid2par(Ctx& c, bool add) {
    if (!add) {
        std::fill(c.dpos.begin(), c.dpos.begin() + 3 * c.n, 0.0);
        std::fill(c.dvor.begin(), c.dvor.begin() + 3 * c.n, 0.0);
    }
#pragma omp parallel for schedule(static)
    for (long n = 0; n < c.n; ++n) {
        double pts[4][3], ww[2][2][2];
        int is, js, ks;
        for (int l = 0; l < 8; ++l) c.strain[8 * n + l] = zero;
        get_points(c, n, false, pts);
        for (int p = 0; p < 4; ++p) {
            trilinear(c, pts[p], is, js, ks, ww);
            check_k(c, ks);
            for (int l = 0; l < 3; ++l) c.dpos[3 * n + l] += f14 * corner_sum(c, c.velog[l], is, js, ks, ww);
            for (int l = 0; l < 8; ++l) c.strain[8 * n + l] += f14 * corner_sum(c, c.velgradg[l], is, js, ks, ww);
            for (int l = 0; l < 3; ++l) c.dvor[3 * n + l] += f14 * corner_sum(c, c.vtend[l], is, js, ks, ww);
        }
    }
}

// get_time_step (rk_utils.f90:70-183)
double get_time_step(Ctx& c, double t) {
    const epic_cfg& g = c.cfg;
    double gmax = 2.220446049250313e-16;
#pragma omp parallel for schedule(static) reduction(max : gmax)
    for (int ix = 0; ix < c.nx; ++ix)
        for (int iy = 0; iy < c.ny; ++iy)
            for (int iz = 0; iz <= c.nz; ++iz) {
                long i = c.fi(iz, iy, ix);
                double v[8];
                for (int l = 0; l < 8; ++l) v[l] = c.velgradg[l][i];
                // get_strain (rk_utils.f90:31-64)
                double S[9];
                M3(S, 0, 0) = v[I_DUDX];
                M3(S, 0, 1) = f12 * (v[I_DUDY] + v[I_DVDX]);
                M3(S, 0, 2) = f12 * (v[I_DUDZ] + v[I_DWDX]);
                M3(S, 1, 0) = M3(S, 0, 1);
                M3(S, 1, 1) = v[I_DVDY];
                M3(S, 1, 2) = f12 * (v[I_DVDZ] + v[I_DWDY]);
                M3(S, 2, 0) = M3(S, 0, 2);
                M3(S, 2, 1) = M3(S, 1, 2);
                M3(S, 2, 2) = -(v[I_DUDX] + v[I_DVDY]);
                double D[3];
                scherzinger_eigenvalues(S, D);
                double m = std::max(std::fabs(D[0]), std::max(std::fabs(D[1]), std::fabs(D[2])));
                gmax = std::max(gmax, m);
            }
    double dbmax = -1.0;
    const Arr& b = c.tbuoyg;
#pragma omp parallel for schedule(static) reduction(max : dbmax)
    for (int ix = 0; ix < c.nx; ++ix)
        for (int iy = 0; iy < c.ny; ++iy)
            for (int iz = 0; iz <= c.nz; ++iz) {
                double gx = f12 * c.dxi[0] * (b[c.fi(iz, iy, c.wrapx(ix + 1))] - b[c.fi(iz, iy, c.wrapx(ix - 1))]);
                double db2 = gx * gx;
                double gy = f12 * c.dxi[1] * (b[c.fi(iz, c.wrapy(iy + 1), ix)] - b[c.fi(iz, c.wrapy(iy - 1), ix)]);
                db2 = db2 + gy * gy;
                double gz = f12 * c.dxi[2] * (b[c.fi(iz + 1, iy, ix)] - b[c.fi(iz - 1, iy, ix)]);
                dbmax = std::max(dbmax, db2 + gz * gz);
            }
    double bmax = std::sqrt(std::sqrt(dbmax));
    bmax = std::max(2.220446049250313e-16, bmax);
    double dt;
    if (g.use_fixed_dt) dt = g.fixed_dt;
    else dt = std::min(g.alpha / gmax, g.alpha / bmax);
    if (g.precise_stop && (t + dt > g.t_limit)) dt = g.t_limit - t;
    if (dt <= zero) throw OracleError(EPIC_ERR_NUMERICAL, "Time step <= 0!");
    return dt;
}

// ---------------------------------------------------------------------------
// Diagnostics
void parcel_diagnostics(Ctx& c, double* st) {
    for (int k = 0; k < 18; ++k) st[k] = 0.0;
    double bmin = zero, bmax = zero;
    st[11] = (double)c.n;
    for (long n = 0; n < c.n; ++n) {
        const double* vel = &c.dpos[3 * n];
        const double* vr = &c.vor[3 * n];
        double vol = c.vol[n], b = c.buoy[n];
        st[1] += (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]) * vol;
        st[12] += (vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]) * vol;
        double ev[3];
        get_eigenvalues(c, n, ev);
        double lam = std::sqrt(ev[0] / ev[2]);
        st[3] += lam;
        st[5] += lam * lam;
        st[7] += vol;
        st[6] += vol * vol;
        if (vol <= c.vmin) st[2] += one;
        bmax = std::max(bmax, b);
        bmin = std::min(bmin, b);
        st[8] += vol * (vr[0] * vr[0]);
        st[9] += vol * (vr[1] * vr[1]);
        st[10] += vol * (vr[2] * vr[2]);
    }
    st[16] = bmin;
    st[17] = bmax;
    st[13] = (double)c.n_parcel_splits;
    st[14] = (double)c.n_big_close;
    st[15] = (double)c.n_parcel_merges;
    double ntoti = one / (double)c.n;
    st[1] = f12 * st[1] * c.vdomaini;
    st[12] = f12 * st[12] * c.vdomaini;
    st[3] = st[3] * ntoti;
    st[5] = std::sqrt(std::fabs(st[5] * ntoti - st[3] * st[3]));
    st[8] = std::sqrt(st[8] / st[7]);
    st[9] = std::sqrt(st[9] / st[7]);
    st[10] = std::sqrt(st[10] / st[7]);
    st[4] = st[7] * ntoti;
    st[6] = std::sqrt(std::fabs(st[6] * ntoti - st[4] * st[4]));
}

void field_diagnostics(Ctx& c, double* st) {
    for (int k = 0; k < 11; ++k) st[k] = 0.0;
    int nz = c.nz;
    double rms = 0, abserr = 0, ke_i = 0, ke_0 = 0, ke_n = 0, en_i = 0, en_0 = 0, en_n = 0;
    int maxn = INT32_MIN, minn = INT32_MAX;
    double sumn = 0, sumsn = 0, bmax = -HUGE_VAL, bmin = HUGE_VAL;
    for (int ix = 0; ix < c.nx; ++ix)
        for (int iy = 0; iy < c.ny; ++iy)
            for (int iz = 0; iz <= nz; ++iz) {
                long i = c.fi(iz, iy, ix);
                double dv = c.volg[i] - c.vcell;
                rms += dv * dv;
                abserr = std::max(abserr, std::fabs(dv));
                if (iz < nz) {
                    maxn = std::max(maxn, c.nparg[i]);
                    minn = std::min(minn, c.nparg[i]);
                    sumn += c.nparg[i];
                    sumsn += c.nsparg[i];
                }
                bmax = std::max(bmax, c.tbuoyg[i]);
                bmin = std::min(bmin, c.tbuoyg[i]);
                double u2 = c.velog[0][i] * c.velog[0][i] + c.velog[1][i] * c.velog[1][i] + c.velog[2][i] * c.velog[2][i];
                double w2 = c.vortg[0][i] * c.vortg[0][i] + c.vortg[1][i] * c.vortg[1][i] + c.vortg[2][i] * c.vortg[2][i];
                if (iz == 0) { ke_0 += c.volg[i] * u2; en_0 += c.volg[i] * w2; }
                else if (iz == nz) { ke_n += c.volg[i] * u2; en_n += c.volg[i] * w2; }
                else { ke_i += c.volg[i] * u2; en_i += c.volg[i] * w2; }
            }
    st[0] = std::sqrt(rms * c.ngridi) * c.vcelli;
    st[1] = sumn * c.ncelli;
    st[2] = sumsn * c.ncelli;
    st[3] = (f12 * ke_i + f14 * ke_0 + f14 * ke_n) * c.vdomaini;
    st[4] = 0.0;
    st[5] = (f12 * en_i + f14 * en_0 + f14 * en_n) * c.vdomaini;
    st[6] = abserr * c.vcelli;
    st[7] = maxn;
    st[8] = bmax;
    st[9] = minn;
    st[10] = bmin;
}

// ---------------------------------------------------------------------------
// Corrections (parcel_correction.f90)
void init_parcel_correction(Ctx& c) {                                    // :42-83
    double vsum = 0, vb[3] = {0, 0, 0};
    for (long n = 0; n < c.n; ++n) {
        vsum = vsum + c.vol[n];
        for (int k = 0; k < 3; ++k) vb[k] = vb[k] + c.vor[3 * n + k] * c.vol[n];
    }
    for (int k = 0; k < 3; ++k) c.vor_bar[k] = vb[k] / vsum;
}

void apply_vortcor(Ctx& c) {                                             // :89-138
    double vsum = 0, dv[3] = {0, 0, 0};
    for (long n = 0; n < c.n; ++n) {
        vsum = vsum + c.vol[n];
        for (int k = 0; k < 3; ++k) dv[k] = dv[k] + c.vor[3 * n + k] * c.vol[n];
    }
    for (int k = 0; k < 3; ++k) dv[k] = dv[k] / vsum - c.vor_bar[k];
    for (long n = 0; n < c.n; ++n)
        for (int k = 0; k < 3; ++k) c.vor[3 * n + k] = c.vor[3 * n + k] - dv[k];
}

void apply_laplace(Ctx& c, bool reuse) {                                 // :142-181
    vol2grid(c, reuse);
    Arr phi(c.fsz), grad[3];
    for (long i = 0; i < c.fsz; ++i) phi[i] = c.volg[i] * c.vcelli - one;
    diverge(c, phi, grad);
    for (int k = 0; k < 3; ++k) extrap_halo(c, grad[k]);
#pragma omp parallel for schedule(static)
    for (long n = 0; n < c.n; ++n) {
        double ww[2][2][2];
        int is, js, ks;
        trilinear(c, &c.pos[3 * n], is, js, ks, ww);
        check_k(c, ks);
        double d[3];
        for (int l = 0; l < 3; ++l) d[l] = corner_sum(c, grad[l], is, js, ks, ww);
        for (int l = 0; l < 3; ++l) c.pos[3 * n + l] = c.pos[3 * n + l] + d[l];
    }
    parcel_communicate(c);
}

void apply_gradient(Ctx& c, double prefactor, double max_compression, bool reuse) {   // :183-259
    vol2grid(c, reuse);
    Arr phi(c.fsz);
    for (long i = 0; i < c.fsz; ++i) phi[i] = c.volg[i] * c.vcelli - one;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < c.n; ++n) {
        double w[2][2][2];
        int is, js, ks;
        trilinear(c, &c.pos[3 * n], is, js, ks, w);
        check_k(c, ks);
        int i0 = c.wrapx(is), i1 = c.wrapx(is + 1), j0 = c.wrapy(js), j1 = c.wrapy(js + 1);
        auto P = [&](int k, int j, int i) { return phi[c.fi(ks + k, j ? j1 : j0, i ? i1 : i0)]; };
        double xf = w[0][0][1] + w[0][1][1] + w[1][0][1] + w[1][1][1];
        double yf = w[0][1][0] + w[0][1][1] + w[1][1][0] + w[1][1][1];
        double zf = w[1][0][0] + w[1][0][1] + w[1][1][0] + w[1][1][1];
        double xfc = one - xf, yfc = one - yf, zfc = one - zf;
        double lim_x = c.dx[0] * xf * xfc;
        double xs = -prefactor * lim_x * (zfc * (yfc * (P(0, 0, 1) - P(0, 0, 0)) + yf * (P(0, 1, 1) - P(0, 1, 0)))
                                        + zf * (yfc * (P(1, 0, 1) - P(1, 0, 0)) + yf * (P(1, 1, 1) - P(1, 1, 0))));
        lim_x = lim_x * max_compression;
        xs = std::max(-lim_x, std::min(xs, lim_x));
        double lim_y = c.dx[1] * yf * yfc;
        double ys = -prefactor * lim_y * (zfc * (xfc * (P(0, 1, 0) - P(0, 0, 0)) + xf * (P(0, 1, 1) - P(0, 0, 1)))
                                        + zf * (xfc * (P(1, 1, 0) - P(1, 0, 0)) + xf * (P(1, 1, 1) - P(1, 0, 1))));
        lim_y = lim_y * max_compression;
        ys = std::max(-lim_y, std::min(ys, lim_y));
        double lim_z = c.dx[2] * zf * zfc;
        double zs = -prefactor * lim_z * (xfc * (yfc * (P(1, 0, 0) - P(0, 0, 0)) + yf * (P(1, 1, 0) - P(0, 1, 0)))
                                        + xf * (yfc * (P(1, 0, 1) - P(0, 0, 1)) + yf * (P(1, 1, 1) - P(0, 1, 1))));
        lim_z = lim_z * max_compression;
        zs = std::max(-lim_z, std::min(zs, lim_z));
        c.pos[3 * n] = c.pos[3 * n] + xs;
        c.pos[3 * n + 1] = c.pos[3 * n + 1] + ys;
        c.pos[3 * n + 2] = c.pos[3 * n + 2] + zs;
    }
    parcel_communicate(c);
}

// ---------------------------------------------------------------------------
// Surface fluxes (bndry_fluxes.f90)

// read_bndry_fluxes (:100-175) given the two datasets: binc = 2 dxi(3) bflux.
void set_bndry_fluxes(Ctx& c, const double* bflux, const double* hflux) {
    c.l_enable_flux = bflux != nullptr;
    if (!c.l_enable_flux) return;
    const long m = (long)c.nx * c.ny;
    c.binc.assign(bflux, bflux + m);
    c.hinc.assign(m, zero);
    if (hflux) c.hinc.assign(hflux, hflux + m);
    c.zdepth = c.lower[2] + c.dx[2];
    for (long i = 0; i < m; ++i) {
        c.binc[i] = two * c.dxi[2] * c.binc[i];
        c.hinc[i] = two * c.dxi[2] * c.hinc[i];
    }
}

// bndry_fluxes_time_step (:180-205)
void bndry_fluxes_time_step(Ctx& c, double& dt) {
    if (!c.l_enable_flux) return;
    double abs_max = 0.0;
    for (double v : c.binc) abs_max = std::max(abs_max, std::fabs(v));
    abs_max = std::pow(c.dx[2] / abs_max, f13);
    dt = std::min(dt, c.cfg.alpha * abs_max);
}

// apply_bndry_fluxes (:209-247) with bilinear (interpl.f90:65-90); ww[j][i]
void apply_bndry_fluxes(Ctx& c, double dt) {
    if (!c.l_enable_flux) return;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < c.n; ++n) {
        const double z = c.pos[3 * n + 2];
        if (!(z < c.zdepth)) continue;
        double xy0 = (c.pos[3 * n] - c.lower[0]) * c.dxi[0];
        double xy1 = (c.pos[3 * n + 1] - c.lower[1]) * c.dxi[1];
        int is = ffloor(xy0), js = ffloor(xy1);
        double px = xy0 - (double)is, pxc = one - px;
        double py = xy1 - (double)js, pyc = one - py;
        double ww[2][2] = {{pyc * pxc, pyc * px}, {py * pxc, py * px}};
        double fac = (c.zdepth - z) * c.dxi[2] * dt;
        double sb = 0.0, sh = 0.0;
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j) {
                long h = c.hi2(c.wrapy(js + j), c.wrapx(is + i));
                sb += ww[j][i] * c.binc[h];
                sh += ww[j][i] * c.hinc[h];
            }
        c.buoy[n] = c.buoy[n] + fac * sb;
        c.hum[n] = c.hum[n] + fac * sh;
    }
}

// ---------------------------------------------------------------------------
// Damping (parcel_damping.f90)

// get_strain_magnitude_field (rk_utils.f90:186-214): sqrt(2 S:S) of the
// symmetrised strain, z halo reflected (the x/y halo is the periodic wrap).
void strain_magnitude_field(Ctx& c) {
    c.strain_mag.assign(c.fsz, 0.0);
    for (int ix = 0; ix < c.nx; ++ix)
        for (int iy = 0; iy < c.ny; ++iy) {
            long t = c.fi(0, iy, ix);
            for (int iz = 0; iz <= c.nz; ++iz) {
                double v[8];
                for (int l = 0; l < 8; ++l) v[l] = c.velgradg[l][t + iz];
                double S[9];
                M3(S, 0, 0) = v[I_DUDX];
                M3(S, 0, 1) = f12 * (v[I_DUDY] + v[I_DVDX]);
                M3(S, 0, 2) = f12 * (v[I_DUDZ] + v[I_DWDX]);
                M3(S, 1, 0) = M3(S, 0, 1);
                M3(S, 1, 1) = v[I_DVDY];
                M3(S, 1, 2) = f12 * (v[I_DVDZ] + v[I_DWDY]);
                M3(S, 2, 0) = M3(S, 0, 2);
                M3(S, 2, 1) = M3(S, 1, 2);
                M3(S, 2, 2) = -(v[I_DUDX] + v[I_DVDY]);
                double q = M3(S, 0, 0) * M3(S, 0, 0) + M3(S, 0, 1) * M3(S, 0, 1);
                q = q + M3(S, 0, 2) * M3(S, 0, 2);
                q = q + M3(S, 1, 0) * M3(S, 1, 0);
                q = q + M3(S, 1, 1) * M3(S, 1, 1);
                q = q + M3(S, 1, 2) * M3(S, 1, 2);
                q = q + M3(S, 2, 0) * M3(S, 2, 0);
                q = q + M3(S, 2, 1) * M3(S, 2, 1);
                q = q + M3(S, 2, 2) * M3(S, 2, 2);
                c.strain_mag[t + iz] = std::sqrt(two * q);
            }
            c.strain_mag[t - 1] = c.strain_mag[t + 1];
            c.strain_mag[t + c.nz + 1] = c.strain_mag[t + c.nz - 1];
        }
}

void check_damping_flags(const epic_cfg& g) {
    if (g.damping_vorticity && g.damping_surface_vorticity)
        throw OracleError(EPIC_ERR_CONFIG,
                          "damping%l_vorticity and  damping%l_surface_vorticity both activated, only one allowed");
    if (g.damping_scalars && g.damping_surface_scalars)
        throw OracleError(EPIC_ERR_CONFIG,
                          "damping%l_scalars and  damping%l_surface_scalars both activated, only one allowed");
}

// perturbation_damping (:82-222), moist build (humidity and dry buoyancy).
// sum(weight * time_fact * (g - a)) over the 2x2x2 corners in Fortran order
// (k fastest); the surface forms sum over the (j, i) slice of level ks + si.
void perturbation_damping(Ctx& c, double dt, bool reuse) {
    const epic_cfg& g = c.cfg;
    const bool lv = g.damping_vorticity, ls = g.damping_scalars;
    const bool lsv = g.damping_surface_vorticity, lss = g.damping_surface_scalars;
    const double pv = g.damping_vorticity_prefactor, ps = g.damping_scalars_prefactor;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < c.n; ++n) {
        if (!(lv || ls)) {
            const double z = c.pos[3 * n + 2];
            if (z > c.lower[2] + 2 * c.dx[2] && z < c.upper[2] - 2 * c.dx[2]) continue;
        }
        double pts[4][3], ww[2][2][2], wt[2][2][2], tf[2][2][2];
        int is, js, ks;
        get_points(c, n, reuse, pts);
        double vortend[3] = {zero, zero, zero}, humtend = zero, dbuoytend = zero;
        const double* vor = &c.vor[3 * n];
        const double hum = c.hum[n], buoy = c.buoy[n];
        auto idx = [&](int k, int j, int i) { return c.fi(ks + k, c.wrapy(js + j), c.wrapx(is + i)); };
        auto time_fact = [&](double pref) {
            for (int i = 0; i < 2; ++i)
                for (int j = 0; j < 2; ++j)
                    for (int k = 0; k < 2; ++k) tf[k][j][i] = one - std::exp(-pref * c.strain_mag[idx(k, j, i)] * dt);
        };
        auto full = [&](const Arr& f, double a) {
            double s = 0.0;
            for (int i = 0; i < 2; ++i)
                for (int j = 0; j < 2; ++j)
                    for (int k = 0; k < 2; ++k) s += wt[k][j][i] * tf[k][j][i] * (f[idx(k, j, i)] - a);
            return s;
        };
        auto slice = [&](const Arr& f, double a, int si) {
            double s = 0.0;
            for (int i = 0; i < 2; ++i)
                for (int j = 0; j < 2; ++j) s += wt[si][j][i] * tf[si][j][i] * (f[idx(si, j, i)] - a);
            return s;
        };
        for (int p = 0; p < 4; ++p) {
            trilinear(c, pts[p], is, js, ks, ww);
            check_k(c, ks);
            for (int i = 0; i < 2; ++i)
                for (int j = 0; j < 2; ++j)
                    for (int k = 0; k < 2; ++k) wt[k][j][i] = f14 * ww[k][j][i];
            if (lv) {
                time_fact(pv);
                for (int l = 0; l < 3; ++l) vortend[l] = vortend[l] + full(c.vortg[l], vor[l]);
            }
            if (ls) {
                time_fact(ps);
                humtend = humtend + full(c.humg, hum);
                dbuoytend = dbuoytend + full(c.dbuoyg, buoy);
            }
            if (!(lsv || lss)) continue;
            int si;
            if (ks == -1 || ks == c.nz - 1) si = 1;
            else if (ks == 0 || ks == c.nz) si = 0;
            else continue;
            if (lsv) {
                time_fact(pv);
                for (int l = 0; l < 3; ++l) vortend[l] = vortend[l] + slice(c.vortg[l], vor[l], si);
            }
            if (lss) {
                time_fact(ps);
                humtend = humtend + slice(c.humg, hum, si);
                dbuoytend = dbuoytend + slice(c.dbuoyg, buoy, si);
            }
        }
        if (lv || lsv)
            for (int l = 0; l < 3; ++l) c.vor[3 * n + l] = c.vor[3 * n + l] + vortend[l];
        if (ls || lss) {
            c.hum[n] = c.hum[n] + humtend;
            c.buoy[n] = c.buoy[n] + dbuoytend;
        }
    }
}

// parcel_damp (:43-78)
void parcel_damp(Ctx& c, double dt) {
    const epic_cfg& g = c.cfg;
    check_damping_flags(g);
    if (!(g.damping_vorticity || g.damping_scalars || g.damping_surface_vorticity || g.damping_surface_scalars))
        return;
    par2grid(c, false);
    vor2vel(c);
    for (int ix = 0; ix < c.nx; ++ix)
        for (int iy = 0; iy < c.ny; ++iy) {
            long t = c.fi(0, iy, ix);
            for (Arr* f : {&c.vortg[0], &c.vortg[1], &c.vortg[2], &c.humg, &c.dbuoyg}) {
                (*f)[t - 1] = (*f)[t + 1];
                (*f)[t + c.nz + 1] = (*f)[t + c.nz - 1];
            }
        }
    strain_magnitude_field(c);
    perturbation_damping(c, dt, true);
}

// ---------------------------------------------------------------------------
// LS-RK (ls_rk.f90:88-217)
void ensure_parcel_capacity(Ctx& c, long need) {
    if ((long)c.vol.size() >= need) return;
    long cap = std::max(need, (long)(c.vol.size() * 1.2) + 16);
    c.pos.resize(3 * cap); c.vor.resize(3 * cap); c.B.resize(5 * cap);
    c.vol.resize(cap); c.buoy.resize(cap); c.hum.resize(cap);
    c.dpos.resize(3 * cap); c.dvor.resize(3 * cap); c.strain.resize(8 * cap); c.dB.resize(5 * cap);
    c.Vetas.resize(3 * cap); c.Vtaus.resize(3 * cap);
    if (c.cfg.labels) { c.label.resize(cap); c.dil.resize(cap); }
}

// The merge's label draw (parcel_merge.f90:196, random_number): U[0, 1) from
// a counter-based SplitMix64 keyed by (label_seed, merge call, merge index m)
// instead of the Fortran generator's stream; the same law of choice.
static uint64_t lab_mix(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double label_draw(int32_t seed, long call, long m) {
    uint64_t key = ((uint64_t)(uint32_t)seed * 0x9E3779B97F4A7C15ull) ^ ((((uint64_t)call << 32) + (uint64_t)m) * 16ull + 15ull);
    return (double)(lab_mix(lab_mix(key)) >> 11) * (1.0 / 9007199254740992.0);
}

// parcel_init.f90:135-139: label of the regular position (sub-cell i, j, k
// 1-based, cell ix, iy, iz 0-based)
static int64_t regular_label(const Ctx& c, int npd, int ix, int iy, int iz, int i, int j, int k) {
    const int64_t nxp = (int64_t)c.nx * npd, nyp = (int64_t)c.ny * npd;
    return 1 + ((int64_t)ix * npd + (i - 1)) + nxp * (((int64_t)iy * npd + (j - 1)) + nyp * ((int64_t)iz * npd + (k - 1)));
}

void rk_substep(Ctx& c, double dt, int step) {
    double ca = c.ca[step - 1], cb = c.cb[step - 1];
    double Bout[5];
    if (step == 1) {
#pragma omp parallel for schedule(static) private(Bout)
        for (long n = 0; n < c.n; ++n) {
            get_dBdt(c, n, Bout);
            for (int k = 0; k < 5; ++k) c.dB[5 * n + k] = Bout[k];
        }
    } else {
        vor2vel(c);
        vorticity_tendency(c);
        grid2par(c, true);
#pragma omp parallel for schedule(static) private(Bout)
        for (long n = 0; n < c.n; ++n) {
            get_dBdt(c, n, Bout);
            for (int k = 0; k < 5; ++k) c.dB[5 * n + k] = c.dB[5 * n + k] + Bout[k];
        }
    }
#pragma omp parallel for schedule(static)
    for (long n = 0; n < c.n; ++n) {
        for (int k = 0; k < 3; ++k) c.pos[3 * n + k] = c.pos[3 * n + k] + cb * dt * c.dpos[3 * n + k];
        for (int k = 0; k < 3; ++k) c.vor[3 * n + k] = c.vor[3 * n + k] + cb * dt * c.dvor[3 * n + k];
        for (int k = 0; k < 5; ++k) c.B[5 * n + k] = c.B[5 * n + k] + cb * dt * c.dB[5 * n + k];
    }
    if (step == c.n_stages) {
        parcel_communicate(c);
        return;
    }
    for (long n = 0; n < c.n; ++n) {
        for (int k = 0; k < 3; ++k) c.dpos[3 * n + k] = ca * c.dpos[3 * n + k];
        for (int k = 0; k < 3; ++k) c.dvor[3 * n + k] = ca * c.dvor[3 * n + k];
        for (int k = 0; k < 5; ++k) c.dB[5 * n + k] = ca * c.dB[5 * n + k];
    }
    parcel_communicate(c);
    par2grid(c, false);
}

double rk_step(Ctx& c, double& t, double* pstats, double* fstats) {
    par2grid(c, t > c.cfg.t_initial);
    vor2vel(c);
    vorticity_tendency(c);
    double dt = get_time_step(c, t);
    if (!c.cfg.use_fixed_dt) bndry_fluxes_time_step(c, dt);
    grid2par(c, false);
    if (pstats) parcel_diagnostics(c, pstats);
    if (fstats) field_diagnostics(c, fstats);
    apply_bndry_fluxes(c, dt);
    for (int n = 1; n <= c.n_stages; ++n) rk_substep(c, dt, n);
    for (long n = 0; n < c.n; ++n) apply_reflective_bc(c, &c.pos[3 * n], &c.B[5 * n]);
    parcel_damp(c, dt);
    t = t + dt;
    return dt;
}

// ---------------------------------------------------------------------------
// Split (parcel_split.f90:37-198)
long parcel_split(Ctx& c) {
    static const double dh = f12 * std::sqrt(three / five);
    long n0 = c.n;
    std::vector<long> indices;
    for (long n = 0; n < n0; ++n) {
        double D[3];
        get_eigenvalues(c, n, D);
        double lam = std::sqrt(D[0] / D[2]);
        if (lam < c.cfg.lambda_max && D[0] < c.amax * c.amax) continue;
        indices.push_back(n);
    }
    ensure_parcel_capacity(c, n0 + (long)indices.size());
    for (long n : indices) {
        double Bv[5];
        for (int k = 0; k < 5; ++k) Bv[k] = c.B[5 * n + k];
        double vol = c.vol[n];
        double D[3], V[9];
        diagonalise(c, n, D, V);
        double* b = &c.B[5 * n];
        b[0] = Bv[0] - f34 * D[0] * (V[0] * V[0]);
        b[1] = Bv[1] - f34 * D[0] * V[0] * V[1];
        b[2] = Bv[2] - f34 * D[0] * V[0] * V[2];
        b[3] = Bv[3] - f34 * D[0] * (V[1] * V[1]);
        b[4] = Bv[4] - f34 * D[0] * V[1] * V[2];
        c.vol[n] = f12 * vol;
        long m = c.n;
        c.n += 1;
        for (int k = 0; k < 5; ++k) c.B[5 * m + k] = c.B[5 * n + k];
        for (int k = 0; k < 3; ++k) c.vor[3 * m + k] = c.vor[3 * n + k];
        c.vol[m] = c.vol[n];
        c.buoy[m] = c.buoy[n];
        c.hum[m] = c.hum[n];
        if (c.cfg.labels) { c.label[m] = c.label[n]; c.dil[m] = c.dil[n]; }   // parcel_split.f90:147-150
        double s = dh * std::sqrt(D[0]);
        double v1[3] = {V[0] * s, V[1] * s, V[2] * s};
        for (int k = 0; k < 3; ++k) {
            c.pos[3 * m + k] = c.pos[3 * n + k] - v1[k];
            c.pos[3 * n + k] = c.pos[3 * n + k] + v1[k];
        }
        apply_reflective_bc(c, &c.pos[3 * m], &c.B[5 * m]);
        apply_reflective_bc(c, &c.pos[3 * n], &c.B[5 * n]);
    }
    // parcel_communicate(parcels, invalid): periodic bc of parents and children
    for (long n : indices) apply_periodic_bc(c, &c.pos[3 * n]);
    for (long m = n0; m < c.n; ++m) apply_periodic_bc(c, &c.pos[3 * m]);
    long ns = c.n - n0;
    c.n_parcel_splits += ns;
    return ns;
}

// ---------------------------------------------------------------------------
// Merge: find_nearest (parcel_nearest.f90:375-624), single-rank semantics.
struct Near {
    int hs1, hs2;            // box%halo_size(1:2)
    long hncell;
    std::vector<int> nppc, kc1, kc2, loca, node;
    double halo_lower[2];
};

// handle_periodic_edge_parcels + parcel_to_local_cell_index (:166-226)
void bin_parcel(Ctx& c, Near& nr, std::vector<double>& P, long n) {
    double* p = &P[3 * n];
    int ix = ffloor((p[0] - c.lower[0]) * c.dxi[0]);
    int iy = ffloor((p[1] - c.lower[1]) * c.dxi[1]);
    if (ix < -1) p[0] = p[0] + c.extent[0];
    if (ix > c.nx) p[0] = p[0] - c.extent[0];
    if (iy < -1) p[1] = p[1] + c.extent[1];
    if (iy > c.ny) p[1] = p[1] - c.extent[1];
    ix = fint(c.dxi[0] * (p[0] - nr.halo_lower[0]));
    iy = fint(c.dxi[1] * (p[1] - nr.halo_lower[1]));
    int iz = std::min(fint(c.dxi[2] * (p[2] - c.lower[2])), c.nz - 1);
    long ijk = 1 + ix + (long)nr.hs1 * iy + (long)nr.hs1 * nr.hs2 * iz;
    if (ijk < 1 || ijk > nr.hncell)
        throw OracleError(EPIC_ERR_NUMERICAL, "in nearest_parcel_to_local_cell_index: Parcel not in local domain.");
    nr.nppc[ijk - 1] += 1;
    nr.loca[n] = (int)ijk;
}

// Directions (mpi_tags.f90:3-11): 1 N, 2 S, 3 W, 4 E, 5 NW, 6 NE, 7 SW, 8 SE.
// parcel_delete (parcel_container.f90:413-458): pid holds the 1-based indices
// of the parcels to delete, ascending; the holes below the new count are
// filled with the last valid parcels, from the top.
void parcel_delete(Ctx& c, const std::vector<long>& pids) {
    const long n_merge = (long)pids.size();
    std::vector<long> pid(n_merge + 1);
    for (long m = 0; m < n_merge; ++m) pid[m + 1] = pids[m];
    long lv = c.n, k = n_merge;
    while (k > 0 && lv == pid[k]) { lv -= 1; k -= 1; }
    long mm = 1;
    auto replace = [&](long dst1, long src1) {
        long d = dst1 - 1, s = src1 - 1;
        for (int q = 0; q < 3; ++q) {
            c.pos[3 * d + q] = c.pos[3 * s + q];
            c.vor[3 * d + q] = c.vor[3 * s + q];
            c.dpos[3 * d + q] = c.dpos[3 * s + q];
            c.dvor[3 * d + q] = c.dvor[3 * s + q];
            c.Vetas[3 * d + q] = c.Vetas[3 * s + q];
            c.Vtaus[3 * d + q] = c.Vtaus[3 * s + q];
        }
        for (int q = 0; q < 5; ++q) { c.B[5 * d + q] = c.B[5 * s + q]; c.dB[5 * d + q] = c.dB[5 * s + q]; }
        for (int q = 0; q < 8; ++q) c.strain[8 * d + q] = c.strain[8 * s + q];
        c.vol[d] = c.vol[s]; c.buoy[d] = c.buoy[s]; c.hum[d] = c.hum[s];
        if (c.cfg.labels) { c.label[d] = c.label[s]; c.dil[d] = c.dil[s]; }
    };
    while (mm <= k) {
        replace(pid[mm], lv);
        lv -= 1;
        while (k > 0 && lv == pid[k]) { lv -= 1; k -= 1; }
        mm += 1;
    }
    c.n = c.n - n_merge;
}

long parcel_merge(Ctx& c) {
    const long N = c.n;
    Near nr;
    nr.hs1 = c.nx + 3; nr.hs2 = c.ny + 3;
    nr.hncell = (long)nr.hs1 * nr.hs2 * (c.nz + 2);
    nr.halo_lower[0] = c.lower[0] - c.dx[0];
    nr.halo_lower[1] = c.lower[1] - c.dx[1];
    nr.nppc.assign(nr.hncell, 0);
    // working copy of positions: locals are modified in place like the
    // reference (handle_periodic_edge_parcels), copies are appended.
    std::vector<double>& P = c.pos;
    std::vector<long> bufs[9];   // per send direction: local small parcel ids (0-based)
    std::vector<int> small_m;    // merge index of local small parcels
    long n_local_small = 0;
    std::vector<long> msm(N, -1);
    nr.loca.assign(N, 0);
    for (long n = 0; n < N; ++n) {
        bin_parcel(c, nr, P, n);
        if (c.vol[n] < c.vmin) {
            n_local_small += 1;
            msm[n] = n_local_small;
            // locate_parcel_in_boundary_cell (:1384-1460)
            int ix = fnint(c.dxi[0] * (P[3 * n] - c.lower[0]));
            int iy = fnint(c.dxi[1] * (P[3 * n + 1] - c.lower[1]));
            if (ix == 0) {
                if (iy == 0) bufs[7].push_back(n);
                else if (iy == c.ny) bufs[5].push_back(n);
                bufs[3].push_back(n);
            }
            if (ix == c.nx) {
                if (iy == 0) bufs[8].push_back(n);
                else if (iy == c.ny) bufs[6].push_back(n);
                bufs[4].push_back(n);
            }
            if (iy == 0) bufs[2].push_back(n);
            if (iy == c.ny) bufs[1].push_back(n);
        }
    }
    if (n_local_small == 0) {
        c.last_isma.clear(); c.last_iclo.clear();
        parcel_communicate(c);
        return 0;
    }
    // send_small_parcel_bndry_info (:1466-1621): receive slot r holds send
    // buffer k with SEND_NEIGHBOUR_TAG(k) = r, shifted by apply_periodic_shift(r).
    static const int send_tag[9] = {0, 2, 1, 4, 3, 8, 7, 6, 5};
    std::vector<long> pid_copy;      // original (0-based) index per copy
    std::vector<long> mid_copy;      // merge index of original
    std::vector<int> slot_of_copy;
    for (int r = 1; r <= 8; ++r) {
        int k = send_tag[r];
        for (long n : bufs[k]) {
            long idx = N + (long)pid_copy.size();
            if ((long)P.size() < 3 * (idx + 1)) P.resize(3 * (idx + 1));
            double* q = &P[3 * idx];
            q[0] = P[3 * n]; q[1] = P[3 * n + 1]; q[2] = P[3 * n + 2];
            // apply_periodic_shift (:630-668)
            int ix = fnint(c.dxi[0] * (q[0] - c.lower[0]));
            int iy = fnint(c.dxi[1] * (q[1] - c.lower[1]));
            bool xe = (ix <= 0) || (ix >= c.nx), ye = (iy <= 0) || (iy >= c.ny);
            switch (r) {
                case 1: if (ye) q[1] += c.extent[1]; break;
                case 2: if (ye) q[1] -= c.extent[1]; break;
                case 3: if (xe) q[0] -= c.extent[0]; break;
                case 4: if (xe) q[0] += c.extent[0]; break;
                case 5: if (xe) q[0] -= c.extent[0]; if (ye) q[1] += c.extent[1]; break;
                case 6: if (xe) q[0] += c.extent[0]; if (ye) q[1] += c.extent[1]; break;
                case 7: if (xe) q[0] -= c.extent[0]; if (ye) q[1] -= c.extent[1]; break;
                case 8: if (xe) q[0] += c.extent[0]; if (ye) q[1] -= c.extent[1]; break;
            }
            nr.loca.push_back(0);
            pid_copy.push_back(n);
            mid_copy.push_back(msm[n]);
            slot_of_copy.push_back(r);
            bin_parcel(c, nr, P, idx);
        }
    }
    const long n_remote = (long)pid_copy.size();
    const long NT = N + n_remote;
    // set_lbound / set_ubound (:232-257), isma (:530-538); 1-based indices
    nr.kc1.assign(nr.hncell, 0); nr.kc2.assign(nr.hncell, 0);
    nr.kc1[0] = 1;
    for (long ijk = 1; ijk < nr.hncell; ++ijk) nr.kc1[ijk] = nr.kc1[ijk - 1] + nr.nppc[ijk - 1];
    for (long ijk = 0; ijk < nr.hncell; ++ijk) nr.kc2[ijk] = nr.kc1[ijk] - 1;
    nr.node.assign(NT + 1, 0);
    long ntot_small = n_local_small + n_remote;
    std::vector<long> isma(ntot_small + 1, -1), iclo(ntot_small + 1, -1);
    std::vector<double> dclo(ntot_small + 1, 0.0);
    long j = 0;
    for (long n1 = 1; n1 <= NT; ++n1) {
        long ijk = nr.loca[n1 - 1];
        long k = nr.kc2[ijk - 1] + 1;
        nr.node[k] = (int)n1;
        nr.kc2[ijk - 1] = k;
        bool small = (n1 <= N) ? (c.vol[n1 - 1] < c.vmin) : true;
        if (small) isma[++j] = n1;
    }
    // find_closest_parcel_locally (:675-747)
    double dsq0 = c.extent[0] * c.extent[0] + c.extent[1] * c.extent[1] + c.extent[2] * c.extent[2];
    for (long m = 1; m <= ntot_small; ++m) {
        long is = isma[m];
        double xs = P[3 * (is - 1)], ys = P[3 * (is - 1) + 1], zs = P[3 * (is - 1) + 2];
        int ix0 = fnint(c.dxi[0] * (xs - nr.halo_lower[0]));
        int iy0 = fnint(c.dxi[1] * (ys - nr.halo_lower[1]));
        int iz0 = fnint(c.dxi[2] * (zs - c.lower[2]));
        double dsqmin = dsq0;
        long ic = 0;
        for (int iz = std::max(0, iz0 - 1); iz <= std::min(c.nz - 1, iz0); ++iz)
            for (int iy = std::max(0, iy0 - 1); iy <= std::min(c.ny + 1, iy0); ++iy)
                for (int ix = std::max(0, ix0 - 1); ix <= std::min(c.nx + 1, ix0); ++ix) {
                    long ijk = 1 + ix + (long)nr.hs1 * iy + (long)nr.hs1 * nr.hs2 * iz;
                    for (long k = nr.kc1[ijk - 1]; k <= nr.kc2[ijk - 1]; ++k) {
                        long n1 = nr.node[k];
                        if (n1 != is) {
                            double delz = P[3 * (n1 - 1) + 2] - zs;
                            if (delz * delz < dsqmin) {
                                double delx = P[3 * (n1 - 1)] - xs;
                                double dely = P[3 * (n1 - 1) + 1] - ys;
                                double dsq = delx * delx + dely * dely + delz * delz;
                                if (dsq < dsqmin) { dsqmin = dsq; ic = n1; }
                            }
                        }
                    }
                }
        iclo[m] = ic;
        dclo[m] = dsqmin;
    }
    // update_remote_indices (:751-794)
    for (long m = 1; m <= ntot_small; ++m) {
        long is = isma[m], ic = iclo[m];
        if (is > N && ic > N) dclo[m] = 1.7976931348623157e308;   // huge(0.0d0)
        else if (ic > N) iclo[m] = pid_copy[ic - N - 1] + 1;
    }
    // find_closest_parcel_globally (:804-930): results of copies return to the
    // originals in send-buffer order 1..8 (receive slot r = SEND(k)).
    std::vector<long> copy_m_of_idx(n_remote);
    for (long q = 0; q < n_remote; ++q) copy_m_of_idx[q] = n_local_small + q + 1;
    for (int k = 1; k <= 8; ++k) {
        int r = send_tag[k];
        for (long q = 0; q < n_remote; ++q) {
            if (slot_of_copy[q] != r) continue;
            long mc = copy_m_of_idx[q];
            long mo = mid_copy[q];
            if (dclo[mo] > dclo[mc]) {
                dclo[mo] = dclo[mc];
                iclo[mo] = iclo[mc];
            }
        }
    }
    for (long m = 1; m <= n_local_small; ++m)
        if (iclo[m] == 0) throw OracleError(EPIC_ERR_NUMERICAL, "Merge error: no near enough neighbour found.");

    // resolve_tree (:937-1377), single rank
    std::vector<char> l_merged(N + 1, 0), l_leaf(N + 1, 0), l_avail(N + 1, 0);
    long nls = n_local_small;
    bool cont = true;
    while (cont) {
        cont = false;
        for (long m = 1; m <= nls; ++m) {
            long is = isma[m];
            if (!l_merged[is]) { l_leaf[is] = 1; l_avail[iclo[m]] = 1; }
        }
        for (long m = 1; m <= nls; ++m) {
            long is = isma[m];
            if (!l_merged[is]) l_leaf[iclo[m]] = 0;
        }
        for (long m = 1; m <= nls; ++m) {
            long is = isma[m];
            if (!l_merged[is] && !l_leaf[is]) l_avail[iclo[m]] = 0;
        }
        for (long m = 1; m <= nls; ++m) {
            long is = isma[m];
            if (!l_merged[is]) {
                long ic = iclo[m];
                bool h = l_avail[ic];
                if (l_leaf[is] && h) {
                    cont = true;
                    l_merged[is] = 1;
                    l_merged[ic] = 1;
                }
            }
        }
    }
    for (long m = 1; m <= nls; ++m) {
        long is = isma[m];
        if (!l_merged[is] && l_leaf[is]) l_avail[iclo[m]] = 1;
    }
    std::vector<char> do_merge(nls + 1, 0), isolated(nls + 1, 0);
    for (long m = 1; m <= nls; ++m) {
        long is = isma[m], ic = iclo[m];
        if (l_merged[is] && l_leaf[is]) {
            do_merge[m] = 1;
            if (l_leaf[ic]) throw OracleError(EPIC_ERR_NUMERICAL, "in parcel_nearest::resolve_tree: First stage error");
        } else if (!l_merged[is]) {
            if (l_leaf[is]) {
                do_merge[m] = 1;
            } else if (!l_avail[is]) {
                if (l_avail[ic]) do_merge[m] = 1;
                else {
                    isolated[m] = 1;
                    l_avail[is] = 1;
                }
            }
        }
    }
    for (long m = 1; m <= nls; ++m)
        if (!do_merge[m] && isolated[m] && l_avail[iclo[m]]) do_merge[m] = 1;
    std::vector<long> ism, icl;
    for (long m = 1; m <= nls; ++m)
        if (do_merge[m]) { ism.push_back(isma[m]); icl.push_back(iclo[m]); }
    const long n_merge = (long)ism.size();
    c.last_isma.assign(ism.begin(), ism.end());
    c.last_iclo.assign(icl.begin(), icl.end());
    c.n_parcel_merges += n_merge;
    if (n_merge == 0) {
        parcel_communicate(c);
        return 0;
    }
    // collect_merge_stats (parcel_merge.f90:365-394)
    for (long m = 0; m < n_merge; ++m)
        if (c.vol[icl[m] - 1] > c.vmin) c.n_big_close += 1;

    // do_group_merge (parcel_merge.f90:118-323), 0-based parcel indices
    std::vector<long> loca(N + 1, 0);
    std::vector<double> x0, y0, vm, posm, buoym, humm, vortm, Bm;
    std::vector<int64_t> labelm;
    std::vector<double> dilm;
    const long call = c.merge_calls++;
    auto delx_p = [&](double x1, double x2) {                  // parcel_ops.f90:17-37
        double d = x1 - x2;
        return d - c.extent[0] * (double)fnint(d * c.extenti[0]);
    };
    auto dely_p = [&](double y1, double y2) {
        double d = y1 - y2;
        return d - c.extent[1] * (double)fnint(d * c.extenti[1]);
    };
    long l = 0;
    for (long m = 0; m < n_merge; ++m) {
        long ic = icl[m] - 1, is = ism[m] - 1;
        apply_periodic_bc(c, &P[3 * is]);
        if (loca[ic + 1] == 0) {
            l += 1;
            loca[ic + 1] = l;
            vm.push_back(c.vol[ic]);
            x0.push_back(P[3 * ic]);
            y0.push_back(P[3 * ic + 1]);
            posm.push_back(0.0); posm.push_back(0.0); posm.push_back(c.vol[ic] * P[3 * ic + 2]);
            buoym.push_back(c.vol[ic] * c.buoy[ic]);
            humm.push_back(c.vol[ic] * c.hum[ic]);
            for (int k = 0; k < 3; ++k) vortm.push_back(c.vol[ic] * c.vor[3 * ic + k]);
            for (int k = 0; k < 6; ++k) Bm.push_back(0.0);
            if (c.cfg.labels) { labelm.push_back(c.label[ic]); dilm.push_back(c.dil[ic]); }
        }
        long g = loca[ic + 1] - 1;
        if (c.cfg.labels) {
            // parcel_merge.f90:193-203
            const double rn = label_draw(c.cfg.label_seed, call, m);
            if (rn * (vm[g] + c.vol[is]) < vm[g]) {
                dilm[g] = dilm[g] + std::log(vm[g] / (vm[g] + c.vol[is]));
            } else {
                labelm[g] = c.label[is];
                dilm[g] = c.dil[is] + std::log(c.vol[is] / (vm[g] + c.vol[is]));
            }
        }
        vm[g] = vm[g] + c.vol[is];
        double dx_ = delx_p(P[3 * is], x0[g]);
        double dy_ = dely_p(P[3 * is + 1], y0[g]);
        posm[3 * g] = posm[3 * g] + c.vol[is] * dx_;
        posm[3 * g + 1] = posm[3 * g + 1] + c.vol[is] * dy_;
        posm[3 * g + 2] = posm[3 * g + 2] + c.vol[is] * P[3 * is + 2];
        buoym[g] = buoym[g] + c.vol[is] * c.buoy[is];
        humm[g] = humm[g] + c.vol[is] * c.hum[is];
        for (int k = 0; k < 3; ++k) vortm[3 * g + k] = vortm[3 * g + k] + c.vol[is] * c.vor[3 * is + k];
    }
    for (long g = 0; g < l; ++g) {
        double vmerge = one / vm[g];
        posm[3 * g] = vmerge * posm[3 * g];
        posm[3 * g + 1] = vmerge * posm[3 * g + 1];
        posm[3 * g] = x0[g] + posm[3 * g];
        posm[3 * g + 1] = y0[g] + posm[3 * g + 1];
        posm[3 * g + 2] = vmerge * posm[3 * g + 2];
        apply_periodic_bc(c, &posm[3 * g]);
        buoym[g] = vmerge * buoym[g];
        humm[g] = vmerge * humm[g];
        for (int k = 0; k < 3; ++k) vortm[3 * g + k] = vmerge * vortm[3 * g + k];
    }
    std::fill(loca.begin(), loca.end(), 0);
    l = 0;
    for (long m = 0; m < n_merge; ++m) {
        long ic = icl[m] - 1, is = ism[m] - 1;
        if (loca[ic + 1] == 0) {
            l += 1;
            loca[ic + 1] = l;
            long g = l - 1;
            double vmerge = one / vm[g];
            double B33 = get_B33(c, ic);
            double ddx = delx_p(P[3 * ic], posm[3 * g]);
            double ddy = dely_p(P[3 * ic + 1], posm[3 * g + 1]);
            double ddz = P[3 * ic + 2] - posm[3 * g + 2];
            double mu = c.vol[ic] * vmerge;
            const double* b = &c.B[5 * ic];
            Bm[6 * g + 0] = mu * (five * (ddx * ddx) + b[0]);
            Bm[6 * g + 1] = mu * (five * ddx * ddy + b[1]);
            Bm[6 * g + 2] = mu * (five * ddx * ddz + b[2]);
            Bm[6 * g + 3] = mu * (five * (ddy * ddy) + b[3]);
            Bm[6 * g + 4] = mu * (five * ddy * ddz + b[4]);
            Bm[6 * g + 5] = mu * (five * (ddz * ddz) + B33);
            c.vol[ic] = vm[g];
            P[3 * ic] = posm[3 * g]; P[3 * ic + 1] = posm[3 * g + 1]; P[3 * ic + 2] = posm[3 * g + 2];
            c.buoy[ic] = buoym[g];
            c.hum[ic] = humm[g];
            for (int k = 0; k < 3; ++k) c.vor[3 * ic + k] = vortm[3 * g + k];
            if (c.cfg.labels) { c.label[ic] = labelm[g]; c.dil[ic] = dilm[g]; }
        }
        long g = loca[ic + 1] - 1;
        double vmerge = one / vm[g];
        double ddx = delx_p(P[3 * is], posm[3 * g]);
        double ddy = dely_p(P[3 * is + 1], posm[3 * g + 1]);
        double ddz = P[3 * is + 2] - posm[3 * g + 2];
        double B33 = get_B33(c, is);
        double mu = vmerge * c.vol[is];
        const double* b = &c.B[5 * is];
        Bm[6 * g + 0] = Bm[6 * g + 0] + mu * (five * (ddx * ddx) + b[0]);
        Bm[6 * g + 1] = Bm[6 * g + 1] + mu * (five * ddx * ddy + b[1]);
        Bm[6 * g + 2] = Bm[6 * g + 2] + mu * (five * ddx * ddz + b[2]);
        Bm[6 * g + 3] = Bm[6 * g + 3] + mu * (five * (ddy * ddy) + b[3]);
        Bm[6 * g + 4] = Bm[6 * g + 4] + mu * (five * ddy * ddz + b[4]);
        Bm[6 * g + 5] = Bm[6 * g + 5] + mu * (five * (ddz * ddz) + B33);
    }
    // geometric_merge (parcel_merge.f90:330-361)
    std::fill(loca.begin(), loca.end(), 0);
    l = 0;
    for (long m = 0; m < n_merge; ++m) {
        long ic = icl[m] - 1;
        if (loca[ic + 1] == 0) {
            l += 1;
            loca[ic + 1] = l;
            const double* Bg = &Bm[6 * (l - 1)];
            double detB = Bg[0] * (Bg[3] * Bg[5] - Bg[4] * Bg[4])
                        - Bg[1] * (Bg[1] * Bg[5] - Bg[2] * Bg[4])
                        + Bg[2] * (Bg[1] * Bg[4] - Bg[2] * Bg[3]);
            double abc = get_abc(vm[l - 1]);
            double factor = std::pow(abc * abc / detB, f13);
            for (int k = 0; k < 5; ++k) c.B[5 * ic + k] = Bg[k] * factor;
        }
    }
    // parcel_delete (parcel_container.f90:413-458) with pid = isma (ascending)
    {
        std::vector<long> pid(ism.begin(), ism.begin() + n_merge);
        parcel_delete(c, pid);
    }
    parcel_communicate(c);
    return n_merge;
}

// ---------------------------------------------------------------------------
void alloc_fields(Ctx& c) {
    c.nzh = c.nz + 3;
    c.fsz = (long)c.nx * c.ny * c.nzh;
    for (int k = 0; k < 3; ++k) { c.velog[k].assign(c.fsz, 0); c.vortg[k].assign(c.fsz, 0); c.vtend[k].assign(c.fsz, 0); }
    for (int k = 0; k < 8; ++k) c.velgradg[k].assign(c.fsz, 0);
    c.tbuoyg.assign(c.fsz, 0); c.dbuoyg.assign(c.fsz, 0); c.humg.assign(c.fsz, 0); c.volg.assign(c.fsz, 0);
    c.nparg.assign(c.fsz, 0); c.nsparg.assign(c.fsz, 0);
}

Arr* field_ptr(Ctx& c, int id) {
    if (id >= 0 && id < 3) return &c.velog[id];
    if (id >= 3 && id < 6) return &c.vortg[id - 3];
    if (id >= 6 && id < 9) return &c.vtend[id - 6];
    if (id >= 9 && id < 17) return &c.velgradg[id - 9];
    if (id == EPIC_FIELD_TBUOYG) return &c.tbuoyg;
    if (id == EPIC_FIELD_DBUOYG) return &c.dbuoyg;
    if (id == EPIC_FIELD_HUMG) return &c.humg;
    if (id == EPIC_FIELD_VOLG) return &c.volg;
    return nullptr;
}

}  // namespace

struct epic_ctx { Ctx c; };

#define GUARD_BEGIN try {
#define GUARD_END                                                        \
    } catch (const OracleError& e) {                                     \
        ctx->c.err = e.what();                                           \
        return e.code;                                                   \
    } catch (const std::exception& e) {                                  \
        ctx->c.err = e.what();                                           \
        return EPIC_ERR_STATE;                                           \
    }                                                                    \
    return EPIC_OK;

extern "C" {

int epic_oracle_default_config(epic_cfg* g) {
    if (!g) return EPIC_ERR_ARG;
    std::memset(g, 0, sizeof(*g));
    g->size_factor = 1.0; g->grow_factor = 1.2; g->shrink_factor = 0.8; g->n_per_cell = 8;
    g->lambda_max = 4.0; g->min_vratio = 20.0; g->correction_iters = 2; g->gradient_pref = 1.8;
    g->max_compression = 0.5; g->t_initial = 0.0; g->t_limit = 0.0; g->alpha = 0.2;
    g->precise_stop = 0; g->use_fixed_dt = 0; g->fixed_dt = 1.0; g->rk_order = 4;
    g->gravity = 9.80616; g->L_v = (double)2.501e6f; g->c_p = 1005.7; g->theta_0 = 288.15;
    g->q_0 = 0.015; g->height_c = 1000.0; g->ang_vel = 0.000072921; g->lat_degrees = 45.0;
    g->l_planetary_vorticity = 0;
    g->bndry_zeta_zero[0] = g->bndry_zeta_zero[1] = 0;
    g->capacity = 0; g->precision = EPIC_PRECISION_FP64; g->keep_order = 1;
    g->damping_vorticity_prefactor = 1.0; g->damping_scalars_prefactor = 1.0;
    return EPIC_OK;
}

int epic_oracle_create(const epic_cfg* cfg, epic_ctx** out) {
    if (!cfg || !out) return EPIC_ERR_ARG;
    if (cfg->nx < 4 || cfg->ny < 4 || cfg->nz < 2) return EPIC_ERR_CONFIG;
    auto* ctx = new epic_ctx();
    ctx->c.cfg = *cfg;
    try {
        check_damping_flags(*cfg);
        update_parameters(ctx->c);
        alloc_fields(ctx->c);
        init_inversion(ctx->c);
    } catch (const OracleError& e) {
        delete ctx;
        return e.code;
    }
    *out = ctx;
    return EPIC_OK;
}

void epic_oracle_destroy(epic_ctx* ctx) { delete ctx; }
const char* epic_oracle_last_error(const epic_ctx* ctx) { return ctx ? ctx->c.err.c_str() : "null context"; }
int epic_oracle_sync(epic_ctx*) { return EPIC_OK; }

int epic_oracle_set_parcels(epic_ctx* ctx, int64_t n, const double* pos, const double* vor, const double* B,
                            const double* vol, const double* buoy, const double* hum) {
    if (!ctx || n < 0 || !pos || !vor || !B || !vol || !buoy) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    c.n = 0;
    ensure_parcel_capacity(c, n);
    c.n = n;
    std::memcpy(c.pos.data(), pos, sizeof(double) * 3 * n);
    std::memcpy(c.vor.data(), vor, sizeof(double) * 3 * n);
    std::memcpy(c.B.data(), B, sizeof(double) * 5 * n);
    std::memcpy(c.vol.data(), vol, sizeof(double) * n);
    std::memcpy(c.buoy.data(), buoy, sizeof(double) * n);
    if (hum) std::memcpy(c.hum.data(), hum, sizeof(double) * n);
    else std::fill(c.hum.begin(), c.hum.begin() + n, 0.0);
    std::fill(c.dpos.begin(), c.dpos.end(), 0.0);
    std::fill(c.dvor.begin(), c.dvor.end(), 0.0);
    std::fill(c.dB.begin(), c.dB.end(), 0.0);
    std::fill(c.strain.begin(), c.strain.end(), 0.0);
    if (c.cfg.labels) {
        std::fill(c.label.begin(), c.label.end(), (int64_t)0);
        std::fill(c.dil.begin(), c.dil.end(), 0.0);
    }
    return EPIC_OK;
}

int epic_oracle_get_labels(epic_ctx* ctx, int64_t cap, int64_t* n, int64_t* label, double* dilution) {
    if (!ctx || !n) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    if (!c.cfg.labels) { c.err = "labels are off (cfg.labels = 0)"; return EPIC_ERR_STATE; }
    *n = c.n;
    if (cap < c.n) { c.err = "get_labels: capacity too small"; return EPIC_ERR_ARG; }
    if (label) std::memcpy(label, c.label.data(), sizeof(int64_t) * c.n);
    if (dilution) std::memcpy(dilution, c.dil.data(), sizeof(double) * c.n);
    return EPIC_OK;
}

int epic_oracle_set_labels(epic_ctx* ctx, int64_t n, const int64_t* label, const double* dilution) {
    if (!ctx || !label || !dilution) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    if (!c.cfg.labels) { c.err = "labels are off (cfg.labels = 0)"; return EPIC_ERR_STATE; }
    if (n != c.n) { c.err = "set_labels: n differs from the number of parcels"; return EPIC_ERR_ARG; }
    std::memcpy(c.label.data(), label, sizeof(int64_t) * n);
    std::memcpy(c.dil.data(), dilution, sizeof(double) * n);
    return EPIC_OK;
}

// Initial states of the benchmark workloads (parcel_init.f90:31-152 placement
// and shapes, beltrami_3d.f90:103-122 vorticity, the rising thermal), the
// same arithmetic as epic_b200/initial.py, with its SplitMix64 counter RNG.
static uint64_t sm64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double u01(uint64_t seed, uint64_t idx, int comp) {
    uint64_t key = (seed * 0x9E3779B97F4A7C15ull) ^ (idx * 16ull + (uint64_t)comp);
    return (double)(sm64(sm64(key)) >> 11) * (1.0 / 9007199254740992.0);
}

int epic_oracle_init_state(epic_ctx* ctx, const epic_init_spec* s) {
    if (!ctx || !s) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    int npd = (int)std::lround(std::cbrt((double)s->n_per_cell));
    if (npd < 1 || npd * npd * npd != s->n_per_cell) return EPIC_ERR_CONFIG;
    if (s->kind != EPIC_INIT_THERMAL && s->kind != EPIC_INIT_BELTRAMI) return EPIC_ERR_CONFIG;
    long n = (long)c.nx * c.ny * c.nz * s->n_per_cell;
    std::vector<double> pos(3 * n), vor(3 * n, 0.0), B(5 * n, 0.0), vol(n), buoy(n, 0.0), hum(n, 0.0);
    const double im = 1.0 / npd;
    const double v = c.vcell / s->n_per_cell;
    const double* d = c.dx;
    double lam = std::max({d[0] / d[1], d[1] / d[0], d[0] / d[2], d[2] / d[0], d[1] / d[2], d[2] / d[1]});
    if (s->kind == EPIC_INIT_BELTRAMI) lam = 1.0;
    const double b11 = std::pow(lam * (0.75 * v * (1.0 / M_PI)), 2.0 / 3.0);
    const double kk = s->k, ll = s->l, mm = s->m;
    const double alpha = std::sqrt(kk * kk + ll * ll + mm * mm);
    const double fk2l2 = s->kind == EPIC_INIT_BELTRAMI ? alpha / (double)(s->k * s->k + s->l * s->l) : 0.0;
    const double zmax = std::nextafter(c.upper[2], c.lower[2]);
    for (long p = 0; p < n; ++p) {
        long q = p;
        int sub[3], cell[3];
        for (int k = 0; k < 3; ++k) { sub[k] = (int)(q % npd) + 1; q /= npd; }
        cell[0] = (int)(q % c.nx); q /= c.nx;
        cell[1] = (int)(q % c.ny); q /= c.ny;
        cell[2] = (int)q;
        double x[3];
        for (int k = 0; k < 3; ++k) {
            double corner = c.lower[k] + (double)cell[k] * d[k];
            x[k] = corner + d[k] * ((double)sub[k] - 0.5) * im;
        }
        if (s->kind == EPIC_INIT_THERMAL) {
            for (int k = 0; k < 3; ++k) x[k] += (2.0 * u01(s->seed, (uint64_t)p, k) - 1.0) * 0.1 * d[k];
            x[2] = std::min(std::max(x[2], c.lower[2]), zmax);
            double b = 0.0;
            for (int q2 = 0; q2 < s->n_bubbles; ++q2) {
                const double* bb = s->bubble[q2];
                double r2 = (x[0] - bb[0]) * (x[0] - bb[0]) + (x[1] - bb[1]) * (x[1] - bb[1]) +
                            (x[2] - bb[2]) * (x[2] - bb[2]);
                b += bb[3] * std::exp(-r2 / 0.25);
            }
            b += (2.0 * u01(s->seed, (uint64_t)p, 3) - 1.0) * 1.0e-3;
            buoy[p] = b;
        } else {
            double cosmz = std::cos(mm * x[2]), sinmz = std::sin(mm * x[2]);
            double sn = std::sin(kk * x[0] + ll * x[1]), cs = std::cos(kk * x[0] + ll * x[1]);
            vor[3 * p] = fk2l2 * (kk * mm * sinmz - ll * alpha * cosmz) * sn;
            vor[3 * p + 1] = fk2l2 * (ll * mm * sinmz + kk * alpha * cosmz) * sn;
            vor[3 * p + 2] = alpha * cosmz * cs;
        }
        for (int k = 0; k < 3; ++k) pos[3 * p + k] = x[k];
        B[5 * p] = b11;
        B[5 * p + 3] = b11;
        vol[p] = v;
    }
    c.n_parcel_splits = c.n_parcel_merges = c.n_big_close = 0;
    int rc = epic_oracle_set_parcels(ctx, n, pos.data(), vor.data(), B.data(), vol.data(), buoy.data(), hum.data());
    if (rc == EPIC_OK && c.cfg.labels)
        for (long p = 0; p < n; ++p) {
            long q = p;
            int sub[3];
            for (int k = 0; k < 3; ++k) { sub[k] = (int)(q % npd) + 1; q /= npd; }
            const int ix = (int)(q % c.nx); q /= c.nx;
            const int iy = (int)(q % c.ny); q /= c.ny;
            c.label[p] = regular_label(c, npd, ix, iy, (int)q, sub[0], sub[1], sub[2]);
        }
    return rc;
}

// The start of a run from a field file (utils.f90:223-234): parcel_default
// with init_regular_positions and init_refine (parcel_init.f90:31-166),
// init_parcels_from_grids (:170-203) and set_zeta_boundary_flag
// (parameters.f90:168-217).  Fields as in epic_oracle_set_field; rows 0..nz.
int epic_oracle_init_from_grids(epic_ctx* ctx, const double* vortg, const double* tbuoyg, const double* humg,
                                int32_t* zeta_flags) {
    if (!ctx || !vortg || !tbuoyg) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    GUARD_BEGIN
    const int npc = c.cfg.n_per_cell;
    const int npd = (int)std::pow((double)npc, f13);
    if (npd * npd * npd != npc) throw OracleError(EPIC_ERR_CONFIG, "Number of parcels per cell not a cubic.");
    const long n = (long)npc * c.nx * c.ny * c.nz;
    std::vector<double> pos(3 * n), zero3(3 * n, 0.0), B(5 * n, 0.0), vol(n), zero1(n, 0.0);
    const double im = one / (double)npd;
    long l = 0;
    for (int iz = 0; iz < c.nz; ++iz)
        for (int iy = 0; iy < c.ny; ++iy)
            for (int ix = 0; ix < c.nx; ++ix) {
                const double corner[3] = {c.lower[0] + (double)ix * c.dx[0], c.lower[1] + (double)iy * c.dx[1],
                                          c.lower[2] + (double)iz * c.dx[2]};
                for (int k = 1; k <= npd; ++k)
                    for (int j = 1; j <= npd; ++j)
                        for (int i = 1; i <= npd; ++i) {
                            pos[3 * l] = corner[0] + c.dx[0] * ((double)i - f12) * im;
                            pos[3 * l + 1] = corner[1] + c.dx[1] * ((double)j - f12) * im;
                            pos[3 * l + 2] = corner[2] + c.dx[2] * ((double)k - f12) * im;
                            ++l;
                        }
            }
    const double* d = c.dx;
    double lam = std::max({d[0] / d[1], d[1] / d[0], d[0] / d[2], d[2] / d[0], d[1] / d[2], d[2] / d[1]});
    for (long q = 0; q < n; ++q) {
        vol[q] = c.vcell / (double)npc;
        const double l23 = std::pow(lam * get_abc(vol[q]), f23);
        B[5 * q] = l23;
        B[5 * q + 3] = l23;
    }
    int rc = epic_oracle_set_parcels(ctx, n, pos.data(), zero3.data(), B.data(), vol.data(), zero1.data(),
                                     zero1.data());
    if (rc != EPIC_OK) return rc;
    if (c.cfg.labels) {
        long q = 0;
        for (int iz = 0; iz < c.nz; ++iz)
            for (int iy = 0; iy < c.ny; ++iy)
                for (int ix = 0; ix < c.nx; ++ix)
                    for (int k = 1; k <= npd; ++k)
                        for (int j = 1; j <= npd; ++j)
                            for (int i = 1; i <= npd; ++i) c.label[q++] = regular_label(c, npd, ix, iy, iz, i, j, k);
    }
    // init_refine: split until parcel 1 is less elongated than lambda_max
    while (lam >= c.cfg.lambda_max) {
        parcel_split(c);
        double D[3];
        get_eigenvalues(c, 0, D);
        lam = std::sqrt(D[0] / D[2]);
    }
    c.n_parcel_splits = c.n_parcel_merges = c.n_big_close = 0;
    // init_parcels_from_grids: the x/y halo is the periodic wrap
    Arr vg[3], bg(tbuoyg, tbuoyg + c.fsz), hg(c.fsz, 0.0);
    for (int k = 0; k < 3; ++k) vg[k].assign(vortg + k * c.fsz, vortg + (k + 1) * c.fsz);
    if (humg) hg.assign(humg, humg + c.fsz);
    for (long q = 0; q < c.n; ++q) {
        int is, js, ks;
        double ww[2][2][2];
        trilinear(c, &c.pos[3 * q], is, js, ks, ww);
        check_k(c, ks);
        for (int k = 0; k < 3; ++k) c.vor[3 * q + k] = c.vor[3 * q + k] + corner_sum(c, vg[k], is, js, ks, ww);
        c.buoy[q] = c.buoy[q] + corner_sum(c, bg, is, js, ks, ww);
        c.hum[q] = c.hum[q] + corner_sum(c, hg, is, js, ks, ww);
    }
    // set_zeta_boundary_flag on the gridded vertical vorticity
    const Arr& zeta = vg[2];
    double val[3] = {0.0, 0.0, 0.0};
    for (int ix = 0; ix < c.nx; ++ix)
        for (int iy = 0; iy < c.ny; ++iy)
            for (int iz = 1; iz <= c.nz - 1; ++iz) val[0] += zeta[c.fi(iz, iy, ix)] * zeta[c.fi(iz, iy, ix)];
    for (int ix = 0; ix < c.nx; ++ix)
        for (int iy = 0; iy < c.ny; ++iy) {
            val[1] += zeta[c.fi(0, iy, ix)] * zeta[c.fi(0, iy, ix)];
            val[2] += zeta[c.fi(c.nz, iy, ix)] * zeta[c.fi(c.nz, iy, ix)];
        }
    const double nhcelli = one / (double)((long)c.nx * c.ny);
    const double rms_interior = std::sqrt(val[0] * nhcelli / (double)(c.nz - 1));
    const double zeta_tol = (double)1.0e-3f;
    const double thres = zeta_tol * rms_interior + 2.220446049250313e-16;
    for (int b = 0; b < 2; ++b) {
        const bool z0 = std::sqrt(val[1 + b] * nhcelli) < thres;
        c.bndry_zeta_zero[b] = z0;
        c.cfg.bndry_zeta_zero[b] = z0 ? 1 : 0;
        if (zeta_flags) zeta_flags[b] = z0 ? 1 : 0;
    }
    GUARD_END
}

int epic_oracle_get_parcels(epic_ctx* ctx, int64_t cap, int64_t* n, double* pos, double* vor, double* B,
                            double* vol, double* buoy, double* hum) {
    if (!ctx || !n) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    *n = c.n;
    if (cap < c.n) { c.err = "get_parcels: capacity too small"; return EPIC_ERR_ARG; }
    if (pos) std::memcpy(pos, c.pos.data(), sizeof(double) * 3 * c.n);
    if (vor) std::memcpy(vor, c.vor.data(), sizeof(double) * 3 * c.n);
    if (B) std::memcpy(B, c.B.data(), sizeof(double) * 5 * c.n);
    if (vol) std::memcpy(vol, c.vol.data(), sizeof(double) * c.n);
    if (buoy) std::memcpy(buoy, c.buoy.data(), sizeof(double) * c.n);
    if (hum) std::memcpy(hum, c.hum.data(), sizeof(double) * c.n);
    return EPIC_OK;
}

int epic_oracle_num_parcels(epic_ctx* ctx, int64_t* n) {
    if (!ctx || !n) return EPIC_ERR_ARG;
    *n = ctx->c.n;
    return EPIC_OK;
}

int epic_oracle_get_parcel_rk(epic_ctx* ctx, int64_t cap, int64_t* n, double* dpos, double* dvor,
                              double* strain, double* dB) {
    if (!ctx || !n) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    *n = c.n;
    if (cap < c.n) return EPIC_ERR_ARG;
    if (dpos) std::memcpy(dpos, c.dpos.data(), sizeof(double) * 3 * c.n);
    if (dvor) std::memcpy(dvor, c.dvor.data(), sizeof(double) * 3 * c.n);
    if (strain) std::memcpy(strain, c.strain.data(), sizeof(double) * 8 * c.n);
    if (dB) std::memcpy(dB, c.dB.data(), sizeof(double) * 5 * c.n);
    return EPIC_OK;
}

int epic_oracle_set_parcel_rk(epic_ctx* ctx, int64_t n, const double* dpos, const double* dvor,
                              const double* dB) {
    if (!ctx) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    if (n != c.n) return EPIC_ERR_ARG;
    if (dpos) std::memcpy(c.dpos.data(), dpos, sizeof(double) * 3 * n);
    if (dvor) std::memcpy(c.dvor.data(), dvor, sizeof(double) * 3 * n);
    if (dB) std::memcpy(c.dB.data(), dB, sizeof(double) * 5 * n);
    return EPIC_OK;
}

int epic_oracle_get_field(epic_ctx* ctx, int id, double* out) {
    if (!ctx || !out) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    if (id == EPIC_FIELD_NPARG || id == EPIC_FIELD_NSPARG) {
        const std::vector<int>& v = (id == EPIC_FIELD_NPARG) ? c.nparg : c.nsparg;
        for (long i = 0; i < c.fsz; ++i) out[i] = v[i];
        return EPIC_OK;
    }
    Arr* f = field_ptr(c, id);
    if (!f) return EPIC_ERR_ARG;
    std::memcpy(out, f->data(), sizeof(double) * c.fsz);
    return EPIC_OK;
}

int epic_oracle_set_field(epic_ctx* ctx, int id, const double* in) {
    if (!ctx || !in) return EPIC_ERR_ARG;
    Arr* f = field_ptr(ctx->c, id);
    if (!f) return EPIC_ERR_ARG;
    std::memcpy(f->data(), in, sizeof(double) * ctx->c.fsz);
    return EPIC_OK;
}

int epic_oracle_init_correction(epic_ctx* ctx) { GUARD_BEGIN init_parcel_correction(ctx->c); GUARD_END }
int epic_oracle_apply_vortcor(epic_ctx* ctx) { GUARD_BEGIN apply_vortcor(ctx->c); GUARD_END }
int epic_oracle_par2grid(epic_ctx* ctx, int reuse) { GUARD_BEGIN par2grid(ctx->c, reuse != 0); GUARD_END }
int epic_oracle_vor2vel(epic_ctx* ctx) { GUARD_BEGIN vor2vel(ctx->c); GUARD_END }
int epic_oracle_vorticity_tendency(epic_ctx* ctx) { GUARD_BEGIN vorticity_tendency(ctx->c); GUARD_END }
int epic_oracle_time_step(epic_ctx* ctx, double t, double* dt) {
    GUARD_BEGIN *dt = get_time_step(ctx->c, t); GUARD_END
}
int epic_oracle_grid2par(epic_ctx* ctx, int add) { GUARD_BEGIN grid2par(ctx->c, add != 0); GUARD_END }
int epic_oracle_rk_step(epic_ctx* ctx, double* t, double* dt) {
    GUARD_BEGIN double d = rk_step(ctx->c, *t, nullptr, nullptr); if (dt) *dt = d; GUARD_END
}
int epic_oracle_merge(epic_ctx* ctx, int64_t* n_merge) {
    GUARD_BEGIN long m = parcel_merge(ctx->c); if (n_merge) *n_merge = m; GUARD_END
}
int epic_oracle_get_merge_pairs(epic_ctx* ctx, int64_t cap, int64_t* n, int32_t* isma, int32_t* iclo) {
    if (!ctx || !n) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    *n = (int64_t)c.last_isma.size();
    if (cap < *n) return EPIC_ERR_ARG;
    for (size_t m = 0; m < c.last_isma.size(); ++m) {
        if (isma) isma[m] = c.last_isma[m];
        if (iclo) iclo[m] = c.last_iclo[m];
    }
    return EPIC_OK;
}
int epic_oracle_split(epic_ctx* ctx, int64_t* n_split) {
    GUARD_BEGIN long s = parcel_split(ctx->c); if (n_split) *n_split = s; GUARD_END
}
int epic_oracle_apply_laplace(epic_ctx* ctx, int reuse) { GUARD_BEGIN apply_laplace(ctx->c, reuse != 0); GUARD_END }
int epic_oracle_apply_gradient(epic_ctx* ctx, int reuse) {
    GUARD_BEGIN apply_gradient(ctx->c, ctx->c.cfg.gradient_pref, ctx->c.cfg.max_compression, reuse != 0); GUARD_END
}
int epic_oracle_vol2grid(epic_ctx* ctx, int reuse) { GUARD_BEGIN vol2grid(ctx->c, reuse != 0); GUARD_END }
int epic_oracle_parcel_damp(epic_ctx* ctx, double dt) { GUARD_BEGIN parcel_damp(ctx->c, dt); GUARD_END }
int epic_oracle_set_bndry_fluxes(epic_ctx* ctx, const double* bflux, const double* hflux) {
    GUARD_BEGIN set_bndry_fluxes(ctx->c, bflux, hflux); GUARD_END
}
int epic_oracle_apply_bndry_fluxes(epic_ctx* ctx, double dt) { GUARD_BEGIN apply_bndry_fluxes(ctx->c, dt); GUARD_END }
int epic_oracle_parcel_diagnostics(epic_ctx* ctx, double* st) { GUARD_BEGIN parcel_diagnostics(ctx->c, st); GUARD_END }
int epic_oracle_field_diagnostics(epic_ctx* ctx, double* st) { GUARD_BEGIN field_diagnostics(ctx->c, st); GUARD_END }

int epic_oracle_step(epic_ctx* ctx, double* t, epic_step_info* info) {
    GUARD_BEGIN
    Ctx& c = ctx->c;
    epic_step_info tmp;
    if (!info) info = &tmp;
    std::memset(info, 0, sizeof(*info));
    long s0 = c.n_parcel_splits, m0 = c.n_parcel_merges;
    apply_vortcor(c);
    info->dt = rk_step(c, *t, info->parcel_stats, info->field_stats);
    parcel_merge(c);
    parcel_split(c);
    for (int it = 1; it <= c.cfg.correction_iters; ++it) {
        apply_laplace(c, it > 1);
        apply_gradient(c, c.cfg.gradient_pref, c.cfg.max_compression, true);
    }
    info->t = *t;
    info->n_parcels = c.n;
    info->n_splits = c.n_parcel_splits - s0;
    info->n_merges = c.n_parcel_merges - m0;
    GUARD_END
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Known-answer hooks for the reference's component unit tests.
extern "C" {

// scherzinger_diagonalise on a batch of symmetric matrices given as
// (B11, B12, B13, B22, B23, B33) rows; V is (n, 9) column-major per matrix.
int epic_oracle_eigen(int64_t n, const double* A6, double* D, double* V, int values_only) {
    for (int64_t i = 0; i < n; ++i) {
        const double* a = A6 + 6 * i;
        double A[9] = {a[0], a[1], a[2], a[1], a[3], a[4], a[2], a[4], a[5]};
        if (values_only) scherzinger_eigenvalues(A, D + 3 * i);
        else scherzinger_diagonalise(A, D + 3 * i, V + 9 * i);
    }
    return EPIC_OK;
}

// forfft / revfft / dst / dct on m lines of length n (dct lines hold n+1 values).
int epic_oracle_transform(int kind, int64_t m, int n, double* x) {
    if (kind <= 1) {
        RealFFT f;
        f.init(n);
        for (int64_t i = 0; i < m; ++i) (kind == 0) ? f.forfft(x + i * n) : f.revfft(x + i * n);
    } else {
        TrigTransform t;
        t.init(n);
        for (int64_t i = 0; i < m; ++i) {
            if (kind == 2) t.dst(x + i * n);
            else t.dct(x + i * (n + 1));
        }
    }
    return EPIC_OK;
}

}  // extern "C"

extern "C" int epic_oracle_test_diverge(epic_ctx* ctx, const double* phi, double* grad) {
    if (!ctx || !phi || !grad) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    Arr p(phi, phi + c.fsz), g[3];
    diverge(c, p, g);
    for (int k = 0; k < 3; ++k) {
        extrap_halo(c, g[k]);
        std::memcpy(grad + (size_t)k * c.fsz, g[k].data(), sizeof(double) * c.fsz);
    }
    return EPIC_OK;
}

// Known-answer hooks of the vertical operators, on a physical field f
// ((nz+3) x ny x nx, z fastest; rows 0 .. nz used and written):
//   op 0: fftxyp2s, lapinv1, fftxys2p              (test_lapinv1.f90)
//   op 1: fftxyp2s, central_diffz_semi_spectral, fftxys2p
//   op 2: field_decompose_physical, diffz, field_combine_physical
//                                                  (test_mpi_diffz0..5.f90)
extern "C" int epic_oracle_test_spectral(epic_ctx* ctx, int op, const double* f, double* out) {
    if (!ctx || !f || !out || op < 0 || op > 2) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    Arr fp(f, f + c.fsz), fs, ds, dp(c.fsz, 0.0);
    if (op == 0) {
        fftxyp2s(c, fp, fs);
        lapinv1(c, fs);
        fftxys2p(c, fs, dp);
    } else if (op == 1) {
        fftxyp2s(c, fp, fs);
        central_diffz_semi_spectral(c, fs, ds);
        fftxys2p(c, ds, dp);
    } else {
        field_decompose_physical(c, fp, fs);
        diffz(c, fs, ds);
        field_combine_physical(c, ds, dp);
    }
    std::memcpy(out, dp.data(), sizeof(double) * c.fsz);
    return EPIC_OK;
}

// apply_reflective_bc (parcel_bc.f90:45-57) on every parcel.
extern "C" int epic_oracle_test_reflective_bc(epic_ctx* ctx) {
    if (!ctx) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    for (long n = 0; n < c.n; ++n) apply_reflective_bc(c, &c.pos[3 * n], &c.B[5 * n]);
    return EPIC_OK;
}

// parcel_delete (test_mpi_parcel_delete.f90) of n distinct 0-based indices.
extern "C" int epic_oracle_test_delete(epic_ctx* ctx, int64_t n, const int32_t* idx) {
    if (!ctx || n < 0 || (n > 0 && !idx)) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    if (n > c.n) return EPIC_ERR_ARG;
    std::vector<long> pid(idx, idx + n);
    std::sort(pid.begin(), pid.end());
    for (auto& p : pid) p += 1;
    parcel_delete(c, pid);
    return EPIC_OK;
}
