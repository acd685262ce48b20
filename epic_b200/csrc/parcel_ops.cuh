// Device helpers shared by the parcel kernels (parcels.cu, stage.cu).
#pragma once
#include "ctx.hpp"
#include "eigen.cuh"

#include <algorithm>

namespace epic {

constexpr int PB = 256;          // threads per block for parcel kernels
constexpr int PGRID = 148 * 8;   // fixed grid for deterministic reductions

inline int pgrid(long long n) {
    long long b = (n + PB - 1) / PB;
    return (int)std::max<long long>(1, std::min<long long>(b, PGRID));
}

#define PLOOP(n) for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); \
                      i += (long long)gridDim.x * blockDim.x)

struct Tri {
    int is, js, ks;
    double w[2][2][2];   // w[k][j][i]
};

// trilinear (interpl.f90:17-56)
EPIC_DEV Tri trilinear(const Params& P, const double* p) {
    Tri t;
    double x = (p[0] - P.lower[0]) * P.dxi[0];
    double y = (p[1] - P.lower[1]) * P.dxi[1];
    double z = (p[2] - P.lower[2]) * P.dxi[2];
    t.is = (int)floor(x); t.js = (int)floor(y); t.ks = (int)floor(z);
    double px = x - (double)t.is, pxc = 1.0 - px;
    double py = y - (double)t.js, pyc = 1.0 - py;
    double pz = z - (double)t.ks, pzc = 1.0 - pz;
    double w00 = pyc * pxc, w10 = pyc * px, w01 = py * pxc, w11 = py * px;
    t.w[0][0][0] = pzc * w00; t.w[0][0][1] = pzc * w10; t.w[0][1][0] = pzc * w01; t.w[0][1][1] = pzc * w11;
    t.w[1][0][0] = pz * w00;  t.w[1][0][1] = pz * w10;  t.w[1][1][0] = pz * w01;  t.w[1][1][1] = pz * w11;
    return t;
}

// Addresses of the 8 corners (periodic in x, y).  Returns false if the
// vertical index leaves the halo (the reference would index out of bounds).
EPIC_DEV bool corners(const Params& P, const Tri& t, long long a[2][2]) {
    if (t.ks < -1 || t.ks > P.nz) return false;
    int i0 = wrapi(t.is, P.nx), i1 = wrapi(t.is + 1, P.nx);
    int j0 = wrapi(t.js, P.ny), j1 = wrapi(t.js + 1, P.ny);
    a[0][0] = fidx(P, t.ks, j0, i0);
    a[0][1] = fidx(P, t.ks, j0, i1);
    a[1][0] = fidx(P, t.ks, j1, i0);
    a[1][1] = fidx(P, t.ks, j1, i1);
    return true;
}

// sum(weights * f(ks:ks+1, js:js+1, is:is+1)) in column-major order
EPIC_DEV double csum(const double* f, const Tri& t, const long long a[2][2]) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            long long b = a[j][i];
            s = fma(t.w[0][j][i], f[b], s);
            s = fma(t.w[1][j][i], f[b + 1], s);
        }
    return s;
}

EPIC_DEV void load_B(const PView& pv, long long i, double* b) {
#pragma unroll
    for (int k = 0; k < 5; ++k) b[k] = pv.get(A_B11 + k, i);
}

// Support vectors: recomputed, or reused from the parcel store (l_reuse).
EPIC_DEV void get_vectors(const PView& pv, long long i, bool reuse, bool store, double* eta, double* tau,
                          double* D, unsigned* err) {
    if (reuse) {
#pragma unroll
        for (int k = 0; k < 3; ++k) { eta[k] = pv.get(A_ETA0 + k, i); tau[k] = pv.get(A_TAU0 + k, i); }
        return;
    }
    double b[5];
    load_B(pv, i, b);
    support_vectors<FastOps>(b, pv.get(A_VOL, i), eta, tau, D, err);
    if (store) {
#pragma unroll
        for (int k = 0; k < 3; ++k) { pv.set(A_ETA0 + k, i, eta[k]); pv.set(A_TAU0 + k, i, tau[k]); }
    }
}

struct ScatterFields {
    double* f[7];   // vortg x,y,z, dbuoyg, humg, tbuoyg, volg
};

struct GatherFields {
    const double* f[14];   // velog 3, velgradg 8, vtend 3
    const double* pack;    // the same, 16 doubles per grid point (fused stage)
};

struct StageArgs {
    int mode;          // 0: grid2par only, 1: RK stage
    int add;           // grid2par(add)
    int stage;         // 1-based
    int last;
    int store_strain;
    int diag;          // accumulate parcel diagnostics (stage 1)
    double ca, cb;
};

// get_dBdt (parcel_ellipsoid.f90:466-507)
EPIC_DEV void dBdt(const double* s, const double* b, double B33, double* o) {
    double dwdz = -(s[I_DUDX] + s[I_DVDY]);
    o[0] = 2.0 * (s[I_DUDX] * b[0] + s[I_DUDY] * b[1] + s[I_DUDZ] * b[2]);
    o[1] = s[I_DVDX] * b[0] - dwdz * b[1] + s[I_DVDZ] * b[2] + s[I_DUDY] * b[3] + s[I_DUDZ] * b[4];
    o[2] = s[I_DWDX] * b[0] + s[I_DWDY] * b[1] - s[I_DVDY] * b[2] + s[I_DUDY] * b[4] + s[I_DUDZ] * B33;
    o[3] = 2.0 * (s[I_DVDX] * b[1] + s[I_DVDY] * b[3] + s[I_DVDZ] * b[4]);
    o[4] = s[I_DWDX] * b[1] + s[I_DVDX] * b[2] + s[I_DWDY] * b[3] - s[I_DUDX] * b[4] + s[I_DVDZ] * B33;
}

// apply_periodic_bc / apply_reflective_bc (parcel_bc.f90:17-42)
EPIC_DEV void periodic_bc(const Params& P, double* p) {
    p[0] = p[0] - P.extent[0] * (double)(int)((p[0] - P.center[0]) * P.hli[0]);
    p[1] = p[1] - P.extent[1] * (double)(int)((p[1] - P.center[1]) * P.hli[1]);
}
EPIC_DEV void reflective_bc(const Params& P, double* p, double* b) {
    if (p[2] > P.upper[2]) {
        p[2] = 2.0 * P.upper[2] - p[2];
        b[2] = -b[2]; b[4] = -b[4];
    } else if (p[2] < P.lower[2]) {
        p[2] = 2.0 * P.lower[2] - p[2];
        b[2] = -b[2]; b[4] = -b[4];
    }
}

// apply_bndry_fluxes (bndry_fluxes.f90:209-247) for one parcel: below
// zdepth = lower + dz the parcel gains fb = fac * bilinear(binc) of buoyancy
// and fh = fac * bilinear(hinc) of humidity, fac = (zdepth - z) dxi dt;
// binc, hinc are (ny, nx), y fastest; bilinear weights ww[j][i]
// (interpl.f90:65-90).  Returns false (no change) above zdepth.
EPIC_DEV bool surface_flux(const Params& P, const double* pos, const double* binc, const double* hinc,
                           double zdepth, double dt, double& fb, double& fh) {
    const double z = pos[2];
    if (!(z < zdepth)) return false;
    const double x = (pos[0] - P.lower[0]) * P.dxi[0];
    const double y = (pos[1] - P.lower[1]) * P.dxi[1];
    const int is = (int)floor(x), js = (int)floor(y);
    const double px = x - (double)is, pxc = 1.0 - px;
    const double py = y - (double)js, pyc = 1.0 - py;
    const double ww[2][2] = {{pyc * pxc, pyc * px}, {py * pxc, py * px}};
    const double fac = (zdepth - z) * P.dxi[2] * dt;
    double sb = 0.0, sh = 0.0;
#pragma unroll
    for (int ii = 0; ii < 2; ++ii)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const long long h = (long long)wrapi(is + ii, P.nx) * P.ny + wrapi(js + j, P.ny);
            sb = sb + __dmul_rn(ww[j][ii], binc[h]);
            sh = sh + __dmul_rn(ww[j][ii], hinc[h]);
        }
    fb = fac * sb;
    fh = fac * sh;
    return true;
}

constexpr int NDIAG = 12;   // KE ENS LAM LAM2 VOL VOL2 NSMALL XI2 ETA2 ZETA2 BMIN BMAX


}  // namespace epic
