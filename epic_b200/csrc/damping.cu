// Damping of parcel perturbations and surface fluxes of buoyancy and humidity.
//
// Reference semantics:
//   parcel_damp / perturbation_damping   parcel_damping.f90:43-222
//   get_strain_magnitude_field           rk_utils.f90:186-214
//   read_bndry_fluxes / bndry_fluxes_time_step / apply_bndry_fluxes
//                                        bndry_fluxes.f90:100-247
//   bilinear                             interpl.f90:65-90
// Both run once per step on the parcels (one thread per parcel) and on the
// grid (one thread per point); neither is on the hot path of a default run.
#include "parcel_ops.cuh"

#include <cmath>
#include <limits>
#include <vector>

namespace epic {

bool damping_on(const epic_cfg& g) {
    return g.damping_vorticity || g.damping_scalars || g.damping_surface_vorticity || g.damping_surface_scalars;
}

int check_damping_flags(const epic_cfg& g, std::string* msg) {
    if (g.damping_vorticity && g.damping_surface_vorticity) {
        if (msg) *msg = "damping%l_vorticity and  damping%l_surface_vorticity both activated, only one allowed";
        return EPIC_ERR_CONFIG;
    }
    if (g.damping_scalars && g.damping_surface_scalars) {
        if (msg) *msg = "damping%l_scalars and  damping%l_surface_scalars both activated, only one allowed";
        return EPIC_ERR_CONFIG;
    }
    return EPIC_OK;
}

struct VelGrad8 {
    const double* p[8];
};

// Strain magnitude sqrt(2 S:S) of the symmetrised velocity gradient at every
// grid point (rows -1 and nz+1 take the values of rows 1 and nz-1), and the
// same z reflection of vortg, humg and dbuoyg (parcel_damping.f90:56-70).
// The threads of the halo rows recompute the mirrored row's value, so no
// thread reads what another writes.
__global__ void k_damp_fields(Params P, VelGrad8 vg, double* smag, double* v0, double* v1, double* v2,
                              double* hum, double* dbuoy) {
    const long long nel = P.fsz;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nel;
         e += (long long)gridDim.x * blockDim.x) {
        const int iz = (int)(e % P.nzh) - 1;
        const long long col = e - (iz + 1);
        const int src = iz == -1 ? 1 : iz == P.nz + 1 ? P.nz - 1 : iz;
        const long long s = col + src + 1;
        double v[8];
#pragma unroll
        for (int l = 0; l < 8; ++l) v[l] = vg.p[l][s];
        const double s11 = v[I_DUDX], s12 = 0.5 * (v[I_DUDY] + v[I_DVDX]), s13 = 0.5 * (v[I_DUDZ] + v[I_DWDX]);
        const double s22 = v[I_DVDY], s23 = 0.5 * (v[I_DVDZ] + v[I_DWDY]), s33 = -(v[I_DUDX] + v[I_DVDY]);
        // row-major sum of the 9 squares, left to right
        double q = __dmul_rn(s11, s11) + __dmul_rn(s12, s12);
        q = q + __dmul_rn(s13, s13);
        q = q + __dmul_rn(s12, s12);
        q = q + __dmul_rn(s22, s22);
        q = q + __dmul_rn(s23, s23);
        q = q + __dmul_rn(s13, s13);
        q = q + __dmul_rn(s23, s23);
        q = q + __dmul_rn(s33, s33);
        smag[e] = sqrt(2.0 * q);
        if (src != iz) {
            v0[e] = v0[s];
            v1[e] = v1[s];
            v2[e] = v2[s];
            hum[e] = hum[s];
            dbuoy[e] = dbuoy[s];
        }
    }
}

struct DampArgs {
    const double* vortg[3];
    const double* humg;
    const double* dbuoyg;
    const double* smag;
    double pref_v, pref_s;
    int lv, lsv, ls, lss;
};

// perturbation_damping (parcel_damping.f90:82-222) with the stored support
// vectors (l_reuse): every support point nudges the parcel's vorticity,
// humidity and dry buoyancy towards the gridded values, weighted by the
// point's trilinear weights and 1 - exp(-prefactor * strain_mag * dt).
// Sums run over the corners in the reference's column-major order.
__global__ void k_damp(Params P, PView pv, long long n, DampArgs A, const double* dtp, unsigned* err) {
    const double dt = *dtp;
    PLOOP(n) {
        double pos[3] = {pv.get(A_X, i), pv.get(A_Y, i), pv.get(A_Z, i)};
        if (!(A.lv || A.ls)) {
            // surface damping only: parcels away from both surfaces keep their values
            if (pos[2] > P.lower[2] + 2.0 * P.dx[2] && pos[2] < P.upper[2] - 2.0 * P.dx[2]) continue;
        }
        double eta[3], tau[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) { eta[k] = pv.get(A_ETA0 + k, i); tau[k] = pv.get(A_TAU0 + k, i); }
        const double vor[3] = {pv.get(A_VX, i), pv.get(A_VY, i), pv.get(A_VZ, i)};
        const double hum = pv.get(A_HUM, i), buoy = pv.get(A_BUOY, i);
        double vortend[3] = {0.0, 0.0, 0.0}, humtend = 0.0, dbuoytend = 0.0;
        for (int p = 0; p < 4; ++p) {
            const double cp = support_cos(p), sp = support_sin(p);
            double pt[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) pt[k] = pos[k] + eta[k] * cp + tau[k] * sp;
            const Tri t = trilinear(P, pt);
            long long a[2][2];
            if (!corners(P, t, a)) { set_err(err, ERRB_ZRANGE); continue; }
            double wt[2][2][2], tf[2][2][2];
#pragma unroll
            for (int k = 0; k < 2; ++k)
#pragma unroll
                for (int j = 0; j < 2; ++j)
#pragma unroll
                    for (int ii = 0; ii < 2; ++ii) wt[k][j][ii] = 0.25 * t.w[k][j][ii];
            auto time_fact = [&](double pref) {
#pragma unroll
                for (int k = 0; k < 2; ++k)
#pragma unroll
                    for (int j = 0; j < 2; ++j)
#pragma unroll
                        for (int ii = 0; ii < 2; ++ii)
                            tf[k][j][ii] = 1.0 - exp(-pref * A.smag[a[j][ii] + k] * dt);
            };
            auto full = [&](const double* f, double x) {
                double s = 0.0;
#pragma unroll
                for (int ii = 0; ii < 2; ++ii)
#pragma unroll
                    for (int j = 0; j < 2; ++j)
#pragma unroll
                        for (int k = 0; k < 2; ++k)
                            s = s + __dmul_rn(__dmul_rn(wt[k][j][ii], tf[k][j][ii]), f[a[j][ii] + k] - x);
                return s;
            };
            auto slice = [&](const double* f, double x, int si) {
                double s = 0.0;
#pragma unroll
                for (int ii = 0; ii < 2; ++ii)
#pragma unroll
                    for (int j = 0; j < 2; ++j)
                        s = s + __dmul_rn(__dmul_rn(wt[si][j][ii], tf[si][j][ii]), f[a[j][ii] + si] - x);
                return s;
            };
            if (A.lv) {
                time_fact(A.pref_v);
#pragma unroll
                for (int l = 0; l < 3; ++l) vortend[l] = vortend[l] + full(A.vortg[l], vor[l]);
            }
            if (A.ls) {
                time_fact(A.pref_s);
                humtend = humtend + full(A.humg, hum);
                dbuoytend = dbuoytend + full(A.dbuoyg, buoy);
            }
            if (!(A.lsv || A.lss)) continue;
            // the cell rows next to a surface damp towards the surface row
            int si;
            if (t.ks == -1 || t.ks == P.nz - 1) si = 1;
            else if (t.ks == 0 || t.ks == P.nz) si = 0;
            else continue;
            if (A.lsv) {
                time_fact(A.pref_v);
#pragma unroll
                for (int l = 0; l < 3; ++l) vortend[l] = vortend[l] + slice(A.vortg[l], vor[l], si);
            }
            if (A.lss) {
                time_fact(A.pref_s);
                humtend = humtend + slice(A.humg, hum, si);
                dbuoytend = dbuoytend + slice(A.dbuoyg, buoy, si);
            }
        }
        if (A.lv || A.lsv) {
            pv.set(A_VX, i, vor[0] + vortend[0]);
            pv.set(A_VY, i, vor[1] + vortend[1]);
            pv.set(A_VZ, i, vor[2] + vortend[2]);
        }
        if (A.ls || A.lss) {
            pv.set(A_HUM, i, hum + humtend);
            pv.set(A_BUOY, i, buoy + dbuoytend);
        }
    }
}

// parcel_damp (parcel_damping.f90:43-78); dt is the step's (device scalar).
void parcel_damp(Ctx& c) {
    const epic_cfg& g = c.cfg;
    if (!damping_on(g)) return;
    par2grid(c, false, true, true);
    vor2vel(c);
    const Params& P = c.P;
    VelGrad8 vg;
    for (int k = 0; k < 8; ++k) vg.p[k] = c.velgrad(k);
    double* smag = c.w(0);   // the spectral work arrays are free until the next vor2vel
    k_damp_fields<<<pgrid(P.fsz), PB, 0, c.stream>>>(P, vg, smag, c.vortg(0), c.vortg(1), c.vortg(2), c.humg(),
                                                     c.dbuoyg());
    CKL();
    if (c.n == 0) return;
    DampArgs A;
    for (int k = 0; k < 3; ++k) A.vortg[k] = c.vortg(k);
    A.humg = c.humg();
    A.dbuoyg = c.dbuoyg();
    A.smag = smag;
    A.pref_v = g.damping_vorticity_prefactor;
    A.pref_s = g.damping_scalars_prefactor;
    A.lv = g.damping_vorticity != 0;
    A.lsv = g.damping_surface_vorticity != 0;
    A.ls = g.damping_scalars != 0;
    A.lss = g.damping_surface_scalars != 0;
    k_damp<<<pgrid(c.n), PB, 0, c.stream>>>(P, c.pv, c.n, A, &c.dsc->dt, &c.dsc->err);
    CKL();
}

// ---------------------------------------------------------------------------
// Surface fluxes

// read_bndry_fluxes (bndry_fluxes.f90:100-175) given the datasets, and the
// time-step bound of bndry_fluxes_time_step (:180-205), which depends on the
// fluxes only: alpha (dz / max|binc|)^(1/3).
void set_bndry_fluxes(Ctx& c, const double* bflux, const double* hflux) {
    const Params& P = c.P;
    c.flux_on = bflux != nullptr;
    if (!c.flux_on) return;
    const size_t m = (size_t)P.nx * P.ny;
    std::vector<double> b(bflux, bflux + m), h(m, 0.0);
    if (hflux) h.assign(hflux, hflux + m);
    double abs_max = 0.0;
    for (size_t i = 0; i < m; ++i) {
        b[i] = 2.0 * P.dxi[2] * b[i];
        h[i] = 2.0 * P.dxi[2] * h[i];
        abs_max = std::max(abs_max, std::fabs(b[i]));
    }
    c.flux_dt = c.cfg.alpha * std::pow(P.dx[2] / abs_max, 1.0 / 3.0);
    c.zdepth = P.lower[2] + P.dx[2];
    if (!c.binc) {
        CK(cudaMalloc(&c.binc, sizeof(double) * 2 * m));
        c.hinc = c.binc + m;
    }
    CK(cudaMemcpyAsync(c.binc, b.data(), sizeof(double) * m, cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(c.hinc, h.data(), sizeof(double) * m, cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
}

double flux_dt_bound(const Ctx& c) {
    return (c.flux_on && !c.cfg.use_fixed_dt) ? c.flux_dt : std::numeric_limits<double>::infinity();
}

// apply_bndry_fluxes (bndry_fluxes.f90:209-247) on its own; ls_rk_step
// applies the fluxes inside the first stage kernel.
__global__ void k_bndry_fluxes(Params P, PView pv, long long n, const double* binc, const double* hinc,
                               double zdepth, const double* dtp) {
    const double dt = *dtp;
    PLOOP(n) {
        const double pos[3] = {pv.get(A_X, i), pv.get(A_Y, i), pv.get(A_Z, i)};
        double fb, fh;
        if (!surface_flux(P, pos, binc, hinc, zdepth, dt, fb, fh)) continue;
        pv.set(A_BUOY, i, pv.get(A_BUOY, i) + fb);
        pv.set(A_HUM, i, pv.get(A_HUM, i) + fh);
    }
}

void apply_bndry_fluxes(Ctx& c) {
    if (!c.flux_on || c.n == 0) return;
    k_bndry_fluxes<<<pgrid(c.n), PB, 0, c.stream>>>(c.P, c.pv, c.n, c.binc, c.hinc, c.zdepth, &c.dsc->dt);
    CKL();
}

}  // namespace epic
