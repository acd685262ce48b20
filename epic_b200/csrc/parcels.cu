// Parcel kernels: parcel -> grid (par2grid, vol2grid), grid -> parcel fused
// with the LS-RK stage update, corrections, diagnostics and splitting.
//
// Reference semantics:
//   par2grid / vol2grid / grid2par  parcel_interpl.f90:92-470
//   trilinear                       interpl.f90:17-56
//   get_points / get_dBdt           parcel_ellipsoid.f90:216-260, 466-507
//   ls_rk_substep                   ls_rk.f90:142-217
//   apply_*                         parcel_correction.f90:42-259, parcel_bc.f90:17-57
//   parcel_split                    parcel_split.f90:37-198
//   diagnostics                     parcel_diagnostics.f90:51-159, field_diagnostics.f90:40-154
#include "parcel_ops.cuh"

#include <cub/cub.cuh>
#include <cstring>
#include <vector>
#include <algorithm>

namespace epic {

// ---------------------------------------------------------------------------
// par2grid scatter (parcel_interpl.f90:160-233)

// The scatter leaves 64-bit integer grid sums in the field arrays (q / s_f,
// s_f = 2^(b - e_f) from the field's bound in pbound, stage.cu); the tail
// folds them in integers and converts them to FP64.
EPIC_DEV double fx_inv(const unsigned long long* pbound, int k, int bits) {
    const double m = __longlong_as_double((long long)pbound[k]);
    if (!(m > 0.0 && m <= 1.0e300)) return 0.0;   // no contribution (or a non-finite one, reported by the scatter)
    int e = 0;
    frexp(m, &e);
    return ldexp(1.0, e - bits);
}

// z folds (parcel_interpl.f90:237-243, 256-275), per (x, y) column, on the
// integer sums (exact)
__global__ void k_p2g_fold(Params P, ScatterFields F, int nf, int* nparg, int* nsparg, long long* count) {
    long long ncol = (long long)P.nx * P.ny;
    long long local = 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncol;
         c += (long long)gridDim.x * blockDim.x) {
        long long t = c * P.nzh + 1;
        int nz = P.nz;
        for (int f = 0; f < nf; ++f) {
            long long* p = reinterpret_cast<long long*>(F.f[f]) + t;
            p[0] = 2 * p[0];
            p[nz] = 2 * p[nz];
            p[1] = p[1] + p[-1];
            p[nz - 1] = p[nz - 1] + p[nz + 1];
        }
        if (nparg) {
            int* q = nparg + t;
            int* s = nsparg + t;
            q[0] += q[-1];
            q[nz - 1] += q[nz];
            s[0] += s[-1];
            s[nz - 1] += s[nz];
            for (int iz = 0; iz < nz; ++iz) local += q[iz];
        }
    }
    if (nparg) {
        for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffff, local, o);
        if ((threadIdx.x & 31) == 0) atomicAdd((unsigned long long*)count, (unsigned long long)local);
    }
}

// The integer sums to FP64 on every row; rows 0 .. nz divided by the gridded
// volume, with the zeta boundary zeroing (parcel_interpl.f90:278-313).
__global__ void k_p2g_divide(Params P, ScatterFields F, const unsigned long long* pbound, int bits) {
    double inv[7];
#pragma unroll
    for (int l = 0; l < 7; ++l) inv[l] = fx_inv(pbound, l, bits);
    const long long nel = (long long)P.nx * P.ny * P.nzh;
    PLOOP(nel) {
        const int iz = (int)(i % P.nzh) - 1;
        double v[7];
#pragma unroll
        for (int l = 0; l < 7; ++l) v[l] = (double)reinterpret_cast<const long long*>(F.f[l])[i] * inv[l];
        if (iz >= 0 && iz <= P.nz) {
#pragma unroll
            for (int l = 0; l < 6; ++l) v[l] = v[l] / v[6];
            if ((iz == 0 && P.zeta_zero[0]) || (iz == P.nz && P.zeta_zero[1])) v[2] = 0.0;
        }
#pragma unroll
        for (int l = 0; l < 7; ++l) F.f[l][i] = v[l];
    }
}

// vol2grid's integer sums to FP64
__global__ void k_v2g_convert(long long fsz, double* volg, const unsigned long long* pbound, int bits) {
    const double inv = fx_inv(pbound, 6, bits);
    PLOOP(fsz) volg[i] = (double)reinterpret_cast<const long long*>(volg)[i] * inv;
}

__global__ void k_p2g_halo(Params P, ScatterFields F) {
    long long ncol = (long long)P.nx * P.ny;
    PLOOP(ncol) {
        long long t = i * P.nzh + 1;
        int nz = P.nz;
        const int which[4] = {0, 1, 2, 5};
        for (int q = 0; q < 4; ++q) {
            double* p = F.f[which[q]] + t;
            p[-1] = 2.0 * p[0] - p[1];
            p[nz + 1] = 2.0 * p[nz] - p[nz - 1];
        }
    }
}

__global__ void k_count_check(StepScalars* sc, long long n) {
    if (sc->count != n) sc->err |= (1u << 30);
}

// z folds, parcel-count check, division by the gridded volume, zeta
// zeroing and halo extrapolation after a par2grid scatter
// (parcel_interpl.f90:235-319).
void p2g_tail(Ctx& c) {
    const Params& P = c.P;
    ScatterFields F;
    F.f[0] = c.vortg(0); F.f[1] = c.vortg(1); F.f[2] = c.vortg(2);
    F.f[3] = c.dbuoyg(); F.f[4] = c.humg(); F.f[5] = c.tbuoyg(); F.f[6] = c.volg();
    long long ncol = (long long)P.nx * P.ny;
    // the parcel-count check (parcel_interpl.f90:245-250) where the scatter counted
    const bool counted = c.p2g_counted;
    k_p2g_fold<<<(int)((ncol + 255) / 256), 256, 0, c.stream>>>(P, F, 7, counted ? c.nparg : nullptr,
                                                                  c.nsparg, &c.dsc->count);
    CKL();
    if (counted) {
        k_count_check<<<1, 1, 0, c.stream>>>(c.dsc, c.n);
        CKL();
    }
    k_p2g_divide<<<pgrid((long long)P.nx * P.ny * P.nzh), PB, 0, c.stream>>>(P, F, c.dsc->pbound, p2g_fx_bits(c));
    CKL();
    k_p2g_halo<<<(int)((ncol + 255) / 256), 256, 0, c.stream>>>(P, F);
    CKL();
}

void par2grid(Ctx& c, bool reuse, bool store_vectors, bool moist) {
    scatter_p2g(c, reuse, store_vectors, moist);
    p2g_tail(c);
}

// vol2grid (parcel_interpl.f90:92-135)

void vol2grid(Ctx& c, bool reuse) {
    const Params& P = c.P;
    scatter_v2g(c, reuse);
    ScatterFields F;
    F.f[0] = c.volg();
    long long ncol = (long long)P.nx * P.ny;
    k_p2g_fold<<<(int)((ncol + 255) / 256), 256, 0, c.stream>>>(P, F, 1, nullptr, nullptr, nullptr);
    CKL();
    k_v2g_convert<<<pgrid(P.fsz), PB, 0, c.stream>>>(P.fsz, c.volg(), c.dsc->pbound, p2g_fx_bits(c));
    CKL();
}

// ---------------------------------------------------------------------------
// grid2par (+ LS-RK stage).  Gathers the 14 interpolated quantities at the 4
// support points, then (stage mode) computes dB/dt and advances the parcel.
__global__ void __launch_bounds__(PB) k_g2p(Params P, PView pv, long long n, GatherFields G, StageArgs S,
                                           const StepScalars* sc, double* partials, unsigned* err) {
    double acc[NDIAG];
#pragma unroll
    for (int k = 0; k < NDIAG; ++k) acc[k] = 0.0;
    acc[10] = 0.0; acc[11] = 0.0;   // bmin, bmax start at zero (parcel_diagnostics.f90:62-63)
    double dt = sc->dt;
    PLOOP(n) {
        double pos[3] = {pv.get(A_X, i), pv.get(A_Y, i), pv.get(A_Z, i)};
        double b[5];
        load_B(pv, i, b);
        double vol = pv.get(A_VOL, i);
        double eta[3], tau[3], D[3];
        support_vectors<FastOps>(b, vol, eta, tau, D, err);
        // grid2par stores the vectors like get_points (parcel_ellipsoid.f90:243-246)
#pragma unroll
        for (int k = 0; k < 3; ++k) { pv.set(A_ETA0 + k, i, eta[k]); pv.set(A_TAU0 + k, i, tau[k]); }
        double g[14];
#pragma unroll
        for (int l = 0; l < 14; ++l) g[l] = 0.0;
        for (int p = 0; p < 4; ++p) {
            double cp = support_cos(p), sp = support_sin(p);
            double pt[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) pt[k] = pos[k] + eta[k] * cp + tau[k] * sp;
            Tri t = trilinear(P, pt);
            long long a[2][2];
            if (!corners(P, t, a)) { set_err(err, ERRB_ZRANGE); continue; }
#pragma unroll
            for (int l = 0; l < 14; ++l) g[l] += 0.25 * csum(G.f[l], t, a);
        }
        double dp[3], dv[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            dp[k] = S.add ? pv.get(A_DX + k, i) + g[k] : g[k];
            dv[k] = S.add ? pv.get(A_DVX + k, i) + g[11 + k] : g[11 + k];
        }
        const double* strain = &g[3];
        if (S.store_strain) {
#pragma unroll
            for (int l = 0; l < 8; ++l) pv.set(A_S0 + l, i, strain[l]);
        }
        if (S.diag) {
            double vx = pv.get(A_VX, i), vy = pv.get(A_VY, i), vz = pv.get(A_VZ, i);
            double bu = pv.get(A_BUOY, i);
            acc[0] += (dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2]) * vol;
            acc[1] += (vx * vx + vy * vy + vz * vz) * vol;
            double lam = sqrt(D[0] / D[2]);
            acc[2] += lam;
            acc[3] += lam * lam;
            acc[4] += vol;
            acc[5] += vol * vol;
            if (vol <= P.vmin) acc[6] += 1.0;
            acc[7] += vol * (vx * vx);
            acc[8] += vol * (vy * vy);
            acc[9] += vol * (vz * vz);
            acc[10] = fmin(acc[10], bu);
            acc[11] = fmax(acc[11], bu);
        }
        if (S.mode == 0) {
#pragma unroll
            for (int k = 0; k < 3; ++k) { pv.set(A_DX + k, i, dp[k]); pv.set(A_DVX + k, i, dv[k]); }
            continue;
        }
        double B33 = get_B33<FastOps>(b, vol, err);
        double db[5];
        dBdt(strain, b, B33, db);
        if (S.stage > 1) {
#pragma unroll
            for (int k = 0; k < 5; ++k) db[k] = pv.get(A_DB0 + k, i) + db[k];
        }
        double cdt = S.cb * dt;
        double vor[3] = {pv.get(A_VX, i), pv.get(A_VY, i), pv.get(A_VZ, i)};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            pos[k] = pos[k] + cdt * dp[k];
            vor[k] = vor[k] + cdt * dv[k];
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) b[k] = b[k] + cdt * db[k];
        periodic_bc(P, pos);
        if (S.last) {
            reflective_bc(P, pos, b);
        } else {
#pragma unroll
            for (int k = 0; k < 3; ++k) { dp[k] = S.ca * dp[k]; dv[k] = S.ca * dv[k]; }
#pragma unroll
            for (int k = 0; k < 5; ++k) db[k] = S.ca * db[k];
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            pv.set(A_X + k, i, pos[k]);
            pv.set(A_VX + k, i, vor[k]);
            pv.set(A_DX + k, i, dp[k]);
            pv.set(A_DVX + k, i, dv[k]);
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            pv.set(A_B11 + k, i, b[k]);
            pv.set(A_DB0 + k, i, db[k]);
        }
    }
    if (S.diag) {
        // deterministic block reduction into partials[block * NDIAG + k]
        __shared__ double red[PB / 32][NDIAG];
        int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
        for (int k = 0; k < NDIAG; ++k) {
            double v = acc[k];
            for (int o = 16; o > 0; o >>= 1) {
                double u = __shfl_xor_sync(0xffffffff, v, o);
                v = (k == 10) ? fmin(v, u) : (k == 11) ? fmax(v, u) : v + u;
            }
            if (l == 0) red[w][k] = v;
        }
        __syncthreads();
        if (threadIdx.x < NDIAG) {
            int k = threadIdx.x;
            double v = red[0][k];
            for (int q = 1; q < PB / 32; ++q)
                v = (k == 10) ? fmin(v, red[q][k]) : (k == 11) ? fmax(v, red[q][k]) : v + red[q][k];
            partials[blockIdx.x * NDIAG + k] = v;
        }
    }
}

static GatherFields gather_fields(Ctx& c) {
    GatherFields G;
    for (int k = 0; k < 3; ++k) G.f[k] = c.velog(k);
    for (int k = 0; k < 8; ++k) G.f[3 + k] = c.velgrad(k);
    for (int k = 0; k < 3; ++k) G.f[11 + k] = c.vtend(k);
    G.pack = nullptr;
    return G;
}

void grid2par(Ctx& c, bool add) {
    StageArgs S;
    std::memset(&S, 0, sizeof(S));
    S.mode = 0;
    S.add = add;
    S.store_strain = 1;
    k_g2p<<<pgrid(c.n), PB, 0, c.stream>>>(c.P, c.pv, c.n, gather_fields(c), S, c.dsc, c.partials, &c.dsc->err);
    CKL();
}

void g2p_rk_stage(Ctx& c, int stage, bool with_diag) {
    StageArgs S;
    std::memset(&S, 0, sizeof(S));
    S.mode = 1;
    S.add = stage > 1;
    S.stage = stage;
    S.last = stage == c.n_stages;
    S.store_strain = 1;
    S.diag = with_diag;
    S.ca = c.ca[stage - 1];
    S.cb = c.cb[stage - 1];
    int g = pgrid(c.n);
    c.n_partials = g;
    prof_begin(c, "g2p");
    k_g2p<<<g, PB, 0, c.stream>>>(c.P, c.pv, c.n, gather_fields(c), S, c.dsc, c.partials, &c.dsc->err);
    CKL();
    prof_end(c, "g2p");
}

// Parcel statistics from the block partials (parcel_diagnostics.f90:126-157).
void finish_parcel_diag(Ctx& c, double* st) {
    std::vector<double> h((size_t)c.n_partials * NDIAG);
    const double* src = c.diag_buf ? c.diag_buf : c.partials;
    CK(cudaMemcpyAsync(h.data(), src, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c.stream));
    c.diag_buf = nullptr;
    CK(cudaStreamSynchronize(c.stream));
    double acc[NDIAG] = {0};
    for (int b = 0; b < c.n_partials; ++b)
        for (int k = 0; k < NDIAG; ++k) {
            double v = h[(size_t)b * NDIAG + k];
            if (k == 10) acc[k] = b == 0 ? v : std::min(acc[k], v);
            else if (k == 11) acc[k] = b == 0 ? v : std::max(acc[k], v);
            else acc[k] += v;
        }
    for (int k = 0; k < 18; ++k) st[k] = 0.0;
    const Params& P = c.P;
    double ntoti = 1.0 / (double)c.n;
    st[1] = 0.5 * acc[0] * P.vdomaini;
    st[12] = 0.5 * acc[1] * P.vdomaini;
    st[2] = acc[6];
    st[3] = acc[2] * ntoti;
    st[5] = std::sqrt(std::fabs(acc[3] * ntoti - st[3] * st[3]));
    st[7] = acc[4];
    st[8] = std::sqrt(acc[7] / acc[4]);
    st[9] = std::sqrt(acc[8] / acc[4]);
    st[10] = std::sqrt(acc[9] / acc[4]);
    st[4] = acc[4] * ntoti;
    st[6] = std::sqrt(std::fabs(acc[5] * ntoti - st[4] * st[4]));
    st[11] = (double)c.n;
    st[13] = (double)c.n_parcel_splits;
    st[14] = (double)c.n_big_close;
    st[15] = (double)c.n_parcel_merges;
    st[16] = std::min(0.0, acc[10]);
    st[17] = std::max(0.0, acc[11]);
}

// Standalone parcel diagnostics: needs delta_pos from a previous grid2par.
__global__ void __launch_bounds__(PB) k_pdiag(Params P, PView pv, long long n, double* partials, unsigned* err) {
    double acc[NDIAG];
#pragma unroll
    for (int k = 0; k < NDIAG; ++k) acc[k] = 0.0;
    PLOOP(n) {
        double b[5];
        load_B(pv, i, b);
        double vol = pv.get(A_VOL, i);
        double U[9], D[3];
        full_matrix<FastOps>(b, get_B33<FastOps>(b, vol, err), U);
        sz_eigenvalues<FastOps>(U, D);
        double dp0 = pv.get(A_DX, i), dp1 = pv.get(A_DY, i), dp2 = pv.get(A_DZ, i);
        double vx = pv.get(A_VX, i), vy = pv.get(A_VY, i), vz = pv.get(A_VZ, i);
        double bu = pv.get(A_BUOY, i);
        acc[0] += (dp0 * dp0 + dp1 * dp1 + dp2 * dp2) * vol;
        acc[1] += (vx * vx + vy * vy + vz * vz) * vol;
        double lam = sqrt(D[0] / D[2]);
        acc[2] += lam;
        acc[3] += lam * lam;
        acc[4] += vol;
        acc[5] += vol * vol;
        if (vol <= P.vmin) acc[6] += 1.0;
        acc[7] += vol * (vx * vx);
        acc[8] += vol * (vy * vy);
        acc[9] += vol * (vz * vz);
        acc[10] = fmin(acc[10], bu);
        acc[11] = fmax(acc[11], bu);
    }
    __shared__ double red[PB / 32][NDIAG];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < NDIAG; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) {
            double u = __shfl_xor_sync(0xffffffff, v, o);
            v = (k == 10) ? fmin(v, u) : (k == 11) ? fmax(v, u) : v + u;
        }
        if (l == 0) red[w][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < NDIAG) {
        int k = threadIdx.x;
        double v = red[0][k];
        for (int q = 1; q < PB / 32; ++q)
            v = (k == 10) ? fmin(v, red[q][k]) : (k == 11) ? fmax(v, red[q][k]) : v + red[q][k];
        partials[blockIdx.x * NDIAG + k] = v;
    }
}

void parcel_diagnostics(Ctx& c, double* out) {
    int g = pgrid(c.n);
    c.n_partials = g;
    k_pdiag<<<g, PB, 0, c.stream>>>(c.P, c.pv, c.n, c.partials, &c.dsc->err);
    CKL();
    finish_parcel_diag(c, out);
}

// ---------------------------------------------------------------------------
// Field diagnostics (field_diagnostics.f90:40-154)
struct FDArgs {
    const double* volg;
    const double* vel[3];
    const double* vor[3];
    const double* b;
    const int* nparg;
    const int* nsparg;
};

__global__ void k_fdiag2(Params P, FDArgs A, double* partials, int* iext) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // rms, abserr, nsum, nssum, ke_i, ke_b, en_i, en_b
    double bmax = -1e308, bmin = 1e308;
    int npmax = -2147483647, npmin = 2147483647;
    long long nel = (long long)P.nx * P.ny * (P.nz + 1);
    int nzp = P.nz + 1;
    PLOOP(nel) {
        long long c = i / nzp;
        int iz = (int)(i - c * nzp);
        long long a = c * P.nzh + 1 + iz;
        double v = A.volg[a];
        double dv = v - P.vcell;
        acc[0] += dv * dv;
        acc[1] = fmax(acc[1], fabs(dv));
        if (iz < P.nz) {
            acc[2] += A.nparg[a];
            acc[3] += A.nsparg[a];
            npmax = max(npmax, A.nparg[a]);
            npmin = min(npmin, A.nparg[a]);
        }
        bmax = fmax(bmax, A.b[a]);
        bmin = fmin(bmin, A.b[a]);
        double u2 = A.vel[0][a] * A.vel[0][a] + A.vel[1][a] * A.vel[1][a] + A.vel[2][a] * A.vel[2][a];
        double w2 = A.vor[0][a] * A.vor[0][a] + A.vor[1][a] * A.vor[1][a] + A.vor[2][a] * A.vor[2][a];
        if (iz == 0 || iz == P.nz) { acc[5] += v * u2; acc[7] += v * w2; }
        else { acc[4] += v * u2; acc[6] += v * w2; }
    }
    __shared__ double red[PB / 32][10];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    double vals[10] = {acc[0], acc[1], acc[2], acc[3], acc[4], acc[5], acc[6], acc[7], bmax, bmin};
#pragma unroll
    for (int k = 0; k < 10; ++k) {
        double v = vals[k];
        for (int o = 16; o > 0; o >>= 1) {
            double u = __shfl_xor_sync(0xffffffff, v, o);
            v = (k == 1 || k == 8) ? fmax(v, u) : (k == 9) ? fmin(v, u) : v + u;
        }
        if (l == 0) red[w][k] = v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        npmax = max(npmax, __shfl_xor_sync(0xffffffff, npmax, o));
        npmin = min(npmin, __shfl_xor_sync(0xffffffff, npmin, o));
    }
    if (l == 0) { atomicMax(&iext[0], npmax); atomicMin(&iext[1], npmin); }
    __syncthreads();
    if (threadIdx.x < 10) {
        int k = threadIdx.x;
        double v = red[0][k];
        for (int q = 1; q < PB / 32; ++q)
            v = (k == 1 || k == 8) ? fmax(v, red[q][k]) : (k == 9) ? fmin(v, red[q][k]) : v + red[q][k];
        partials[blockIdx.x * 10 + k] = v;
    }
}

void field_diagnostics(Ctx& c, double* st) {
    const Params& P = c.P;
    FDArgs A;
    A.volg = c.volg();
    for (int k = 0; k < 3; ++k) { A.vel[k] = c.velog(k); A.vor[k] = c.vortg(k); }
    A.b = c.tbuoyg();
    A.nparg = c.nparg;
    A.nsparg = c.nsparg;
    long long nel = (long long)P.nx * P.ny * (P.nz + 1);
    int g = pgrid(nel);
    int* iext = reinterpret_cast<int*>(c.partials + (size_t)PGRID * 40);   // past both partial blocks
    int init[2] = {-2147483647, 2147483647};
    CK(cudaMemcpyAsync(iext, init, sizeof(init), cudaMemcpyHostToDevice, c.stream));
    double* part = c.partials + (size_t)PGRID * NDIAG;
    k_fdiag2<<<g, PB, 0, c.stream>>>(P, A, part, iext);
    CKL();
    std::vector<double> h((size_t)g * 10);
    int ie[2];
    CK(cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(ie, iext, sizeof(ie), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    double a[10] = {0};
    for (int b = 0; b < g; ++b)
        for (int k = 0; k < 10; ++k) {
            double v = h[(size_t)b * 10 + k];
            if (b == 0) a[k] = v;
            else if (k == 1 || k == 8) a[k] = std::max(a[k], v);
            else if (k == 9) a[k] = std::min(a[k], v);
            else a[k] += v;
        }
    double ncelli = 1.0 / ((double)P.nx * P.ny * P.nz);
    double ngridi = 1.0 / ((double)P.nx * P.ny * (P.nz + 1));
    for (int k = 0; k < 11; ++k) st[k] = 0.0;
    st[0] = std::sqrt(a[0] * ngridi) * P.vcelli;
    st[1] = a[2] * ncelli;
    st[2] = a[3] * ncelli;
    st[3] = (0.5 * a[4] + 0.25 * a[5]) * P.vdomaini;
    st[5] = (0.5 * a[6] + 0.25 * a[7]) * P.vdomaini;
    st[6] = a[1] * P.vcelli;
    st[7] = ie[0];
    st[8] = a[8];
    st[9] = ie[1];
    st[10] = a[9];
}

// ---------------------------------------------------------------------------
// Vorticity correction (parcel_correction.f90:42-138)
__global__ void __launch_bounds__(PB) k_vortsum(PView pv, long long n, double* partials) {
    double acc[4] = {0, 0, 0, 0};
    PLOOP(n) {
        double v = pv.get(A_VOL, i);
        acc[0] += v;
        acc[1] += pv.get(A_VX, i) * v;
        acc[2] += pv.get(A_VY, i) * v;
        acc[3] += pv.get(A_VZ, i) * v;
    }
    __shared__ double red[PB / 32][4];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffff, v, o);
        if (l == 0) red[w][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0.0;
        for (int q = 0; q < PB / 32; ++q) v += red[q][threadIdx.x];
        partials[blockIdx.x * 4 + threadIdx.x] = v;
    }
}

// one warp: fixed-order sum of the partials -> dvor (or vor_bar).  Lane l
// sums blocks l, l + 32, ... in order, then a fixed butterfly adds the lanes,
// so the result does not depend on timing.
__global__ void k_vortsum_final(const double* partials, int nb, const double* vor_bar, double* out, int mode) {
    double s[4] = {0, 0, 0, 0};
    for (int b = threadIdx.x; b < nb; b += 32)
        for (int k = 0; k < 4; ++k) s[k] += partials[b * 4 + k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        for (int k = 0; k < 4; ++k) s[k] += __shfl_xor_sync(0xffffffffu, s[k], off);
    if (threadIdx.x != 0) return;
    for (int k = 0; k < 3; ++k) out[k] = mode == 0 ? s[1 + k] / s[0] : s[1 + k] / s[0] - vor_bar[k];
}

__global__ void k_vortcor_apply(PView pv, long long n, const double* dvor) {
    double d0 = dvor[0], d1 = dvor[1], d2 = dvor[2];
    PLOOP(n) {
        pv.set(A_VX, i, pv.get(A_VX, i) - d0);
        pv.set(A_VY, i, pv.get(A_VY, i) - d1);
        pv.set(A_VZ, i, pv.get(A_VZ, i) - d2);
    }
}

void init_correction(Ctx& c) {
    int g = pgrid(c.n);
    k_vortsum<<<g, PB, 0, c.stream>>>(c.pv, c.n, c.partials);
    CKL();
    k_vortsum_final<<<1, 32, 0, c.stream>>>(c.partials, g, nullptr, c.dvor_bar, 0);
    CKL();
}

void apply_vortcor(Ctx& c) {
    int g = pgrid(c.n);
    k_vortsum<<<g, PB, 0, c.stream>>>(c.pv, c.n, c.partials);
    CKL();
    double* dv = c.dvor_bar + 3;
    k_vortsum_final<<<1, 32, 0, c.stream>>>(c.partials, g, c.dvor_bar, dv, 1);
    CKL();
    k_vortcor_apply<<<g, PB, 0, c.stream>>>(c.pv, c.n, dv);
    CKL();
}

// ---------------------------------------------------------------------------
// Corrections
struct Grad3 {
    const double* g[3];
};

__global__ void k_laplace_move(Params P, PView pv, long long n, Grad3 G, unsigned* err) {
    PLOOP(n) {
        double pos[3] = {pv.get(A_X, i), pv.get(A_Y, i), pv.get(A_Z, i)};
        Tri t = trilinear(P, pos);
        long long a[2][2];
        if (!corners(P, t, a)) { set_err(err, ERRB_ZRANGE); continue; }
        double d[3];
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            double s = 0.0;
#pragma unroll
            for (int ii = 0; ii < 2; ++ii)
#pragma unroll
                for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) s += t.w[kk][jj][ii] * G.g[l][a[jj][ii] + kk];
            d[l] = s;
        }
#pragma unroll
        for (int l = 0; l < 3; ++l) pos[l] = pos[l] + d[l];
        periodic_bc(P, pos);
        pv.set(A_X, i, pos[0]);
        pv.set(A_Y, i, pos[1]);
        pv.set(A_Z, i, pos[2]);
    }
}

void apply_laplace(Ctx& c, bool reuse) {
    vol2grid(c, reuse);
    const Params& P = c.P;
    double* phi = c.w(7);
    make_phi(c, phi);
    double* grad[3] = {c.w(8), c.w(9), c.w(10)};
    diverge_laplace(c, phi, grad);
    Grad3 G;
    for (int k = 0; k < 3; ++k) G.g[k] = grad[k];
    k_laplace_move<<<pgrid(c.n), PB, 0, c.stream>>>(P, c.pv, c.n, G, &c.dsc->err);
    CKL();
}

// apply_gradient (parcel_correction.f90:183-259)
__global__ void k_gradient_move(Params P, PView pv, long long n, const double* volg, double pref, double maxc,
                                unsigned* err) {
    PLOOP(n) {
        double pos[3] = {pv.get(A_X, i), pv.get(A_Y, i), pv.get(A_Z, i)};
        Tri t = trilinear(P, pos);
        long long a[2][2];
        if (!corners(P, t, a)) { set_err(err, ERRB_ZRANGE); continue; }
        auto phi = [&](int k, int j, int ii) { return volg[a[j][ii] + k] * P.vcelli - 1.0; };
        const auto& w = t.w;
        double xf = w[0][0][1] + w[0][1][1] + w[1][0][1] + w[1][1][1];
        double yf = w[0][1][0] + w[0][1][1] + w[1][1][0] + w[1][1][1];
        double zf = w[1][0][0] + w[1][0][1] + w[1][1][0] + w[1][1][1];
        double xfc = 1.0 - xf, yfc = 1.0 - yf, zfc = 1.0 - zf;
        double lim_x = P.dx[0] * xf * xfc;
        double xs = -pref * lim_x * (zfc * (yfc * (phi(0, 0, 1) - phi(0, 0, 0)) + yf * (phi(0, 1, 1) - phi(0, 1, 0)))
                                   + zf * (yfc * (phi(1, 0, 1) - phi(1, 0, 0)) + yf * (phi(1, 1, 1) - phi(1, 1, 0))));
        lim_x = lim_x * maxc;
        xs = fmax(-lim_x, fmin(xs, lim_x));
        double lim_y = P.dx[1] * yf * yfc;
        double ys = -pref * lim_y * (zfc * (xfc * (phi(0, 1, 0) - phi(0, 0, 0)) + xf * (phi(0, 1, 1) - phi(0, 0, 1)))
                                   + zf * (xfc * (phi(1, 1, 0) - phi(1, 0, 0)) + xf * (phi(1, 1, 1) - phi(1, 0, 1))));
        lim_y = lim_y * maxc;
        ys = fmax(-lim_y, fmin(ys, lim_y));
        double lim_z = P.dx[2] * zf * zfc;
        double zs = -pref * lim_z * (xfc * (yfc * (phi(1, 0, 0) - phi(0, 0, 0)) + yf * (phi(1, 1, 0) - phi(0, 1, 0)))
                                   + xf * (yfc * (phi(1, 0, 1) - phi(0, 0, 1)) + yf * (phi(1, 1, 1) - phi(0, 1, 1))));
        lim_z = lim_z * maxc;
        zs = fmax(-lim_z, fmin(zs, lim_z));
        pos[0] = pos[0] + xs;
        pos[1] = pos[1] + ys;
        pos[2] = pos[2] + zs;
        periodic_bc(P, pos);
        pv.set(A_X, i, pos[0]);
        pv.set(A_Y, i, pos[1]);
        pv.set(A_Z, i, pos[2]);
    }
}

void apply_gradient(Ctx& c, bool reuse) {
    vol2grid(c, reuse);
    k_gradient_move<<<pgrid(c.n), PB, 0, c.stream>>>(c.P, c.pv, c.n, c.volg(), c.cfg.gradient_pref,
                                                      c.cfg.max_compression, &c.dsc->err);
    CKL();
}

__global__ void k_periodic(Params P, PView pv, long long n) {
    PLOOP(n) {
        double p[3] = {pv.get(A_X, i), pv.get(A_Y, i), pv.get(A_Z, i)};
        periodic_bc(P, p);
        pv.set(A_X, i, p[0]);
        pv.set(A_Y, i, p[1]);
    }
}

void periodic_all(Ctx& c) {
    k_periodic<<<pgrid(c.n), PB, 0, c.stream>>>(c.P, c.pv, c.n);
    CKL();
}

__global__ void k_reflective(Params P, PView pv, long long n) {
    PLOOP(n) {
        double p[3] = {pv.get(A_X, i), pv.get(A_Y, i), pv.get(A_Z, i)};
        double b[5];
        load_B(pv, i, b);
        const double z0 = p[2];
        reflective_bc(P, p, b);
        if (p[2] != z0) {
            pv.set(A_Z, i, p[2]);
            pv.set(A_B13, i, b[2]);
            pv.set(A_B23, i, b[4]);
        }
    }
}

void reflective_all(Ctx& c) {
    if (c.n == 0) return;
    k_reflective<<<pgrid(c.n), PB, 0, c.stream>>>(c.P, c.pv, c.n);
    CKL();
}

// ---------------------------------------------------------------------------
// Split (parcel_split.f90:37-198).  The test uses non-contracted arithmetic
// so the decision rounds like the oracle; children are appended in
// ascending parent order (the reference's single-thread order).
// Also bounds 0.25 V over the parcels (vbound, cleared by the host), which
// covers the children's volumes: the scale of the corrections' vol2grid.
__global__ void k_split_flag(Params P, PView pv, long long n, int* flag, unsigned long long* vbound, unsigned* err) {
    double vmax = 0.0;
    PLOOP(n) {
        double b[5];
        load_B(pv, i, b);
        const double vol = pv.get(A_VOL, i);
        vmax = (0.25 * vol > vmax || vol != vol) ? 0.25 * vol : vmax;
        const double B33 = get_B33<FastOps>(b, vol, err);
        // No split without eigenvalues when a bound proves it: every
        // eigenvalue is at most the Frobenius norm F of the full matrix, and
        // det B = abc^2 (the volume constraint that defines B33), so
        // lambda^2 = D0 / D2 = D0^2 D1 / det <= F^3 / abc^2.  The 1e-9 margin
        // covers the rounding of F and of B33; the decision is then the same
        // as the eigenvalue test's.
        const double f2 = b[0] * b[0] + b[3] * b[3] + B33 * B33 + 2.0 * (b[1] * b[1] + b[2] * b[2] + b[4] * b[4]);
        const double abc = get_abc(vol);
        const double m = 1.0 - 1e-9;
        if (f2 < P.amax2 * P.amax2 * m && f2 * sqrt(f2) < abc * abc * (P.lambda_max * P.lambda_max) * m) {
            flag[i] = 0;
            continue;
        }
        double U[9], D[3];
        // The fast eigenvalues decide where both tests are clear of their
        // thresholds by 1e-9 (they agree with the non-contracted ones to a few
        // ulps); near a threshold the decision is the oracle's arithmetic.
        full_matrix<FastOps>(b, B33, U);
        sz_eigenvalues<FastOps>(U, D);
        double lam = sqrt(D[0] / D[2]);
        const bool clear = fabs(lam - P.lambda_max) > 1e-9 * P.lambda_max && fabs(D[0] - P.amax2) > 1e-9 * P.amax2;
        if (!clear) {
            full_matrix<ExactOps>(b, get_B33<ExactOps>(b, vol, err), U);
            sz_eigenvalues<ExactOps>(U, D);
            lam = sqrt(D[0] / D[2]);
        }
        flag[i] = (lam < P.lambda_max && D[0] < P.amax2) ? 0 : 1;
    }
    vmax = isnan(vmax) ? INFINITY : vmax;
    for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffff, vmax, o));
    if ((threadIdx.x & 31) == 0 && vmax > 0.0) atomicMax(vbound, (unsigned long long)__double_as_longlong(vmax));
}

__global__ void k_split_apply(Params P, PView pv, long long n, const int* flag, const int* offs, long long* label,
                              double* dil, unsigned* err) {
    const double dh = 0.5 * 0.7745966692414834;   // f12 * sqrt(3/5)
    PLOOP(n) {
        if (!flag[i]) continue;
        long long m = n + offs[i];
        double b[5];
        load_B(pv, i, b);
        double vol = pv.get(A_VOL, i);
        double U[9], D[3], V[9];
        full_matrix<FastOps>(b, get_B33<FastOps>(b, vol, err), U);
        sz_diagonalise<FastOps>(U, D, V);
        double nb[5];
        nb[0] = b[0] - 0.75 * D[0] * (V[0] * V[0]);
        nb[1] = b[1] - 0.75 * D[0] * V[0] * V[1];
        nb[2] = b[2] - 0.75 * D[0] * V[0] * V[2];
        nb[3] = b[3] - 0.75 * D[0] * (V[1] * V[1]);
        nb[4] = b[4] - 0.75 * D[0] * V[1] * V[2];
        double hv = 0.5 * vol;
        double s = dh * sqrt(D[0]);
        double pos[3] = {pv.get(A_X, i), pv.get(A_Y, i), pv.get(A_Z, i)};
        double pc[3], pp[3], bc[5], bp[5];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double v = V[k] * s;
            pc[k] = pos[k] - v;
            pp[k] = pos[k] + v;
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) { bc[k] = nb[k]; bp[k] = nb[k]; }
        reflective_bc(P, pc, bc);
        reflective_bc(P, pp, bp);
        periodic_bc(P, pc);
        periodic_bc(P, pp);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            pv.set(A_X + k, m, pc[k]);
            pv.set(A_X + k, i, pp[k]);
            pv.set(A_VX + k, m, pv.get(A_VX + k, i));
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            pv.set(A_B11 + k, m, bc[k]);
            pv.set(A_B11 + k, i, bp[k]);
        }
        pv.set(A_VOL, m, hv);
        pv.set(A_VOL, i, hv);
        pv.set(A_BUOY, m, pv.get(A_BUOY, i));
        pv.set(A_HUM, m, pv.get(A_HUM, i));
        if (label) {   // parcel_split.f90:147-150
            label[m] = label[i];
            dil[m] = dil[i];
        }
    }
}

// Container indices of the children (box-ordered store): the reference
// appends them in ascending parent index (parcel_split.f90:132-137 with one
// thread), so child of parent i gets n + (splitting parents before rank[i]).
__global__ void k_flags_by_rank(const int* flag, const int* ord, long long n, int* flagr) {
    PLOOP(n) flagr[i] = flag[ord[i]];
}
__global__ void k_split_rank(const int* flag, const int* offs, const int* offr, long long n, int* rank) {
    PLOOP(n) {
        if (flag[i]) rank[n + offs[i]] = (int)(n + offr[rank[i]]);
    }
}

long long parcel_split(Ctx& c) {
    long long n = c.n;
    if (n == 0) return 0;
    int* flag = reinterpret_cast<int*>(c.get_scratch(0));
    // scratch layout: flag[n+1], offs[n+1], cub temp
    size_t need_cub = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need_cub, (int*)nullptr, (int*)nullptr, (int)n + 1, c.stream);
    size_t bytes = sizeof(int) * 2 * (size_t)(n + 1) + need_cub + 256;
    char* base = reinterpret_cast<char*>(c.get_scratch(bytes));
    flag = reinterpret_cast<int*>(base);
    int* offs = flag + (n + 1);
    void* tmp = reinterpret_cast<void*>((reinterpret_cast<uintptr_t>(offs + (n + 1)) + 255) & ~(uintptr_t)255);
    CK(cudaMemsetAsync(flag + n, 0, sizeof(int), c.stream));
    CK(cudaMemsetAsync(&c.dsc->vbound, 0, sizeof(unsigned long long), c.stream));
    k_split_flag<<<pgrid(n), PB, 0, c.stream>>>(c.P, c.pv, n, flag, &c.dsc->vbound, &c.dsc->err);
    CKL();
    CK(cub::DeviceScan::ExclusiveSum(tmp, need_cub, flag, offs, (int)n + 1, c.stream));
    int ns = 0;
    CK(cudaMemcpyAsync(&ns, offs + n, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if (ns == 0) return 0;
    // parcel_split.f90:91-94: a full container grows to grow_factor x the parcels needed
    const bool grow = n + ns > c.cap;
    if (grow) grow_store(c, n + ns);
    k_split_apply<<<pgrid(n), PB, 0, c.stream>>>(c.P, c.pv, n, flag, offs, c.label, c.dil, &c.dsc->err);
    CKL();
    if (c.rank) {
        auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
        char* b2 = reinterpret_cast<char*>(c.get_scratch2(al(sizeof(int) * n) + 2 * al(sizeof(int) * (n + 1)) + al(need_cub)));
        int* ord = reinterpret_cast<int*>(b2);
        int* flagr = reinterpret_cast<int*>(b2 + al(sizeof(int) * n));
        int* offr = reinterpret_cast<int*>(b2 + al(sizeof(int) * n) + al(sizeof(int) * (n + 1)));
        void* tmp2 = b2 + al(sizeof(int) * n) + 2 * al(sizeof(int) * (n + 1));
        container_order(c, ord);
        k_flags_by_rank<<<pgrid(n), PB, 0, c.stream>>>(flag, ord, n, flagr);
        CKL();
        CK(cudaMemsetAsync(flagr + n, 0, sizeof(int), c.stream));
        CK(cub::DeviceScan::ExclusiveSum(tmp2, need_cub, flagr, offr, (int)n + 1, c.stream));
        k_split_rank<<<pgrid(n), PB, 0, c.stream>>>(flag, offs, offr, n, c.rank);
        CKL();
    }
    // flag and offs live in the sort scratch: it is resized for the new
    // capacity only now, behind the kernel that reads them
    if (grow) grow_scratch_for_capacity(c);
    c.n = n + ns;
    c.n_parcel_splits += ns;
    return ns;
}

}  // namespace epic
