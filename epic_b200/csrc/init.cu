// Device-side initial states (parcel_init.f90:31-152 placement and shapes,
// models/3d/beltrami_3d.f90:103-122 vorticity, the rising-thermal buoyancy of
// the benchmark workloads).  The arithmetic follows epic_b200/initial.py
// operation by operation (non-contracted products and sums), so positions
// and volumes match it bit for bit; exp/sin/cos may differ in the last bit.
#include "parcel_ops.cuh"

#include <algorithm>
#include <cmath>
#include <initializer_list>

namespace epic {

constexpr unsigned long long SM_GOLD = 0x9E3779B97F4A7C15ull;

EPIC_DEV unsigned long long splitmix64(unsigned long long x) {
    unsigned long long z = x + SM_GOLD;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// U[0, 1) keyed by (seed, parcel index, component)
EPIC_DEV double uniform01(unsigned long long seed, unsigned long long idx, int comp) {
    unsigned long long key = (seed * SM_GOLD) ^ (idx * 16ull + (unsigned long long)comp);
    unsigned long long r = splitmix64(splitmix64(key));
    return (double)(r >> 11) * (1.0 / 9007199254740992.0);
}

struct InitArgs {
    Params P;
    int kind, npd;
    long long n;
    unsigned long long seed;
    double im;            // 1 / npd
    double vol, b11;      // Vcell / n_per_cell, (lam abc)^(2/3)
    double k, l, m, alpha, fk2l2;
    int nb;
    double bub[4][4];
    double zmax;          // nextafter(upper z, lower z)
    long long* label;     // labels (cfg.labels) or null
    double* dil;
};

__global__ void k_init_state(InitArgs A, PView pv) {
    const Params& P = A.P;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < A.n;
         p += (long long)gridDim.x * blockDim.x) {
        long long q = p;
        const int i = (int)(q % A.npd) + 1; q /= A.npd;
        const int j = (int)(q % A.npd) + 1; q /= A.npd;
        const int k = (int)(q % A.npd) + 1; q /= A.npd;
        const int ix = (int)(q % P.nx); q /= P.nx;
        const int iy = (int)(q % P.ny); q /= P.ny;
        const int iz = (int)q;
        const int sub[3] = {i, j, k}, cell[3] = {ix, iy, iz};
        double pos[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            // corner + dx * (s - 0.5) * im, left to right as in initial.py
            double corner = __dadd_rn(P.lower[c], __dmul_rn((double)cell[c], P.dx[c]));
            pos[c] = __dadd_rn(corner, __dmul_rn(__dmul_rn(P.dx[c], (double)sub[c] - 0.5), A.im));
        }
        double vor[3] = {0.0, 0.0, 0.0}, buoy = 0.0;
        if (A.kind == EPIC_INIT_DEFAULT) {
            // parcel_default: regular positions, zero attributes
        } else if (A.kind == EPIC_INIT_THERMAL) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double u = uniform01(A.seed, (unsigned long long)p, c);
                pos[c] = __dadd_rn(pos[c], __dmul_rn(__dmul_rn(__dsub_rn(2.0 * u, 1.0), 0.1), P.dx[c]));
            }
            pos[2] = fmin(fmax(pos[2], P.lower[2]), A.zmax);
            for (int b = 0; b < A.nb; ++b) {
                double dx = __dsub_rn(pos[0], A.bub[b][0]), dy = __dsub_rn(pos[1], A.bub[b][1]);
                double dz = __dsub_rn(pos[2], A.bub[b][2]);
                double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                buoy = __dadd_rn(buoy, __dmul_rn(A.bub[b][3], exp(-r2 / 0.25)));
            }
            double u = uniform01(A.seed, (unsigned long long)p, 3);
            buoy = __dadd_rn(buoy, __dmul_rn(__dsub_rn(2.0 * u, 1.0), 1.0e-3));
        } else {
            // get_flow_vorticity (beltrami_3d.f90:103-122)
            double cosmz = cos(__dmul_rn(A.m, pos[2])), sinmz = sin(__dmul_rn(A.m, pos[2]));
            double arg = __dadd_rn(__dmul_rn(A.k, pos[0]), __dmul_rn(A.l, pos[1]));
            double s = sin(arg), c = cos(arg);
            vor[0] = __dmul_rn(__dmul_rn(A.fk2l2, __dsub_rn(__dmul_rn(__dmul_rn(A.k, A.m), sinmz),
                                                              __dmul_rn(__dmul_rn(A.l, A.alpha), cosmz))), s);
            vor[1] = __dmul_rn(__dmul_rn(A.fk2l2, __dadd_rn(__dmul_rn(__dmul_rn(A.l, A.m), sinmz),
                                                              __dmul_rn(__dmul_rn(A.k, A.alpha), cosmz))), s);
            vor[2] = __dmul_rn(__dmul_rn(A.alpha, cosmz), c);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            pv.set(A_X + c, p, pos[c]);
            pv.set(A_VX + c, p, vor[c]);
        }
        pv.set(A_B11, p, A.b11);
        pv.set(A_B12, p, 0.0);
        pv.set(A_B13, p, 0.0);
        pv.set(A_B22, p, A.b11);
        pv.set(A_B23, p, 0.0);
        pv.set(A_VOL, p, A.vol);
        pv.set(A_BUOY, p, buoy);
        pv.set(A_HUM, p, 0.0);
        if (A.label) {
            // parcel_init.f90:135-139
            const long long nxp = (long long)P.nx * A.npd, nyp = (long long)P.ny * A.npd;
            A.label[p] = 1 + ((long long)ix * A.npd + (i - 1)) +
                         nxp * (((long long)iy * A.npd + (j - 1)) + nyp * ((long long)iz * A.npd + (k - 1)));
            A.dil[p] = 0.0;
        }
    }
}

static void launch_init(Ctx& c, const epic_init_spec& s, int npd);

void init_state(Ctx& c, const epic_init_spec& s) {
    int npd = (int)std::lround(std::cbrt((double)s.n_per_cell));
    if (npd < 1 || npd * npd * npd != s.n_per_cell)
        throw CudaError(EPIC_ERR_CONFIG, "init_state: n_per_cell must be a cube");
    if (s.kind != EPIC_INIT_THERMAL && s.kind != EPIC_INIT_BELTRAMI)
        throw CudaError(EPIC_ERR_CONFIG, "init_state: unknown kind");
    launch_init(c, s, npd);
}

static void launch_init(Ctx& c, const epic_init_spec& s, int npd) {
    const Params& P = c.P;
    if (s.kind == EPIC_INIT_THERMAL && (s.n_bubbles < 0 || s.n_bubbles > 4))
        throw CudaError(EPIC_ERR_CONFIG, "init_state: 0 .. 4 bubbles");
    long long n = (long long)P.nx * P.ny * P.nz * s.n_per_cell;
    if (n > c.cap) throw CudaError(EPIC_ERR_CAPACITY, "init_state: more parcels than the device capacity");
    InitArgs A;
    A.P = P;
    A.kind = s.kind;
    A.npd = npd;
    A.n = n;
    A.seed = s.seed;
    A.im = 1.0 / npd;
    A.vol = P.vcell / s.n_per_cell;
    // parcel_default: spheroids of the largest cell aspect ratio (thermal), spheres (Beltrami)
    const double* d = P.dx;
    double lam = std::max({d[0] / d[1], d[1] / d[0], d[0] / d[2], d[2] / d[0], d[1] / d[2], d[2] / d[1]});
    if (s.kind == EPIC_INIT_BELTRAMI) lam = 1.0;
    double abc = 0.75 * A.vol * (1.0 / M_PI);
    A.b11 = std::pow(lam * abc, 2.0 / 3.0);
    A.k = s.k; A.l = s.l; A.m = s.m;
    A.alpha = std::sqrt(A.k * A.k + A.l * A.l + A.m * A.m);
    A.fk2l2 = s.kind == EPIC_INIT_BELTRAMI ? A.alpha / (double)(s.k * s.k + s.l * s.l) : 0.0;
    A.nb = s.kind == EPIC_INIT_THERMAL ? s.n_bubbles : 0;
    for (int b = 0; b < 4; ++b)
        for (int q = 0; q < 4; ++q) A.bub[b][q] = s.bubble[b][q];
    A.zmax = std::nextafter(P.upper[2], P.lower[2]);
    A.label = c.label;
    A.dil = c.dil;
    c.n = n;
    c.n_box = 0;
    c.n_parcel_splits = c.n_parcel_merges = c.n_big_close = 0;
    CK(cudaMemsetAsync(c.pv.base, 0, c.store_bytes(), c.stream));
    int grid = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 16));
    k_init_state<<<grid, 256, 0, c.stream>>>(A, c.pv);
    CKL();
    reset_rank(c);
    c.has_parcels = true;
}

// ---------------------------------------------------------------------------
// The start of a run from a field file (utils.f90:223-234).

// lam = sqrt(a^2 / c^2) of parcel 0 (get_eigenvalues, parcel_ellipsoid.f90:288-305)
__global__ void k_first_lambda(PView pv, double* out, unsigned* err) {
    double b[5], U[9], D[3];
    load_B(pv, 0, b);
    full_matrix<ExactOps>(b, get_B33<ExactOps>(b, pv.get(A_VOL, 0), err), U);
    sz_eigenvalues<ExactOps>(U, D);
    *out = sqrt(D[0] / D[2]);
}

// init_parcels_from_grids (parcel_init.f90:170-203): each parcel adds the
// trilinear interpolation of the gridded vorticity, buoyancy and humidity
// at its centre (x/y halo = periodic wrap).
__global__ void k_from_grids(Params P, PView pv, long long n, const double* vx, const double* vy, const double* vz,
                             const double* b, const double* h, unsigned* err) {
    PLOOP(n) {
        const double pos[3] = {pv.get(A_X, i), pv.get(A_Y, i), pv.get(A_Z, i)};
        const Tri t = trilinear(P, pos);
        long long a[2][2];
        if (!corners(P, t, a)) { set_err(err, ERRB_ZRANGE); continue; }
        pv.set(A_VX, i, pv.get(A_VX, i) + csum(vx, t, a));
        pv.set(A_VY, i, pv.get(A_VY, i) + csum(vy, t, a));
        pv.set(A_VZ, i, pv.get(A_VZ, i) + csum(vz, t, a));
        pv.set(A_BUOY, i, pv.get(A_BUOY, i) + csum(b, t, a));
        pv.set(A_HUM, i, pv.get(A_HUM, i) + csum(h, t, a));
    }
}

void init_from_grids(Ctx& c, const double* vortg, const double* tbuoyg, const double* humg, int* zeta_flags) {
    const Params& P = c.P;
    // parcel_default + init_regular_positions (parcel_init.f90:31-152)
    const int npc = c.cfg.n_per_cell;
    const int npd = (int)std::pow((double)npc, 1.0 / 3.0);
    if (npd < 1 || npd * npd * npd != npc) throw CudaError(EPIC_ERR_CONFIG, "Number of parcels per cell not a cubic.");
    epic_init_spec s{};
    s.kind = EPIC_INIT_DEFAULT;
    s.n_per_cell = npc;
    launch_init(c, s, npd);
    // init_refine (:156-166): split until parcel 1 is less elongated than lambda_max
    const double* d = P.dx;
    double lam = std::max({d[0] / d[1], d[1] / d[0], d[0] / d[2], d[2] / d[0], d[1] / d[2], d[2] / d[1]});
    while (lam >= c.cfg.lambda_max) {
        parcel_split(c);
        k_first_lambda<<<1, 1, 0, c.stream>>>(c.pv, c.partials, &c.dsc->err);
        CKL();
        CK(cudaMemcpyAsync(&lam, c.partials, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
    }
    c.n_parcel_splits = c.n_parcel_merges = c.n_big_close = 0;
    // the gridded fields into vortg, tbuoyg, humg (overwritten by the next par2grid)
    const size_t fb = sizeof(double) * (size_t)P.fsz;
    CK(cudaMemcpyAsync(c.vortg(0), vortg, 3 * fb, cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(c.tbuoyg(), tbuoyg, fb, cudaMemcpyHostToDevice, c.stream));
    if (humg) CK(cudaMemcpyAsync(c.humg(), humg, fb, cudaMemcpyHostToDevice, c.stream));
    else CK(cudaMemsetAsync(c.humg(), 0, fb, c.stream));
    k_from_grids<<<pgrid(c.n), PB, 0, c.stream>>>(P, c.pv, c.n, c.vortg(0), c.vortg(1), c.vortg(2), c.tbuoyg(),
                                                  c.humg(), &c.dsc->err);
    CKL();
    // set_zeta_boundary_flag (parameters.f90:168-217) on the host copy of zeta,
    // summed in the reference's column-major order
    const double* zeta = vortg + 2 * P.fsz;
    auto z = [&](int iz, int iy, int ix) { return zeta[fidx(P, iz, iy, ix)]; };
    double val[3] = {0.0, 0.0, 0.0};
    for (int ix = 0; ix < P.nx; ++ix)
        for (int iy = 0; iy < P.ny; ++iy)
            for (int iz = 1; iz <= P.nz - 1; ++iz) val[0] += z(iz, iy, ix) * z(iz, iy, ix);
    for (int ix = 0; ix < P.nx; ++ix)
        for (int iy = 0; iy < P.ny; ++iy) {
            val[1] += z(0, iy, ix) * z(0, iy, ix);
            val[2] += z(P.nz, iy, ix) * z(P.nz, iy, ix);
        }
    const double nhcelli = 1.0 / (double)((long long)P.nx * P.ny);
    const double rms_interior = std::sqrt(val[0] * nhcelli / (double)(P.nz - 1));
    const double thres = (double)1.0e-3f * rms_interior + 2.220446049250313e-16;   // zeta_tol, epsilon
    for (int b = 0; b < 2; ++b) {
        const bool z0 = std::sqrt(val[1 + b] * nhcelli) < thres;
        c.cfg.bndry_zeta_zero[b] = z0 ? 1 : 0;
        c.P.zeta_zero[b] = z0 ? 1 : 0;
        if (zeta_flags) zeta_flags[b] = z0 ? 1 : 0;
    }
    CK(cudaStreamSynchronize(c.stream));
}

}  // namespace epic
