// Windowed shared-memory scatter (par2grid, vol2grid), the fused LS-RK
// stage kernel, and the cell-tile ordering of the parcel store.
//
// Scatter: a CTA takes a contiguous chunk of SCHUNK parcels, finds the
// bounding box of their cells, and accumulates the 4 support points x 8
// corners of every parcel into a shared-memory window of the grid covering
// that box plus the support-point reach (parcel_interpl.f90:160-233).  The
// window is added to the global fields once per CTA; points outside the
// window (strays, or a chunk too spread out for the window) go straight to
// global memory.  When the parcel store is ordered by cell tiles a chunk
// spans ~8x8x4 cells, so the global updates drop from 224 per parcel to
// about 7 per grid point of a window.
//
// Fused stage (ls_rk.f90:142-217 + parcel_interpl.f90:405-470 + the next
// stage's par2grid): pass A gathers the 14 interpolated quantities at the
// support points (using the support vectors stored by the preceding scatter,
// computed from the same B, parcel_ellipsoid.f90:216-247), computes dB/dt,
// advances x, w, B and scales the accumulators; pass B (same chunk, data hot
// in L2) computes the support vectors of the advanced shape, stores them,
// and scatters into the next stage's fields.  One parcel pass and one
// eigen-decomposition per parcel per stage instead of two of each.
#include "parcel_ops.cuh"

#include <cub/cub.cuh>
#include <cstring>

namespace epic {

constexpr int SCHUNK = 2048;     // parcels per CTA
constexpr int WMAX = 1536;       // grid points per shared-memory window

// Parcel slot of iteration k of this thread in a scatter pass: the 32 lanes
// of a warp take parcels 64 apart in the (cell-ordered) chunk, i.e. about 8
// cells apart, so one warp-wide shared-memory atomic rarely has two lanes on
// the same grid point (same-address FP64 atomics serialise); a thread's
// consecutive iterations take consecutive parcels.
EPIC_DEV int scatter_slot(int k) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    return lane * (SCHUNK / 32) + warp * (SCHUNK / PB) + k;
}

struct Window {
    int gx0, gy0, gz0;           // window origin (grid point, unwrapped)
    int WX, WY, WZ;              // extents
    int ok;
};

// Cell of a position (get_index, fields.f90:165-172).
EPIC_DEV void cell_of(const Params& P, const double* p, int& ci, int& cj, int& ck) {
    ci = (int)floor((p[0] - P.lower[0]) * P.dxi[0]);
    cj = (int)floor((p[1] - P.lower[1]) * P.dxi[1]);
    ck = (int)floor((p[2] - P.lower[2]) * P.dxi[2]);
}

struct WinBuild {
    int mn[3], mx[3];
};

EPIC_DEV void win_init(WinBuild* wb) {
    if (threadIdx.x == 0) {
        for (int k = 0; k < 3; ++k) { wb->mn[k] = 2147483647; wb->mx[k] = -2147483647; }
    }
}

EPIC_DEV void win_add(WinBuild* wb, int lmn[3], int lmx[3]) {
    for (int k = 0; k < 3; ++k) {
        int a = lmn[k], b = lmx[k];
        for (int o = 16; o > 0; o >>= 1) {
            a = min(a, __shfl_xor_sync(0xffffffff, a, o));
            b = max(b, __shfl_xor_sync(0xffffffff, b, o));
        }
        if ((threadIdx.x & 31) == 0) { atomicMin(&wb->mn[k], a); atomicMax(&wb->mx[k], b); }
    }
}

EPIC_DEV Window win_make(const Params& P, const WinBuild* wb) {
    Window W;
    W.gx0 = wb->mn[0] - 1;
    W.gy0 = wb->mn[1] - 1;
    W.gz0 = max(wb->mn[2] - 1, -1);
    W.WX = wb->mx[0] - wb->mn[0] + 4;
    W.WY = wb->mx[1] - wb->mn[1] + 4;
    int gz1 = min(wb->mx[2] + 2, P.nz + 1);
    W.WZ = gz1 - W.gz0 + 1;
    W.ok = (wb->mn[0] <= wb->mx[0]) && W.WX > 0 && W.WY > 0 && W.WZ > 0 &&
           W.WX <= P.nx && W.WY <= P.ny && (long long)W.WX * W.WY * W.WZ <= WMAX;
    return W;
}

// Scatter NF values (val[f] * weight) of one support point.  Window layout
// z fastest: w = ((x - gx0) * WY + (y - gy0)) * WZ + (z - gz0).
template <int NF>
EPIC_DEV void scatter_point(const Params& P, const Window& W, double* acc, double* const* F, const double* pt,
                            const double* val, double pw, unsigned* err) {
    Tri t = trilinear(P, pt);
    if (t.ks < -1 || t.ks > P.nz) { set_err(err, ERRB_ZRANGE); return; }
    int lx = t.is - W.gx0, ly = t.js - W.gy0, lz = t.ks - W.gz0;
    if (W.ok && lx >= 0 && lx + 1 < W.WX && ly >= 0 && ly + 1 < W.WY && lz >= 0 && lz + 1 < W.WZ) {
        int base = (lx * W.WY + ly) * W.WZ + lz;
#pragma unroll
        for (int ii = 0; ii < 2; ++ii)
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    int w = base + (ii * W.WY + jj) * W.WZ + kk;
                    double wt = pw * t.w[kk][jj][ii];
#pragma unroll
                    for (int f = 0; f < NF; ++f) atomicAdd(&acc[f * WMAX + w], wt * val[f]);
                }
    } else {
        long long a[2][2];
        corners(P, t, a);
#pragma unroll
        for (int ii = 0; ii < 2; ++ii)
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    long long g = a[jj][ii] + kk;
                    double wt = pw * t.w[kk][jj][ii];
#pragma unroll
                    for (int f = 0; f < NF; ++f) atomicAdd(&F[f][g], wt * val[f]);
                }
    }
}

template <int NF>
EPIC_DEV void win_zero(double* acc, const Window& W) {
    if (!W.ok) return;
    int n = W.WX * W.WY * W.WZ;
    for (int f = 0; f < NF; ++f)
        for (int w = threadIdx.x; w < n; w += blockDim.x) acc[f * WMAX + w] = 0.0;
}

template <int NF>
EPIC_DEV void win_flush(const Params& P, const double* acc, const Window& W, double* const* F) {
    if (!W.ok) return;
    int n = W.WX * W.WY * W.WZ;
    for (int w = threadIdx.x; w < n; w += blockDim.x) {
        int z = w % W.WZ;
        int r = w / W.WZ;
        int y = r % W.WY;
        int x = r / W.WY;
        long long g = fidx(P, W.gz0 + z, wrapi(W.gy0 + y, P.ny), wrapi(W.gx0 + x, P.nx));
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            double v = acc[f * WMAX + w];
            if (v != 0.0) atomicAdd(&F[f][g], v);
        }
    }
}

struct Fields7 {
    double* f[7];   // vortg x,y,z, dbuoyg, humg, tbuoyg, volg
};

// Values scattered by par2grid for one parcel (parcel_interpl.f90:177-230).
EPIC_DEV void p2g_values(const Params& P, const PView& pv, long long i, double* val, double& pw) {
    double z = pv.at(A_Z, i);
    double vol = pv.at(A_VOL, i), buoy = pv.at(A_BUOY, i), hum = pv.at(A_HUM, i);
    double q_c = hum - P.q_0 * exp(P.lambda_c * (P.lower[2] - z));
    q_c = fmax(0.0, q_c);
    val[0] = pv.at(A_VX, i);
    val[1] = pv.at(A_VY, i);
    val[2] = pv.at(A_VZ, i);
    val[3] = buoy;
    val[4] = hum;
    val[5] = buoy + P.glat * q_c;
    val[6] = 1.0;
    pw = 0.25 * vol;
}

EPIC_DEV void count_parcel(const Params& P, const double* pos, double vol, int* nparg, int* nsparg, unsigned* err) {
    int ci, cj, ck;
    cell_of(P, pos, ci, cj, ck);
    if (ck < -1 || ck > P.nz) { set_err(err, ERRB_ZRANGE); return; }
    long long g = fidx(P, ck, wrapi(cj, P.ny), wrapi(ci, P.nx));
    atomicAdd(&nparg[g], 1);
    if (vol <= P.vmin) atomicAdd(&nsparg[g], 1);
}

// par2grid scatter (mode 0) and vol2grid (mode 1).
template <int NF>
__global__ void __launch_bounds__(PB) k_scatter(Params P, PView pv, long long n, Fields7 F, int* nparg, int* nsparg,
                                               int reuse, int store, unsigned* err) {
    extern __shared__ double acc[];
    __shared__ WinBuild wb;
    __shared__ Window Ws;
    long long b0 = (long long)blockIdx.x * SCHUNK;
    long long b1 = min(b0 + (long long)SCHUNK, n);
    win_init(&wb);
    __syncthreads();
    int lmn[3] = {2147483647, 2147483647, 2147483647}, lmx[3] = {-2147483647, -2147483647, -2147483647};
    for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        double p[3] = {pv.at(A_X, i), pv.at(A_Y, i), pv.at(A_Z, i)};
        int c[3];
        cell_of(P, p, c[0], c[1], c[2]);
        for (int k = 0; k < 3; ++k) { lmn[k] = min(lmn[k], c[k]); lmx[k] = max(lmx[k], c[k]); }
    }
    win_add(&wb, lmn, lmx);
    __syncthreads();
    if (threadIdx.x == 0) Ws = win_make(P, &wb);
    __syncthreads();
    const Window W = Ws;
    win_zero<NF>(acc, W);
    __syncthreads();
    for (int k = 0; k < SCHUNK / PB; ++k) {
        long long i = b0 + scatter_slot(k);
        if (i >= b1) continue;
        double pos[3] = {pv.at(A_X, i), pv.at(A_Y, i), pv.at(A_Z, i)};
        double eta[3], tau[3];
        get_vectors(pv, i, reuse != 0, store != 0, eta, tau, nullptr, err);
        double val[7], pw;
        if (NF == 7) {
            p2g_values(P, pv, i, val, pw);
            count_parcel(P, pos, pv.at(A_VOL, i), nparg, nsparg, err);
        } else {
            val[0] = 1.0;
            pw = 0.25 * pv.at(A_VOL, i);
        }
        for (int p = 0; p < 4; ++p) {
            double cp = support_cos(p), sp = support_sin(p);
            double pt[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) pt[k] = pos[k] + eta[k] * cp + tau[k] * sp;
            scatter_point<NF>(P, W, acc, F.f, pt, val, pw, err);
        }
    }
    __syncthreads();
    win_flush<NF>(P, acc, W, F.f);
}

// ---------------------------------------------------------------------------
// Fused stage kernel.
struct FusedArgs {
    int stage, last, diag, scatter;
    double ca, cb;
};

__global__ void __launch_bounds__(PB) k_stage(Params P, PView pv, long long n, GatherFields G, Fields7 F, int* nparg,
                                             int* nsparg, FusedArgs S, const StepScalars* sc, double* partials,
                                             unsigned* err) {
    extern __shared__ double acc[];
    __shared__ WinBuild wb;
    __shared__ Window Ws;
    __shared__ double red[PB / 32][NDIAG];
    double dacc[NDIAG];
#pragma unroll
    for (int k = 0; k < NDIAG; ++k) dacc[k] = 0.0;
    const double dt = sc->dt;
    long long b0 = (long long)blockIdx.x * SCHUNK;
    long long b1 = min(b0 + (long long)SCHUNK, n);
    win_init(&wb);
    __syncthreads();
    int lmn[3] = {2147483647, 2147483647, 2147483647}, lmx[3] = {-2147483647, -2147483647, -2147483647};
    // pass A: grid2par + dB/dt + LS-RK update
    for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        double pos[3] = {pv.at(A_X, i), pv.at(A_Y, i), pv.at(A_Z, i)};
        double b[5];
        load_B(pv, i, b);
        double vol = pv.at(A_VOL, i);
        double eta[3], tau[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) { eta[k] = pv.at(A_ETA0 + k, i); tau[k] = pv.at(A_TAU0 + k, i); }
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
        double dp[3], dv[3], vor[3] = {pv.at(A_VX, i), pv.at(A_VY, i), pv.at(A_VZ, i)};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            dp[k] = S.stage > 1 ? pv.at(A_DX + k, i) + g[k] : g[k];
            dv[k] = S.stage > 1 ? pv.at(A_DVX + k, i) + g[11 + k] : g[11 + k];
        }
        const double* strain = &g[3];
        if (S.diag) {
            // parcel diagnostics before the update (ls_rk.f90:116, parcel_diagnostics.f90:66-120)
            double U[9], D[3];
            full_matrix<FastOps>(b, get_B33<FastOps>(b, vol, err), U);
            sz_eigenvalues<FastOps>(U, D);
            double bu = pv.at(A_BUOY, i);
            dacc[0] += (dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2]) * vol;
            dacc[1] += (vor[0] * vor[0] + vor[1] * vor[1] + vor[2] * vor[2]) * vol;
            double lam = sqrt(D[0] / D[2]);
            dacc[2] += lam;
            dacc[3] += lam * lam;
            dacc[4] += vol;
            dacc[5] += vol * vol;
            if (vol <= P.vmin) dacc[6] += 1.0;
            dacc[7] += vol * (vor[0] * vor[0]);
            dacc[8] += vol * (vor[1] * vor[1]);
            dacc[9] += vol * (vor[2] * vor[2]);
            dacc[10] = fmin(dacc[10], bu);
            dacc[11] = fmax(dacc[11], bu);
        }
        double B33 = get_B33<FastOps>(b, vol, err);
        double db[5];
        dBdt(strain, b, B33, db);
        if (S.stage > 1) {
#pragma unroll
            for (int k = 0; k < 5; ++k) db[k] = pv.at(A_DB0 + k, i) + db[k];
        }
        double cdt = S.cb * dt;
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
            pv.at(A_X + k, i) = pos[k];
            pv.at(A_VX + k, i) = vor[k];
            pv.at(A_DX + k, i) = dp[k];
            pv.at(A_DVX + k, i) = dv[k];
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            pv.at(A_B11 + k, i) = b[k];
            pv.at(A_DB0 + k, i) = db[k];
        }
        int c[3];
        cell_of(P, pos, c[0], c[1], c[2]);
        for (int k = 0; k < 3; ++k) { lmn[k] = min(lmn[k], c[k]); lmx[k] = max(lmx[k], c[k]); }
    }
    if (S.diag) {
        int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
        for (int k = 0; k < NDIAG; ++k) {
            double v = dacc[k];
            for (int o = 16; o > 0; o >>= 1) {
                double u = __shfl_xor_sync(0xffffffff, v, o);
                v = (k == 10) ? fmin(v, u) : (k == 11) ? fmax(v, u) : v + u;
            }
            if (l == 0) red[w][k] = v;
        }
    }
    if (!S.scatter) {
        if (S.diag) {
            __syncthreads();
            if (threadIdx.x < NDIAG) {
                int k = threadIdx.x;
                double v = red[0][k];
                for (int q = 1; q < PB / 32; ++q)
                    v = (k == 10) ? fmin(v, red[q][k]) : (k == 11) ? fmax(v, red[q][k]) : v + red[q][k];
                partials[blockIdx.x * NDIAG + k] = v;
            }
        }
        return;
    }
    win_add(&wb, lmn, lmx);
    __syncthreads();
    if (S.diag && threadIdx.x < NDIAG) {
        int k = threadIdx.x;
        double v = red[0][k];
        for (int q = 1; q < PB / 32; ++q)
            v = (k == 10) ? fmin(v, red[q][k]) : (k == 11) ? fmax(v, red[q][k]) : v + red[q][k];
        partials[blockIdx.x * NDIAG + k] = v;
    }
    if (threadIdx.x == 0) Ws = win_make(P, &wb);
    __syncthreads();
    const Window W = Ws;
    win_zero<7>(acc, W);
    __syncthreads();
    // pass B: support vectors of the advanced shape + next par2grid
    for (int k = 0; k < SCHUNK / PB; ++k) {
        long long i = b0 + scatter_slot(k);
        if (i >= b1) continue;
        double pos[3] = {pv.at(A_X, i), pv.at(A_Y, i), pv.at(A_Z, i)};
        double eta[3], tau[3];
        get_vectors(pv, i, false, true, eta, tau, nullptr, err);
        double val[7], pw;
        p2g_values(P, pv, i, val, pw);
        count_parcel(P, pos, pv.at(A_VOL, i), nparg, nsparg, err);
        for (int p = 0; p < 4; ++p) {
            double cp = support_cos(p), sp = support_sin(p);
            double pt[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) pt[k] = pos[k] + eta[k] * cp + tau[k] * sp;
            scatter_point<7>(P, W, acc, F.f, pt, val, pw, err);
        }
    }
    __syncthreads();
    win_flush<7>(P, acc, W, F.f);
}

// ---------------------------------------------------------------------------
static Fields7 fields7(Ctx& c) {
    Fields7 F;
    F.f[0] = c.vortg(0); F.f[1] = c.vortg(1); F.f[2] = c.vortg(2);
    F.f[3] = c.dbuoyg(); F.f[4] = c.humg(); F.f[5] = c.tbuoyg(); F.f[6] = c.volg();
    return F;
}

static int sgrid(long long n) { return (int)std::max<long long>(1, (n + SCHUNK - 1) / SCHUNK); }

static void zero_p2g_fields(Ctx& c) {
    const Params& P = c.P;
    // the 7 scattered fields are contiguous slots 3..5 and 17..20 of the field block
    CK(cudaMemsetAsync(c.vortg(0), 0, sizeof(double) * 3 * P.fsz, c.stream));
    CK(cudaMemsetAsync(c.tbuoyg(), 0, sizeof(double) * 4 * P.fsz, c.stream));
    CK(cudaMemsetAsync(c.nparg, 0, sizeof(int) * P.fsz, c.stream));
    CK(cudaMemsetAsync(c.nsparg, 0, sizeof(int) * P.fsz, c.stream));
    CK(cudaMemsetAsync(&c.dsc->count, 0, sizeof(long long), c.stream));
}

void scatter_p2g(Ctx& c, bool reuse, bool store) {
    zero_p2g_fields(c);
    if (c.n == 0) return;
    size_t sm = sizeof(double) * 7 * WMAX;
    CK(cudaFuncSetAttribute(k_scatter<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    prof_begin(c, "p2g");
    k_scatter<7><<<sgrid(c.n), PB, sm, c.stream>>>(c.P, c.pv, c.n, fields7(c), c.nparg, c.nsparg, reuse, store,
                                                     &c.dsc->err);
    CKL();
    prof_end(c, "p2g");
}

void scatter_v2g(Ctx& c, bool reuse) {
    CK(cudaMemsetAsync(c.volg(), 0, sizeof(double) * c.P.fsz, c.stream));
    if (c.n == 0) return;
    Fields7 F;
    F.f[0] = c.volg();
    size_t sm = sizeof(double) * 1 * WMAX;
    prof_begin(c, "v2g");
    k_scatter<1><<<sgrid(c.n), PB, sm, c.stream>>>(c.P, c.pv, c.n, F, nullptr, nullptr, reuse, 1, &c.dsc->err);
    CKL();
    prof_end(c, "v2g");
}

// One LS-RK stage (grid2par + update) fused with the next stage's par2grid
// scatter (not after the last stage).
void fused_stage(Ctx& c, int stage, bool with_diag) {
    FusedArgs S;
    S.stage = stage;
    S.last = stage == c.n_stages;
    S.diag = with_diag;
    S.scatter = !S.last;
    S.ca = c.ca[stage - 1];
    S.cb = c.cb[stage - 1];
    GatherFields G;
    for (int k = 0; k < 3; ++k) G.f[k] = c.velog(k);
    for (int k = 0; k < 8; ++k) G.f[3 + k] = c.velgrad(k);
    for (int k = 0; k < 3; ++k) G.f[11 + k] = c.vtend(k);
    if (S.scatter) zero_p2g_fields(c);
    int g = sgrid(c.n);
    if (with_diag) {
        c.n_partials = g;
        c.diag_buf = c.stage_partials;
    }
    size_t sm = S.scatter ? sizeof(double) * 7 * WMAX : 0;
    CK(cudaFuncSetAttribute(k_stage, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(double) * 7 * WMAX)));
    prof_begin(c, "stage");
    k_stage<<<g, PB, sm, c.stream>>>(c.P, c.pv, c.n, G, fields7(c), c.nparg, c.nsparg, S, c.dsc, c.stage_partials,
                                      &c.dsc->err);
    CKL();
    prof_end(c, "stage");
}

// ---------------------------------------------------------------------------
// Cell-tile ordering of the parcel store: key = 8^3-cell tile (x fastest),
// then the cell inside the tile (x fastest).  Only the attributes live at the
// start of a step are moved (state and support vectors).
__global__ void k_sort_keys(Params P, PView pv, long long n, unsigned* key, int* idx) {
    int ntx = (P.nx + 7) >> 3, nty = (P.ny + 7) >> 3;
    PLOOP(n) {
        double p[3] = {pv.at(A_X, i), pv.at(A_Y, i), pv.at(A_Z, i)};
        int ci, cj, ck;
        cell_of(P, p, ci, cj, ck);
        ci = min(max(ci, 0), P.nx - 1);
        cj = min(max(cj, 0), P.ny - 1);
        ck = min(max(ck, 0), P.nz - 1);
        unsigned tile = (unsigned)(((ck >> 3) * nty + (cj >> 3)) * ntx + (ci >> 3));
        unsigned local = (unsigned)(((ck & 7) * 8 + (cj & 7)) * 8 + (ci & 7));
        key[i] = tile * 512u + local;
        idx[i] = (int)i;
    }
}

__global__ void k_permute(PView src, PView dst, long long n, const int* perm) {
    const int attrs[20] = {A_X, A_Y, A_Z, A_VX, A_VY, A_VZ, A_B11, A_B12, A_B13, A_B22, A_B23, A_VOL, A_BUOY, A_HUM,
                           A_ETA0, A_ETA0 + 1, A_ETA0 + 2, A_TAU0, A_TAU0 + 1, A_TAU0 + 2};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * 20;
         t += (long long)gridDim.x * blockDim.x) {
        int a = (int)(t / n);
        long long i = t - (long long)a * n;
        int k = attrs[a];
        dst.at(k, i) = src.at(k, perm[i]);
    }
}

void sort_parcels(Ctx& c) {
    long long n = c.n;
    if (n < 2 || c.pv_alt == nullptr) return;
    size_t cubb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, cubb, (unsigned*)0, (unsigned*)0, (int*)0, (int*)0, (int)n, 0, 32,
                                    c.stream);
    size_t bytes = 4 * ((sizeof(unsigned) * n + 255) & ~(size_t)255) + cubb + 1024;
    char* base = reinterpret_cast<char*>(c.get_scratch(bytes));
    auto take = [&](size_t b) { char* p = base; base += (b + 255) & ~(size_t)255; return p; };
    unsigned* k0 = reinterpret_cast<unsigned*>(take(sizeof(unsigned) * n));
    unsigned* k1 = reinterpret_cast<unsigned*>(take(sizeof(unsigned) * n));
    int* i0 = reinterpret_cast<int*>(take(sizeof(int) * n));
    int* i1 = reinterpret_cast<int*>(take(sizeof(int) * n));
    void* tmp = take(cubb);
    k_sort_keys<<<pgrid(n), PB, 0, c.stream>>>(c.P, c.pv, n, k0, i0);
    CKL();
    int ntx = (c.P.nx + 7) >> 3, nty = (c.P.ny + 7) >> 3, ntz = (c.P.nz + 7) >> 3;
    unsigned long long maxkey = (unsigned long long)ntx * nty * ntz * 512ull;
    int endbit = 1;
    while ((1ull << endbit) < maxkey) ++endbit;
    CK(cub::DeviceRadixSort::SortPairs(tmp, cubb, k0, k1, i0, i1, (int)n, 0, endbit, c.stream));
    PView dst{c.pv_alt, c.cap};
    k_permute<<<pgrid(n * 20), PB, 0, c.stream>>>(c.pv, dst, n, i1);
    CKL();
    std::swap(c.pv.base, c.pv_alt);
}

}  // namespace epic
