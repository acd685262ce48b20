// C ABI of the B200 EPIC step (include/epic_gpu.h): context lifecycle,
// host <-> device parcel/field exchange and the step driver
// (epic3d.f90:135-153, ls_rk.f90:88-217).
#include "ctx.hpp"
#include "ncfile.hpp"
#include "../../include/epic_nc.h"

#include <cmath>
#include <cstring>
#include <algorithm>

using namespace epic;

struct epic_ctx {
    Ctx c;
};

namespace epic {

std::atomic<long long> g_launches{0};

// parcels%resize (parcel_container.f90:273-308): reallocate the store for at
// least grow_factor x need parcels, keeping parcels [0, n); the sort buffer
// and the per-CTA partials follow the new capacity.  The sort and merge
// scratch are not touched here (the caller may still have live data in them):
// grow_scratch_for_capacity sizes them once that data is read.
void grow_store(Ctx& c, long long need) {
    long long ncap = std::max(need, (long long)std::llround(c.cfg.grow_factor * (double)need));
    ncap = (ncap + 63) & ~63LL;
    PView nv{nullptr, ncap, c.pv.mixed};
    const size_t nbytes = (size_t)(c.pv.mixed ? PARCEL_BYTES_MIXED : PARCEL_BYTES_PLAIN) * (size_t)ncap;
    CK(cudaMalloc(&nv.base, nbytes));
    for (int k = 0; k < N_ATTR; ++k) {
        const size_t es = c.pv.f32(k) ? 4 : 8;
        CK(cudaMemcpyAsync(reinterpret_cast<char*>(nv.base) + nv.off(k), reinterpret_cast<char*>(c.pv.base) + c.pv.off(k),
                           es * (size_t)c.n, cudaMemcpyDeviceToDevice, c.stream));
    }
    long long* nlabel = nullptr;
    double* ndil = nullptr;
    if (c.label) {
        CK(cudaMalloc(&nlabel, sizeof(long long) * (size_t)ncap));
        CK(cudaMalloc(&ndil, sizeof(double) * (size_t)ncap));
        CK(cudaMemsetAsync(nlabel, 0, sizeof(long long) * (size_t)ncap, c.stream));
        CK(cudaMemsetAsync(ndil, 0, sizeof(double) * (size_t)ncap, c.stream));
        CK(cudaMemcpyAsync(nlabel, c.label, sizeof(long long) * (size_t)c.n, cudaMemcpyDeviceToDevice, c.stream));
        CK(cudaMemcpyAsync(ndil, c.dil, sizeof(double) * (size_t)c.n, cudaMemcpyDeviceToDevice, c.stream));
    }
    int* nrank = nullptr;
    if (c.rank) {
        CK(cudaMalloc(&nrank, sizeof(int) * (size_t)ncap));
        CK(cudaMemcpyAsync(nrank, c.rank, sizeof(int) * (size_t)c.n, cudaMemcpyDeviceToDevice, c.stream));
    }
    CK(cudaStreamSynchronize(c.stream));
    CK(cudaFree(c.pv.base));
    if (c.rank) {
        CK(cudaFree(c.rank));
        c.rank = nrank;
    }
    if (c.label) {
        CK(cudaFree(c.label));
        CK(cudaFree(c.dil));
        c.label = nlabel;
        c.dil = ndil;
    }
    c.pv = nv;
    c.cap = ncap;
    if (c.pv_alt) {
        CK(cudaFree(c.pv_alt));
        c.pv_alt = nullptr;
        CK(cudaMalloc(&c.pv_alt, nbytes));
    }
    CK(cudaFree(c.stage_partials));
    c.stage_partials = nullptr;
    CK(cudaMalloc(&c.stage_partials, sizeof(double) * 16 * (size_t)stage_grid_max(c.P, c.cap)));
}

// The sort and merge scratch for the current capacity, so that no step
// allocates them mid-step.  A regrowth frees the old scratch in stream order,
// after the kernels already queued that read it.
void grow_scratch_for_capacity(Ctx& c) {
    if (c.box_start) c.get_scratch(sort_scratch_bytes(c.cap));
    c.get_scratch2(merge_scratch_bytes(c.cap));
}

int smem_optin() {
    static std::atomic<int> cache[64];   // per device, 0 = not queried yet
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) dev = 63;
    int v = cache[dev].load();
    if (v == 0) {
        CK(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        cache[dev].store(v);
    }
    return v;
}

void prof_begin(Ctx& c, const char* name) {
    if (c.prof.target.empty() || c.prof.target != name) return;
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    CK(cudaEventRecord(e, c.stream));
    c.prof.ev.push_back(e);
}

void prof_end(Ctx& c, const char* name) {
    if (c.prof.target.empty() || c.prof.target != name) return;
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    CK(cudaEventRecord(e, c.stream));
    c.prof.ev.push_back(e);
    c.prof.launches += 1;
}

static void prof_resolve(Ctx& c) {
    CK(cudaStreamSynchronize(c.stream));
    for (size_t k = 0; k + 1 < c.prof.ev.size(); k += 2) {
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, c.prof.ev[k], c.prof.ev[k + 1]));
        c.prof.ms += ms;
    }
    for (auto e : c.prof.ev) cudaEventDestroy(e);
    c.prof.ev.clear();
}

void* Ctx::get_scratch(size_t bytes) {
    if (bytes > scratch_bytes) {
        if (scratch) CK(cudaFreeAsync(scratch, stream));
        size_t nb = std::max(bytes, scratch_bytes + scratch_bytes / 2);
        CK(cudaMallocAsync(&scratch, nb, stream));
        scratch_bytes = nb;
    }
    return scratch;
}

void* Ctx::get_scratch2(size_t bytes) {
    if (bytes > scratch2_bytes) {
        if (scratch2) CK(cudaFreeAsync(scratch2, stream));
        size_t nb = std::max(bytes, scratch2_bytes + scratch2_bytes / 2);
        CK(cudaMallocAsync(&scratch2, nb, stream));
        scratch2_bytes = nb;
    }
    return scratch2;
}

// Reads the device error word once and turns it into the reference's abort
// messages (mpi_exit_on_error call sites).
void check_device_error(Ctx& c) {
    unsigned e = 0;
    CK(cudaMemcpyAsync(&e, &c.dsc->err, sizeof(unsigned), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if (!e) return;
    CK(cudaMemsetAsync(&c.dsc->err, 0, sizeof(unsigned), c.stream));
    if (e & ERRB_B33) throw CudaError(EPIC_ERR_NUMERICAL, "in parcel_ellipsoid::get_B33: Division by small number!");
    if (e & ERRB_NO_NEIGHBOUR) throw CudaError(EPIC_ERR_NUMERICAL, "Merge error: no near enough neighbour found.");
    if (e & ERRB_TREE) throw CudaError(EPIC_ERR_NUMERICAL, "in parcel_nearest::resolve_tree: First stage error");
    if (e & ERRB_CELL) throw CudaError(EPIC_ERR_NUMERICAL, "in nearest_parcel_to_local_cell_index: Parcel not in local domain.");
    if (e & ERRB_DT) throw CudaError(EPIC_ERR_NUMERICAL, "Time step <= 0!");
    if (e & ERRB_ZRANGE) throw CudaError(EPIC_ERR_NUMERICAL, "interpolation point outside the vertical halo");
    if (e & ERRB_NONFINITE) throw CudaError(EPIC_ERR_NUMERICAL, "par2grid: non-finite parcel attribute");
    if (e & (1u << 30)) throw CudaError(EPIC_ERR_PARCEL_COUNT, "par2grid: Wrong total number of parcels!");
    throw CudaError(EPIC_ERR_NUMERICAL, "device error word " + std::to_string(e));
}

}  // namespace epic

// ---------------------------------------------------------------------------
// layout conversion kernels: Fortran (ncomp, n) <-> structure of arrays
__global__ void k_deinterleave(const double* src, int ncomp, long long n, PView pv, int a0) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * ncomp;
         i += (long long)gridDim.x * blockDim.x) {
        long long p = i / ncomp;
        int k = (int)(i - p * ncomp);
        pv.set(a0 + k, p, src[i]);
    }
}
__global__ void k_interleave(double* dst, int ncomp, long long n, PView pv, int a0) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * ncomp;
         i += (long long)gridDim.x * blockDim.x) {
        long long p = i / ncomp;
        int k = (int)(i - p * ncomp);
        dst[i] = pv.get(a0 + k, p);
    }
}
// Container order of the box-ordered store (Ctx::rank).
__global__ void k_rank_iota(int* rank, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        rank[i] = (int)i;
}
__global__ void k_rank_inverse(const int* rank, long long n, int* ord) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        ord[rank[i]] = (int)i;
}
// dst[r * ncomp + k] = attribute a0 + k of the parcel with container index r
__global__ void k_interleave_ord(double* dst, int ncomp, long long n, PView pv, int a0, const int* ord) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * ncomp;
         i += (long long)gridDim.x * blockDim.x) {
        long long r = i / ncomp;
        int k = (int)(i - r * ncomp);
        dst[i] = pv.get(a0 + k, ord[r]);
    }
}
__global__ void k_deinterleave_ord(const double* src, int ncomp, long long n, PView pv, int a0, const int* ord) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * ncomp;
         i += (long long)gridDim.x * blockDim.x) {
        long long r = i / ncomp;
        int k = (int)(i - r * ncomp);
        pv.set(a0 + k, ord[r], src[i]);
    }
}
template <class T>
__global__ void k_gather_ord(T* dst, const T* src, long long n, const int* ord) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[ord[i]];
}
template <class T>
__global__ void k_scatter_ord(T* dst, const T* src, long long n, const int* ord) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[ord[i]] = src[i];
}
__global__ void k_int_to_double(const int* a, double* b, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

static int cgrid(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 16)); }

namespace epic {
void reset_rank(Ctx& c) {
    if (!c.rank || c.n == 0) return;
    k_rank_iota<<<cgrid(c.n), 256, 0, c.stream>>>(c.rank, c.n);
    CKL();
}
void container_order(Ctx& c, int* ord) {
    if (!c.rank || c.n == 0) return;
    k_rank_inverse<<<cgrid(c.n), 256, 0, c.stream>>>(c.rank, c.n, ord);
    CKL();
}
}  // namespace epic

// Container order for the ABI's parcel arrays: the slot of each container
// index in the sort scratch, or null when slots are container indices.
static const int* abi_order(Ctx& c) {
    if (!c.rank || c.n == 0) return nullptr;
    int* ord = reinterpret_cast<int*>(c.get_scratch(sizeof(int) * (size_t)c.n));
    container_order(c, ord);
    return ord;
}

static void upload_attr(Ctx& c, const double* h, int ncomp, int a0) {
    long long n = c.n;
    if (n == 0) return;
    double* tmp = reinterpret_cast<double*>(c.get_scratch2(sizeof(double) * ncomp * n));
    CK(cudaMemcpyAsync(tmp, h, sizeof(double) * ncomp * n, cudaMemcpyHostToDevice, c.stream));
    k_deinterleave<<<cgrid(n * ncomp), 256, 0, c.stream>>>(tmp, ncomp, n, c.pv, a0);
    CKL();
}

// An attribute of the parcels in container order into the box-ordered store.
static void upload_attr_ord(Ctx& c, const double* h, int ncomp, int a0, const int* ord) {
    if (!ord) return upload_attr(c, h, ncomp, a0);
    long long n = c.n;
    if (n == 0) return;
    double* tmp = reinterpret_cast<double*>(c.get_scratch2(sizeof(double) * ncomp * n));
    CK(cudaMemcpyAsync(tmp, h, sizeof(double) * ncomp * n, cudaMemcpyHostToDevice, c.stream));
    k_deinterleave_ord<<<cgrid(n * ncomp), 256, 0, c.stream>>>(tmp, ncomp, n, c.pv, a0, ord);
    CKL();
}

// An attribute of every parcel, in container order (ord: slot of each
// container index, null when the slots are in container order).
static void download_attr(Ctx& c, double* h, int ncomp, int a0, const int* ord = nullptr) {
    long long n = c.n;
    if (n == 0 || !h) return;
    double* tmp = reinterpret_cast<double*>(c.get_scratch2(sizeof(double) * ncomp * n));
    if (ord) k_interleave_ord<<<cgrid(n * ncomp), 256, 0, c.stream>>>(tmp, ncomp, n, c.pv, a0, ord);
    else k_interleave<<<cgrid(n * ncomp), 256, 0, c.stream>>>(tmp, ncomp, n, c.pv, a0);
    CKL();
    CK(cudaMemcpyAsync(h, tmp, sizeof(double) * ncomp * n, cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
}

// parameters.f90:93-165, physics.f90:170-185
static void setup_params(Ctx& c) {
    const epic_cfg& g = c.cfg;
    Params& P = c.P;
    std::memset(&P, 0, sizeof(P));
    P.nx = g.nx; P.ny = g.ny; P.nz = g.nz;
    P.nzh = g.nz + 3;
    P.fsz = (long long)g.nx * g.ny * P.nzh;
    int nn[3] = {g.nx, g.ny, g.nz};
    for (int k = 0; k < 3; ++k) {
        P.lower[k] = g.lower[k];
        P.extent[k] = g.extent[k];
        P.upper[k] = P.lower[k] + P.extent[k];
        P.extenti[k] = 1.0 / P.extent[k];
        P.dx[k] = P.extent[k] / (double)nn[k];
        P.dxi[k] = 1.0 / P.dx[k];
        P.center[k] = 0.5 * (P.lower[k] + P.upper[k]);
        P.hli[k] = 1.0 / (P.extent[k] / 2.0);
    }
    P.halo_lower[0] = P.lower[0] - P.dx[0];
    P.halo_lower[1] = P.lower[1] - P.dx[1];
    P.vcell = P.dx[0] * P.dx[1] * P.dx[2];
    P.vcelli = 1.0 / P.vcell;
    P.vdomaini = 1.0 / (P.extent[0] * P.extent[1] * P.extent[2]);
    P.vmin = P.vcell / g.min_vratio;
    double amax = std::pow(0.75 * (1.0 / M_PI), 1.0 / 3.0) * std::min(P.dx[0], std::min(P.dx[1], P.dx[2]));
    P.amax2 = amax * amax;
    P.lambda_max = g.lambda_max;
    P.glat = g.gravity * g.L_v / (g.c_p * g.theta_0);
    P.lambda_c = 1.0 / g.height_c;
    P.q_0 = g.q_0;
    if (g.l_planetary_vorticity) {
        double lat = g.lat_degrees * (M_PI / 180.0);
        P.f_cor[1] = 2.0 * g.ang_vel * std::cos(lat);
        P.f_cor[2] = 2.0 * g.ang_vel * std::sin(lat);
    }
    P.zeta_zero[0] = g.bndry_zeta_zero[0] != 0;
    P.zeta_zero[1] = g.bndry_zeta_zero[1] != 0;
    P.dzi = P.dxi[2];
    P.hdzi = 0.5 * P.dxi[2];
    P.ap = P.dxi[2] * P.dxi[2];
    // ls_rk.f90:32-54
    if (g.rk_order == 4) {
        const double ca[5] = {-567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                              -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0, 0.0};
        const double cb[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                              1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                              2277821191437.0 / 14882151754819.0};
        std::memcpy(c.ca, ca, sizeof(ca));
        std::memcpy(c.cb, cb, sizeof(cb));
        c.n_stages = 5;
    } else if (g.rk_order == 3) {
        const double ca[3] = {-5.0 / 9.0, -153.0 / 128.0, 0.0};
        const double cb[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
        std::memcpy(c.ca, ca, sizeof(ca));
        std::memcpy(c.cb, cb, sizeof(cb));
        c.n_stages = 3;
    } else {
        throw CudaError(EPIC_ERR_CONFIG, "Only third and fourth order RK supported.");
    }
}

static void free_ctx(Ctx& c) {
    if (c.stream) cudaStreamSynchronize(c.stream);
    for (auto e : c.prof.ev) cudaEventDestroy(e);
    c.prof.ev.clear();
    spectral_free(c);
    void* ptrs[] = {c.pv.base, c.pv_alt, c.fields, c.nparg, c.nsparg, c.work, c.dsc, c.partials, c.stage_partials,
                    c.dvor_bar, c.box_start, c.gpack, c.binc, c.label, c.dil, c.rank, c.pairs_dev};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c.scratch) cudaFree(c.scratch);
    if (c.scratch2) cudaFree(c.scratch2);
    if (c.hsc) cudaFreeHost(c.hsc);
    if (c.stream) cudaStreamDestroy(c.stream);
    c.stream = nullptr;
}

#define API_BEGIN                                   \
    if (!ctx) return EPIC_ERR_ARG;                  \
    try {
#define API_END                                     \
    } catch (const CudaError& e) {                  \
        ctx->c.err = e.what();                      \
        return e.code;                              \
    } catch (const std::exception& e) {             \
        ctx->c.err = e.what();                      \
        return EPIC_ERR_STATE;                      \
    }                                               \
    return EPIC_OK;

#define NEED_PARCELS                                                           \
    if (!ctx->c.has_parcels) throw CudaError(EPIC_ERR_STATE, "no parcels set (call epic_gpu_set_parcels first)");

extern "C" {

int epic_gpu_default_config(epic_cfg* g) {
    if (!g) return EPIC_ERR_ARG;
    std::memset(g, 0, sizeof(*g));
    g->size_factor = 1.0; g->grow_factor = 1.2; g->shrink_factor = 0.8; g->n_per_cell = 8;
    g->lambda_max = 4.0; g->min_vratio = 20.0; g->correction_iters = 2; g->gradient_pref = 1.8;
    g->max_compression = 0.5; g->t_initial = 0.0; g->t_limit = 0.0; g->alpha = 0.2;
    g->precise_stop = 0; g->use_fixed_dt = 0; g->fixed_dt = 1.0; g->rk_order = 4;
    g->gravity = 9.80616; g->L_v = (double)2.501e6f; g->c_p = 1005.7; g->theta_0 = 288.15;
    g->q_0 = 0.015; g->height_c = 1000.0; g->ang_vel = 0.000072921; g->lat_degrees = 45.0;
    g->l_planetary_vorticity = 0;
    g->capacity = 0; g->precision = EPIC_PRECISION_FP64; g->keep_order = 1;
    g->damping_vorticity_prefactor = 1.0; g->damping_scalars_prefactor = 1.0;
    return EPIC_OK;
}

int epic_gpu_create(const epic_cfg* cfg, epic_ctx** out) {
    if (!cfg || !out) return EPIC_ERR_ARG;
    if (cfg->nx < 4 || cfg->ny < 4 || cfg->nz < 2 || cfg->nx % 2 || cfg->ny % 2) return EPIC_ERR_CONFIG;
    if (cfg->extent[0] <= 0 || cfg->extent[1] <= 0 || cfg->extent[2] <= 0) return EPIC_ERR_CONFIG;
    if (cfg->precision != EPIC_PRECISION_FP64 && cfg->precision != EPIC_PRECISION_MIXED) return EPIC_ERR_CONFIG;
    if (check_damping_flags(*cfg, nullptr) != EPIC_OK) return EPIC_ERR_CONFIG;
    auto* ctx = new epic_ctx();
    Ctx& c = ctx->c;
    c.cfg = *cfg;
    try {
        setup_params(c);
        int dev_count = 0;
        CK(cudaGetDeviceCount(&dev_count));

        CK(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        const Params& P = c.P;
        c.cap = cfg->capacity > 0 ? cfg->capacity
                                  : (long long)(2.0 * (double)P.nx * P.ny * P.nz * std::max(1, cfg->n_per_cell)) + 1024;
        c.cap = (c.cap + 63) & ~63LL;   // every slot starts on a 256-byte boundary
        c.pv.cap = c.cap;
        c.pv.mixed = cfg->precision == EPIC_PRECISION_MIXED;
        CK(cudaMalloc(&c.pv.base, c.store_bytes()));
        CK(cudaMemsetAsync(c.pv.base, 0, c.store_bytes(), c.stream));
        if (cfg->labels) {
            CK(cudaMalloc(&c.label, sizeof(long long) * (size_t)c.cap));
            CK(cudaMalloc(&c.dil, sizeof(double) * (size_t)c.cap));
            CK(cudaMemsetAsync(c.label, 0, sizeof(long long) * (size_t)c.cap, c.stream));
            CK(cudaMemsetAsync(c.dil, 0, sizeof(double) * (size_t)c.cap, c.stream));
        }
        CK(cudaMalloc(&c.fields, sizeof(double) * (size_t)N_FIELDS * P.fsz));
        CK(cudaMemsetAsync(c.fields, 0, sizeof(double) * (size_t)N_FIELDS * P.fsz, c.stream));
        CK(cudaMalloc(&c.nparg, sizeof(int) * P.fsz));
        CK(cudaMalloc(&c.nsparg, sizeof(int) * P.fsz));
        CK(cudaMemsetAsync(c.nparg, 0, sizeof(int) * P.fsz, c.stream));
        CK(cudaMemsetAsync(c.nsparg, 0, sizeof(int) * P.fsz, c.stream));
        c.n_work = N_WORK;
        CK(cudaMalloc(&c.work, sizeof(double) * (size_t)N_WORK * P.fsz));
        CK(cudaMemsetAsync(c.work, 0, sizeof(double) * (size_t)N_WORK * P.fsz, c.stream));
        CK(cudaMalloc(&c.dsc, sizeof(StepScalars)));
        CK(cudaMemsetAsync(c.dsc, 0, sizeof(StepScalars), c.stream));
        CK(cudaMallocHost(&c.hsc, sizeof(StepScalars)));
        CK(cudaMalloc(&c.partials, sizeof(double) * 148 * 8 * 64));
        CK(cudaMalloc(&c.stage_partials, sizeof(double) * 16 * (size_t)stage_grid_max(P, c.cap)));
        // gather records: 16 values per grid point (FP32 in the mixed form)
        CK(cudaMalloc(&c.gpack, (c.pv.mixed ? sizeof(float) : sizeof(double)) * 16 * (size_t)P.fsz));
        if (!cfg->keep_order) {
            CK(cudaMalloc(&c.rank, sizeof(int) * (size_t)c.cap));
            c.nbox = box_count(P);
            CK(cudaMalloc(&c.box_start, sizeof(int) * ((size_t)c.nbox + 1)));
            // a second store lets the sort permute in one pass; without room
            // for it the sort permutes slot by slot through a scratch array
            if (cudaMalloc(&c.pv_alt, c.store_bytes()) != cudaSuccess) {
                cudaGetLastError();
                c.pv_alt = nullptr;
            }
        }
        CK(cudaMalloc(&c.dvor_bar, sizeof(double) * 8));
        CK(cudaMemsetAsync(c.dvor_bar, 0, sizeof(double) * 8, c.stream));
        // scratch for the sort (keep_order == 0) and the merge's binning, sized
        // for the capacity: a step never grows them (a growth maps new device
        // memory mid-step, tens of milliseconds at these sizes)
        if (!cfg->keep_order) c.get_scratch(sort_scratch_bytes(c.cap));
        c.get_scratch2(merge_scratch_bytes(c.cap));
        spectral_init(c);
        CK(cudaStreamSynchronize(c.stream));
    } catch (const CudaError& e) {
        int code = e.code;
        free_ctx(c);
        delete ctx;
        return code;
    } catch (const std::exception&) {
        // host memory for the tables or the scratch bookkeeping: no exception
        // leaves the C ABI
        free_ctx(c);
        delete ctx;
        return EPIC_ERR_CUDA;
    }
    *out = ctx;
    return EPIC_OK;
}

void epic_gpu_destroy(epic_ctx* ctx) {
    if (!ctx) return;
    free_ctx(ctx->c);
    delete ctx;
}

const char* epic_gpu_last_error(const epic_ctx* ctx) { return ctx ? ctx->c.err.c_str() : "null context"; }

int epic_gpu_sync(epic_ctx* ctx) {
    API_BEGIN
    CK(cudaStreamSynchronize(ctx->c.stream));
    check_device_error(ctx->c);
    API_END
}

int epic_gpu_set_parcels(epic_ctx* ctx, int64_t n, const double* pos, const double* vor, const double* B,
                         const double* vol, const double* buoy, const double* hum) {
    API_BEGIN
    Ctx& c = ctx->c;
    if (n < 0 || !pos || !vor || !B || !vol || !buoy) throw CudaError(EPIC_ERR_ARG, "set_parcels: bad arguments");
    if (n > c.cap) throw CudaError(EPIC_ERR_CAPACITY, "set_parcels: more parcels than the device capacity");
    c.n = n;
    c.n_box = 0;
    CK(cudaMemsetAsync(c.pv.base, 0, c.store_bytes(), c.stream));
    if (c.label) {
        CK(cudaMemsetAsync(c.label, 0, sizeof(long long) * (size_t)c.cap, c.stream));
        CK(cudaMemsetAsync(c.dil, 0, sizeof(double) * (size_t)c.cap, c.stream));
    }
    upload_attr(c, pos, 3, A_X);
    upload_attr(c, vor, 3, A_VX);
    upload_attr(c, B, 5, A_B11);
    upload_attr(c, vol, 1, A_VOL);
    upload_attr(c, buoy, 1, A_BUOY);
    if (hum) upload_attr(c, hum, 1, A_HUM);
    reset_rank(c);
    c.has_parcels = true;
    CK(cudaStreamSynchronize(c.stream));
    API_END
}

int epic_gpu_init_state(epic_ctx* ctx, const epic_init_spec* spec) {
    API_BEGIN
    if (!spec) throw CudaError(EPIC_ERR_ARG, "init_state: null spec");
    init_state(ctx->c, *spec);
    CK(cudaStreamSynchronize(ctx->c.stream));
    API_END
}

int epic_gpu_init_from_grids(epic_ctx* ctx, const double* vortg, const double* tbuoyg, const double* humg,
                             int32_t zeta_flags[2]) {
    API_BEGIN
    if (!vortg || !tbuoyg) throw CudaError(EPIC_ERR_ARG, "init_from_grids: null field");
    int f[2];
    init_from_grids(ctx->c, vortg, tbuoyg, humg, f);
    if (zeta_flags) { zeta_flags[0] = f[0]; zeta_flags[1] = f[1]; }
    check_device_error(ctx->c);
    API_END
}

int epic_gpu_autotune(epic_ctx* ctx, epic_tuning* out) {
    API_BEGIN
    autotune(ctx->c, out);
    check_device_error(ctx->c);
    API_END
}

int epic_gpu_get_parcels(epic_ctx* ctx, int64_t cap, int64_t* n, double* pos, double* vor, double* B,
                         double* vol, double* buoy, double* hum) {
    API_BEGIN
    Ctx& c = ctx->c;
    if (!n) throw CudaError(EPIC_ERR_ARG, "get_parcels: null count");
    *n = c.n;
    if (cap < c.n) throw CudaError(EPIC_ERR_ARG, "get_parcels: capacity too small");
    const int* ord = abi_order(c);
    download_attr(c, pos, 3, A_X, ord);
    download_attr(c, vor, 3, A_VX, ord);
    download_attr(c, B, 5, A_B11, ord);
    download_attr(c, vol, 1, A_VOL, ord);
    download_attr(c, buoy, 1, A_BUOY, ord);
    download_attr(c, hum, 1, A_HUM, ord);
    API_END
}

int epic_gpu_get_labels(epic_ctx* ctx, int64_t cap, int64_t* n, int64_t* label, double* dilution) {
    API_BEGIN
    Ctx& c = ctx->c;
    if (!c.label) throw CudaError(EPIC_ERR_STATE, "labels are off (cfg.labels = 0)");
    if (!n) throw CudaError(EPIC_ERR_ARG, "get_labels: null count");
    *n = c.n;
    if (cap < c.n) throw CudaError(EPIC_ERR_ARG, "get_labels: capacity too small");
    const int* ord = abi_order(c);
    const long long* lsrc = c.label;
    const double* dsrc = c.dil;
    if (ord) {
        char* t = reinterpret_cast<char*>(c.get_scratch2(16 * (size_t)c.n + 256));
        long long* tl = reinterpret_cast<long long*>(t);
        double* td = reinterpret_cast<double*>(t + ((8 * (size_t)c.n + 255) & ~(size_t)255));
        k_gather_ord<long long><<<cgrid(c.n), 256, 0, c.stream>>>(tl, c.label, c.n, ord);
        CKL();
        k_gather_ord<double><<<cgrid(c.n), 256, 0, c.stream>>>(td, c.dil, c.n, ord);
        CKL();
        lsrc = tl;
        dsrc = td;
    }
    if (label) CK(cudaMemcpyAsync(label, lsrc, sizeof(long long) * (size_t)c.n, cudaMemcpyDeviceToHost, c.stream));
    if (dilution) CK(cudaMemcpyAsync(dilution, dsrc, sizeof(double) * (size_t)c.n, cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    API_END
}

int epic_gpu_set_labels(epic_ctx* ctx, int64_t n, const int64_t* label, const double* dilution) {
    API_BEGIN
    Ctx& c = ctx->c;
    if (!c.label) throw CudaError(EPIC_ERR_STATE, "labels are off (cfg.labels = 0)");
    if (!label || !dilution || n != c.n) throw CudaError(EPIC_ERR_ARG, "set_labels: bad arguments");
    const int* ord = abi_order(c);
    if (ord && n > 0) {
        char* t = reinterpret_cast<char*>(c.get_scratch2(16 * (size_t)n + 256));
        long long* tl = reinterpret_cast<long long*>(t);
        double* td = reinterpret_cast<double*>(t + ((8 * (size_t)n + 255) & ~(size_t)255));
        CK(cudaMemcpyAsync(tl, label, sizeof(long long) * (size_t)n, cudaMemcpyHostToDevice, c.stream));
        CK(cudaMemcpyAsync(td, dilution, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, c.stream));
        k_scatter_ord<long long><<<cgrid(n), 256, 0, c.stream>>>(c.label, tl, n, ord);
        CKL();
        k_scatter_ord<double><<<cgrid(n), 256, 0, c.stream>>>(c.dil, td, n, ord);
        CKL();
    } else {
        CK(cudaMemcpyAsync(c.label, label, sizeof(long long) * (size_t)n, cudaMemcpyHostToDevice, c.stream));
        CK(cudaMemcpyAsync(c.dil, dilution, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, c.stream));
    }
    CK(cudaStreamSynchronize(c.stream));
    API_END
}

int epic_gpu_num_parcels(epic_ctx* ctx, int64_t* n) {
    API_BEGIN
    if (!n) throw CudaError(EPIC_ERR_ARG, "null");
    *n = ctx->c.n;
    API_END
}

int epic_gpu_get_parcel_rk(epic_ctx* ctx, int64_t cap, int64_t* n, double* dpos, double* dvor, double* strain,
                           double* dB) {
    API_BEGIN
    Ctx& c = ctx->c;
    if (!n) throw CudaError(EPIC_ERR_ARG, "null");
    *n = c.n;
    if (cap < c.n) throw CudaError(EPIC_ERR_ARG, "get_parcel_rk: capacity too small");
    const int* ord = abi_order(c);
    download_attr(c, dpos, 3, A_DX, ord);
    download_attr(c, dvor, 3, A_DVX, ord);
    download_attr(c, strain, 8, A_S0, ord);
    download_attr(c, dB, 5, A_DB0, ord);
    API_END
}

int epic_gpu_set_parcel_rk(epic_ctx* ctx, int64_t n, const double* dpos, const double* dvor, const double* dB) {
    API_BEGIN
    Ctx& c = ctx->c;
    if (n != c.n) throw CudaError(EPIC_ERR_ARG, "set_parcel_rk: count mismatch");
    const int* ord = abi_order(c);
    if (dpos) upload_attr_ord(c, dpos, 3, A_DX, ord);
    if (dvor) upload_attr_ord(c, dvor, 3, A_DVX, ord);
    if (dB) upload_attr_ord(c, dB, 5, A_DB0, ord);
    CK(cudaStreamSynchronize(c.stream));
    API_END
}

int epic_gpu_get_field(epic_ctx* ctx, int id, double* out) {
    API_BEGIN
    Ctx& c = ctx->c;
    if (!out || id < 0 || id >= EPIC_FIELD_COUNT) throw CudaError(EPIC_ERR_ARG, "get_field: bad field id");
    if (id == EPIC_FIELD_NPARG || id == EPIC_FIELD_NSPARG) {
        double* tmp = reinterpret_cast<double*>(c.get_scratch2(sizeof(double) * c.P.fsz));
        k_int_to_double<<<cgrid(c.P.fsz), 256, 0, c.stream>>>(id == EPIC_FIELD_NPARG ? c.nparg : c.nsparg, tmp, c.P.fsz);
        CKL();
        CK(cudaMemcpyAsync(out, tmp, sizeof(double) * c.P.fsz, cudaMemcpyDeviceToHost, c.stream));
    } else {
        CK(cudaMemcpyAsync(out, c.field(id), sizeof(double) * c.P.fsz, cudaMemcpyDeviceToHost, c.stream));
    }
    CK(cudaStreamSynchronize(c.stream));
    API_END
}

int epic_gpu_set_field(epic_ctx* ctx, int id, const double* in) {
    API_BEGIN
    Ctx& c = ctx->c;
    if (!in || id < 0 || id >= EPIC_FIELD_NPARG) throw CudaError(EPIC_ERR_ARG, "set_field: bad field id");
    CK(cudaMemcpyAsync(c.field(id), in, sizeof(double) * c.P.fsz, cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    API_END
}

int epic_gpu_init_correction(epic_ctx* ctx) {
    API_BEGIN NEED_PARCELS init_correction(ctx->c); check_device_error(ctx->c); API_END
}
int epic_gpu_apply_vortcor(epic_ctx* ctx) {
    API_BEGIN NEED_PARCELS apply_vortcor(ctx->c); check_device_error(ctx->c); API_END
}
int epic_gpu_par2grid(epic_ctx* ctx, int reuse) {
    API_BEGIN NEED_PARCELS par2grid(ctx->c, reuse != 0, true); check_device_error(ctx->c); API_END
}
int epic_gpu_vor2vel(epic_ctx* ctx) { API_BEGIN vor2vel(ctx->c); check_device_error(ctx->c); API_END }
int epic_gpu_vorticity_tendency(epic_ctx* ctx) {
    API_BEGIN vorticity_tendency(ctx->c); check_device_error(ctx->c); API_END
}
int epic_gpu_time_step(epic_ctx* ctx, double t, double* dt) {
    API_BEGIN
    Ctx& c = ctx->c;
    if (!dt) throw CudaError(EPIC_ERR_ARG, "null dt");
    CK(cudaMemcpyAsync(&c.dsc->t, &t, sizeof(double), cudaMemcpyHostToDevice, c.stream));
    time_step_reduce(c);
    CK(cudaMemcpyAsync(dt, &c.dsc->dt, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    check_device_error(c);
    API_END
}
int epic_gpu_grid2par(epic_ctx* ctx, int add) {
    API_BEGIN NEED_PARCELS grid2par(ctx->c, add != 0); check_device_error(ctx->c); API_END
}

static double rk_step(Ctx& c, double& t, double* pstats, double* fstats) {
    // ls_rk_step (ls_rk.f90:88-136); each stage's grid2par + update is fused
    // with the following par2grid (stage.cu)
    double tt = t;
    CK(cudaMemcpyAsync(&c.dsc->t, &tt, sizeof(double), cudaMemcpyHostToDevice, c.stream));
    // the first par2grid's scales and the step bounds of the later scatters
    // (surface fluxes change buoyancy and humidity in stage 1: then every
    // scatter bounds its own values)
    p2g_step_bounds(c);
    c.p2g_bound_ready = true;
    par2grid(c, t > c.cfg.t_initial, true, c.n_stages == 1);
    c.p2g_bound_ready = false;
    c.pstep_valid = !c.flux_on;
    prof_begin(c, "vor2vel");
    vor2vel(c);
    prof_end(c, "vor2vel");
    prof_begin(c, "vtend");
    vorticity_tendency(c);
    prof_end(c, "vtend");
    prof_begin(c, "timestep");
    time_step_reduce(c, flux_dt_bound(c));
    prof_end(c, "timestep");
    if (fstats) field_diagnostics(c, fstats);
    for (int s = 1; s <= c.n_stages; ++s) {
        if (s > 1) {
            prof_begin(c, "vor2vel");
            vor2vel(c);
            prof_end(c, "vor2vel");
            prof_begin(c, "vtend");
            vorticity_tendency(c);
            prof_end(c, "vtend");
        }
        fused_stage(c, s, s == 1 && pstats != nullptr);
        if (s < c.n_stages) {
            prof_begin(c, "p2g_tail");
            p2g_tail(c);
            prof_end(c, "p2g_tail");
        }
    }
    if (damping_on(c.cfg)) {
        prof_begin(c, "damping");
        parcel_damp(c);
        prof_end(c, "damping");
    }
    c.pstep_valid = false;
    if (pstats) finish_parcel_diag(c, pstats);
    double dt = 0.0;
    CK(cudaMemcpyAsync(&dt, &c.dsc->dt, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    check_device_error(c);
    t = t + dt;
    return dt;
}

int epic_gpu_rk_step(epic_ctx* ctx, double* t, double* dt) {
    API_BEGIN
    NEED_PARCELS
    if (!t) throw CudaError(EPIC_ERR_ARG, "null t");
    double d = rk_step(ctx->c, *t, nullptr, nullptr);
    if (dt) *dt = d;
    API_END
}

int epic_gpu_parcel_damp(epic_ctx* ctx, double dt) {
    API_BEGIN
    NEED_PARCELS
    Ctx& c = ctx->c;
    std::string msg;
    if (check_damping_flags(c.cfg, &msg) != EPIC_OK) throw CudaError(EPIC_ERR_CONFIG, msg);
    CK(cudaMemcpyAsync(&c.dsc->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, c.stream));
    parcel_damp(c);
    check_device_error(c);
    API_END
}

int epic_gpu_set_bndry_fluxes(epic_ctx* ctx, const double* bflux, const double* hflux) {
    API_BEGIN set_bndry_fluxes(ctx->c, bflux, hflux); API_END
}

int epic_gpu_apply_bndry_fluxes(epic_ctx* ctx, double dt) {
    API_BEGIN
    NEED_PARCELS
    Ctx& c = ctx->c;
    CK(cudaMemcpyAsync(&c.dsc->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, c.stream));
    apply_bndry_fluxes(c);
    check_device_error(c);
    API_END
}

int epic_gpu_merge(epic_ctx* ctx, int64_t* n_merge) {
    API_BEGIN
    NEED_PARCELS
    long long m = parcel_merge(ctx->c);
    check_device_error(ctx->c);
    if (n_merge) *n_merge = m;
    API_END
}

int epic_gpu_get_merge_pairs(epic_ctx* ctx, int64_t cap, int64_t* n, int32_t* isma, int32_t* iclo) {
    API_BEGIN
    Ctx& c = ctx->c;
    if (!n) throw CudaError(EPIC_ERR_ARG, "null");
    *n = (int64_t)c.n_pairs;
    if (cap < *n) throw CudaError(EPIC_ERR_ARG, "get_merge_pairs: capacity too small");
    if (c.n_pairs > 0) {
        std::vector<int> h(2 * (size_t)c.n_pairs);
        CK(cudaMemcpyAsync(h.data(), c.pairs_dev, sizeof(int) * h.size(), cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
        for (long long m = 0; m < c.n_pairs; ++m) {
            if (isma) isma[m] = h[m] + 1;
            if (iclo) iclo[m] = h[c.n_pairs + m] + 1;
        }
    }
    API_END
}

int epic_gpu_split(epic_ctx* ctx, int64_t* n_split) {
    API_BEGIN
    NEED_PARCELS
    long long s = parcel_split(ctx->c);
    check_device_error(ctx->c);
    if (n_split) *n_split = s;
    API_END
}

int epic_gpu_apply_laplace(epic_ctx* ctx, int reuse) {
    API_BEGIN NEED_PARCELS apply_laplace(ctx->c, reuse != 0); check_device_error(ctx->c); API_END
}
int epic_gpu_apply_gradient(epic_ctx* ctx, int reuse) {
    API_BEGIN NEED_PARCELS apply_gradient(ctx->c, reuse != 0); check_device_error(ctx->c); API_END
}
int epic_gpu_vol2grid(epic_ctx* ctx, int reuse) {
    API_BEGIN NEED_PARCELS vol2grid(ctx->c, reuse != 0); check_device_error(ctx->c); API_END
}
int epic_gpu_parcel_diagnostics(epic_ctx* ctx, double* st) {
    API_BEGIN NEED_PARCELS parcel_diagnostics(ctx->c, st); check_device_error(ctx->c); API_END
}
int epic_gpu_field_diagnostics(epic_ctx* ctx, double* st) {
    API_BEGIN field_diagnostics(ctx->c, st); check_device_error(ctx->c); API_END
}

int epic_gpu_step(epic_ctx* ctx, double* t, epic_step_info* info) {
    API_BEGIN
    NEED_PARCELS
    Ctx& c = ctx->c;
    if (!t) throw CudaError(EPIC_ERR_ARG, "null t");
    epic_step_info tmp;
    if (!info) info = &tmp;
    std::memset(info, 0, sizeof(*info));
    long long s0 = c.n_parcel_splits, m0 = c.n_parcel_merges;
    prof_begin(c, "sort");
    if (!c.cfg.keep_order) sort_parcels(c);
    prof_end(c, "sort");
    apply_vortcor(c);
    info->dt = rk_step(c, *t, info->parcel_stats, info->field_stats);
    prof_begin(c, "merge");
    parcel_merge(c, true);
    prof_end(c, "merge");
    prof_begin(c, "split");
    parcel_split(c);
    prof_end(c, "split");
    // the split test bounded the volumes (children halve theirs): the
    // corrections' vol2grid scales
    c.v2g_bound_ready = c.n > 0;
    for (int it = 1; it <= c.cfg.correction_iters; ++it) {
        prof_begin(c, "laplace");
        apply_laplace(c, it > 1);
        prof_end(c, "laplace");
        prof_begin(c, "gradient");
        apply_gradient(c, true);
        prof_end(c, "gradient");
    }
    c.v2g_bound_ready = false;
    check_device_error(c);
    info->t = *t;
    info->n_parcels = c.n;
    info->n_splits = c.n_parcel_splits - s0;
    info->n_merges = c.n_parcel_merges - m0;
    API_END
}

// ---------------------------------------------------------------------------
// Instrumentation (no counterpart in the reference)

int epic_gpu_get_stream(epic_ctx* ctx, void** stream) {
    if (!ctx || !stream) return EPIC_ERR_ARG;
    *stream = (void*)ctx->c.stream;
    return EPIC_OK;
}

int epic_gpu_profile_kernel(epic_ctx* ctx, const char* name) {
    API_BEGIN
    Ctx& c = ctx->c;
    prof_resolve(c);
    c.prof.target = name ? name : "";
    c.prof.ms = 0.0;
    c.prof.launches = 0;
    API_END
}

int epic_gpu_kernel_time(epic_ctx* ctx, double* total_ms, int64_t* launches) {
    API_BEGIN
    Ctx& c = ctx->c;
    prof_resolve(c);
    if (total_ms) *total_ms = c.prof.ms;
    if (launches) *launches = c.prof.launches;
    c.prof.ms = 0.0;
    c.prof.launches = 0;
    API_END
}

int epic_gpu_launch_count(int64_t* n) {
    if (!n) return EPIC_ERR_ARG;
    *n = g_launches.load();
    return EPIC_OK;
}


// ---- parcel and field files (include/epic_nc.h) ----------------------------
static ncio::Box ctx_box(const Ctx& c) {
    ncio::Box b;
    const int32_t n[3] = {c.cfg.nx, c.cfg.ny, c.cfg.nz};
    for (int k = 0; k < 3; ++k) {
        b.ncells[k] = n[k];
        b.origin[k] = c.cfg.lower[k];
        b.extent[k] = c.cfg.extent[k];
    }
    return b;
}

#define NC_TRY(stmt)                                                    \
    try {                                                               \
        stmt;                                                           \
    } catch (const ncio::Error& e) {                                    \
        throw CudaError(EPIC_ERR_IO, e.what());                         \
    }

int epic_gpu_write_parcels_nc(epic_ctx* ctx, const char* path, double t) {
    API_BEGIN
    NEED_PARCELS
    Ctx& c = ctx->c;
    if (!path) throw CudaError(EPIC_ERR_ARG, "write_parcels_nc: null path");
    const int64_t n = c.n;
    std::vector<double> pos(3 * n), vor(3 * n), B(5 * n), vol(n), buoy(n), hum(n);
    int64_t m = 0;
    const int rc = epic_gpu_get_parcels(ctx, n, &m, pos.data(), vor.data(), B.data(), vol.data(), buoy.data(),
                                        hum.data());
    if (rc != EPIC_OK) throw CudaError(rc, c.err);
    std::vector<int64_t> lab;
    std::vector<double> dil;
    if (c.label) {
        lab.resize(n);
        dil.resize(n);
        int64_t ml = 0;
        const int rl = epic_gpu_get_labels(ctx, n, &ml, lab.data(), dil.data());
        if (rl != EPIC_OK) throw CudaError(rl, c.err);
    }
    NC_TRY(ncio::write_parcels(path, ctx_box(c), c.cfg.bndry_zeta_zero, t, n, pos.data(), vor.data(), B.data(),
                               vol.data(), buoy.data(), hum.data(), 0, c.label ? lab.data() : nullptr,
                               c.label ? dil.data() : nullptr))
    API_END
}

int epic_gpu_read_parcels_nc(epic_ctx* ctx, const char* path, double* t) {
    API_BEGIN
    Ctx& c = ctx->c;
    if (!path) throw CudaError(EPIC_ERR_ARG, "read_parcels_nc: null path");
    ncio::Info in;
    NC_TRY(in = ncio::info(path))
    if (in.file_type != "parcels") throw CudaError(EPIC_ERR_IO, std::string(path) + " is not a parcel file");
    NC_TRY(ncio::check_box(in.box, ctx_box(c), path))
    const int64_t n = in.n_parcels;
    if (n > c.cap) throw CudaError(EPIC_ERR_CAPACITY, "read_parcels_nc: more parcels than the device capacity");
    std::vector<double> pos(3 * n), vor(3 * n), B(5 * n), vol(n), buoy(n), hum(n);
    int64_t m = 0;
    NC_TRY(ncio::read_parcels(path, n, &m, pos.data(), vor.data(), B.data(), vol.data(), buoy.data(), hum.data()))
    const int rc = epic_gpu_set_parcels(ctx, n, pos.data(), vor.data(), B.data(), vol.data(), buoy.data(),
                                        hum.data());
    if (rc != EPIC_OK) throw CudaError(rc, c.err);
    if (c.label) {
        // read_chunk resets the labels to the file index and the dilution to 0
        // (parcel_netcdf.f90:709-716)
        std::vector<int64_t> lab(n);
        for (int64_t k = 0; k < n; ++k) lab[k] = k + 1;
        std::vector<double> dil(n, 0.0);
        const int rl = epic_gpu_set_labels(ctx, n, lab.data(), dil.data());
        if (rl != EPIC_OK) throw CudaError(rl, c.err);
    }
    if (in.has_zeta)   // read_zeta_boundary_flag (parameters.f90:220-250)
        for (int b = 0; b < 2; ++b) {
            c.cfg.bndry_zeta_zero[b] = in.zeta[b];
            c.P.zeta_zero[b] = in.zeta[b];
        }
    if (t) *t = in.t;
    API_END
}

int epic_gpu_write_fields_nc(epic_ctx* ctx, const char* path, double t) {
    API_BEGIN
    Ctx& c = ctx->c;
    if (!path) throw CudaError(EPIC_ERR_ARG, "write_fields_nc: null path");
    const size_t fsz = (size_t)c.P.fsz;
    struct Item { int id; const char *name, *long_name, *unit; bool integer; };
    // field_netcdf.f90:460-560 (names, long names and units), in the order of
    // write_netcdf_fields (:214-248)
    const Item items[] = {
        {EPIC_FIELD_VELOG_X, "x_velocity", "x velocity component", "m/s", false},
        {EPIC_FIELD_VELOG_Y, "y_velocity", "y velocity component", "m/s", false},
        {EPIC_FIELD_VELOG_Z, "z_velocity", "z velocity component", "m/s", false},
        {EPIC_FIELD_VTEND_X, "x_vorticity_tendency", "x vorticity tendency", "1/s", false},
        {EPIC_FIELD_VTEND_Y, "y_vorticity_tendency", "y vorticity tendency", "1/s", false},
        {EPIC_FIELD_VTEND_Z, "z_vorticity_tendency", "z vorticity tendency", "1/s", false},
        {EPIC_FIELD_NPARG, "nparg", "number of parcels per cell", "1", true},
        {EPIC_FIELD_NSPARG, "nsparg", "number of small parcels per cell", "1", true},
        {EPIC_FIELD_VORTG_X, "x_vorticity", "x vorticity component", "1/s", false},
        {EPIC_FIELD_VORTG_Y, "y_vorticity", "y vorticity component", "1/s", false},
        {EPIC_FIELD_VORTG_Z, "z_vorticity", "z vorticity component", "1/s", false},
        {EPIC_FIELD_TBUOYG, "buoyancy", "total buoyancy", "m/s^2", false},
        {EPIC_FIELD_DBUOYG, "dry_buoyancy", "dry buoyancy", "m/s^2", false},
        {-1, "liquid_water_content", "liquid-water content", "1", false},
        {EPIC_FIELD_HUMG, "humidity", "specific humidity", "kg/kg", false},
        {EPIC_FIELD_VOLG, "volume", "volume", "m^3", false},
    };
    const int nitems = (int)(sizeof(items) / sizeof(items[0]));
    std::vector<std::vector<double>> data(nitems, std::vector<double>(fsz));
    int it_t = -1, it_d = -1, it_l = -1;
    for (int k = 0; k < nitems; ++k) {
        if (items[k].id == EPIC_FIELD_TBUOYG) it_t = k;
        if (items[k].id == EPIC_FIELD_DBUOYG) it_d = k;
        if (items[k].id < 0) { it_l = k; continue; }
        const int rc = epic_gpu_get_field(ctx, items[k].id, data[k].data());
        if (rc != EPIC_OK) throw CudaError(rc, c.err);
    }
    // glati * (tbuoyg - dbuoyg) (field_netcdf.f90:244)
    const double glati = c.P.glat != 0.0 ? 1.0 / c.P.glat : 0.0;
    for (size_t g = 0; g < fsz; ++g) data[it_l][g] = glati * (data[it_t][g] - data[it_d][g]);
    std::vector<ncio::FieldOut> out;
    for (int k = 0; k < nitems; ++k)
        out.push_back({items[k].name, items[k].long_name, items[k].unit, data[k].data(), items[k].integer});
    NC_TRY(ncio::write_fields(path, ctx_box(c), c.cfg.bndry_zeta_zero, t, out))
    API_END
}

int epic_gpu_init_from_field_file(epic_ctx* ctx, const char* path, int32_t zeta_flags[2]) {
    API_BEGIN
    Ctx& c = ctx->c;
    if (!path) throw CudaError(EPIC_ERR_ARG, "init_from_field_file: null path");
    ncio::Info in;
    NC_TRY(in = ncio::info(path))
    if (in.file_type != "fields") throw CudaError(EPIC_ERR_IO, std::string(path) + " is not a field file");
    const ncio::Box box = ctx_box(c);
    NC_TRY(ncio::check_box(in.box, box, path))
    const size_t fsz = (size_t)c.P.fsz;
    std::vector<double> vort(3 * fsz, 0.0), buoy(fsz, 0.0), hum(fsz, 0.0);
    // read_netcdf_fields(field_file, -1) (field_netcdf.f90:306-389): the last
    // record; datasets the file lacks stay zero
    const char* vn[3] = {"x_vorticity", "y_vorticity", "z_vorticity"};
    for (int k = 0; k < 3; ++k) NC_TRY(ncio::read_field(path, vn[k], -1, box, vort.data() + k * fsz))
    NC_TRY(ncio::read_field(path, "buoyancy", -1, box, buoy.data()))
    NC_TRY(ncio::read_field(path, "humidity", -1, box, hum.data()))
    const int rc = epic_gpu_init_from_grids(ctx, vort.data(), buoy.data(), hum.data(), zeta_flags);
    if (rc != EPIC_OK) throw CudaError(rc, c.err);
    API_END
}

}  // extern "C"
