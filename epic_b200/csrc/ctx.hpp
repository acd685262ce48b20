// Host-side context of one simulation: device state, tables and launchers.
#pragma once
#include "../../include/epic_gpu.h"
#include "common.cuh"

#include <atomic>
#include <limits>
#include <string>
#include <vector>
#include <stdexcept>

namespace epic {

struct CudaError : std::runtime_error {
    int code;
    CudaError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(call)                                                                            \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            throw ::epic::CudaError(EPIC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
// Every kernel launch of the library is followed by CKL(), which also counts it.
extern std::atomic<long long> g_launches;
#define CKL()                                                        \
    do {                                                             \
        ::epic::g_launches.fetch_add(1, std::memory_order_relaxed);  \
        CK(cudaGetLastError());                                      \
    } while (0)

// Mixed-radix plan for the shared-memory Stockham FFT.
struct FFTPlan {
    int n = 0;
    int nfac = 0;
    int fac[16] = {0};
    double2* tw = nullptr;   // device: exp(-2 pi i m / n), m = 0 .. n-1
};

// Spectral tables (inversion_utils.f90:23-48, sta3dfft.f90:17-22).
struct Tables {
    // per (kx, ky): k2l2i, hrkx factor for diffx, hrky factor for diffy
    double* k2l2i = nullptr;       // nx*ny, index kx*ny + ky
    double* fdx = nullptr;         // nx: si * hrkx(dkx) (0 at kx = 0 and Nyquist)
    double* fdy = nullptr;         // ny
    // per column (kx, ky) x z: layout like spectral fields (fidx)
    double* filt = nullptr, *green = nullptr, *phim = nullptr, *phip = nullptr;
    double* thetam = nullptr, *thetap = nullptr, *dthetam = nullptr, *dthetap = nullptr;
    double* etdv = nullptr, *htdv = nullptr;
    double* rkz = nullptr, *rkzi = nullptr, *gamtop = nullptr, *gambot = nullptr;  // nz+1
    // z-transform matrices, (nz+1) x (nz+1) row-major: DST-I (rows/cols 1..nz-1), DCT-I
    double* mdst = nullptr, *mdct = nullptr;
    float* mdst32 = nullptr, *mdct32 = nullptr;   // FP32 copies (mixed form)
    // quarter tables of the symmetric z transforms (even nz): rows k < nz/2
    // grouped by parity, columns j = j0 .. nz/2; qld entries per j
    double* qdst = nullptr, *qdct = nullptr;
    float* qdst32 = nullptr, *qdct32 = nullptr;
    int qld_dst = 0, qld_dct = 0;
};

// Device scalars of one step (kept on the device between kernels).
struct StepScalars {
    double dt;
    double t;
    unsigned long long gmax_bits;   // max |eigenvalue| of the strain (as ordered bits)
    unsigned long long bmax_bits;   // max |grad b|^2
    unsigned err;
    int n_iter_flag;
    long long n;                    // parcel count
    long long count;                // scratch counter
    double vsum, vor[3];            // vorticity correction sums
    // largest |value| of each par2grid field over the parcels (ordered bits
    // of non-negative doubles): vortg x, y, z, dbuoyg, humg, tbuoyg, volg;
    // the fixed-point scales of a scatter and of its tail
    unsigned long long pbound[8];
    // bounds that hold for a whole RK step (volume, buoyancy and humidity do
    // not change between its stages): 0.25 V |b|, 0.25 V |h|,
    // 0.25 V (|b| + glat max(h, 0)) (above |tbuoyg|'s values), 0.25 V
    unsigned long long pstep[4];
    // 0.25 V over the parcels after the split test (vol2grid of the corrections)
    unsigned long long vbound;
};

// CUDA-event timing of every launch of one named kernel on the context stream.
struct KernelTimer {
    std::string target;
    std::vector<cudaEvent_t> ev;   // begin/end pairs
    double ms = 0.0;
    long long launches = 0;
};

struct Ctx {
    KernelTimer prof;
    epic_cfg cfg;
    Params P;
    std::string err;
    cudaStream_t stream = nullptr;
    int n_stages = 5;
    double ca[5], cb[5];
    // parcels
    long long cap = 0;
    long long n = 0;
    PView pv{nullptr, 0, 0};
    // fields: velog 3, vortg 3, vtend 3, velgradg 8, tbuoyg, dbuoyg, humg, volg = 21
    double* fields = nullptr;
    int* nparg = nullptr, *nsparg = nullptr;
    // spectral work arrays (each fsz doubles)
    int n_work = 0;
    double* work = nullptr;
    FFTPlan px, py;
    // horizontal FFT: 0 = 2-D plane kernel where the grid allows it, else the
    // tiled line kernel, else Stockham lines; 1 = tiled, else Stockham; 2 = Stockham;
    // 3 = half-plane cluster kernel (square 64, 128), else as 0
    int fft_path = 0;
    double* gpack = nullptr;     // gathered fields, 16 doubles per grid point
    // log2 of the consecutive parcels a lane group scatters (vol2grid,
    // par2grid, fused stage); the defaults are the tuner's choice on the
    // 128^3 thermal and the 64^3 Beltrami flow (the sums do not depend on it)
    int scatter_lg[3] = {3, 1, 0};
    bool vectors_kernel = true;   // support vectors by their own kernel before a scatter that recomputes them
    int stage_recwin = 0;         // split-form stage kernel gathers from records staged in shared memory
    bool stage_vectors = false;   // split-form stage kernel computes the next par2grid's support vectors
    bool p2g_counted = true;      // the last par2grid scatter counted parcels per cell (nparg, nsparg)
    // mixed form with FP64 spectral work (an accuracy experiment; test toggle)
    bool spectral_fp64 = false;
    // the next scatter's bounds are already in pbound (computed by the
    // kernel that produced its values); else a bound pass runs first
    bool p2g_bound_ready = false;
    // vol2grid may take its volume bound from vbound (set by the step between
    // its split and its corrections)
    bool v2g_bound_ready = false;
    // StepScalars::pstep holds this step's bounds (set by rk_step's first
    // par2grid when the stages change no volume, buoyancy or humidity)
    bool pstep_valid = false;
    // labels (cfg.labels): label and dilution per parcel, capacity cap
    long long* label = nullptr;
    double* dil = nullptr;
    long long merge_calls = 0;    // merge calls that merged at least one parcel (key of the label draws)
    Tables T;
    StepScalars* dsc = nullptr;     // device
    StepScalars* hsc = nullptr;     // pinned host mirror
    double vor_bar[3] = {0, 0, 0};
    double* dvor_bar = nullptr;
    // reduction partials
    double* partials = nullptr;
    double* stage_partials = nullptr;   // per-CTA diagnostics of the fused stage kernel
    const double* diag_buf = nullptr;   // partials read by finish_parcel_diag
    int n_partials = 0;
    // second parcel store for the box reordering (keep_order == 0)
    double* pv_alt = nullptr;
    // keep_order == 0: rank[i] is the index the parcel in slot i has in the
    // reference's container (parcels%position(:, rank + 1)).  The box sort
    // moves it with the parcel; merge (nearest-search order, merge index m,
    // parcel_delete's hole filling) and split (child indices) follow it, so the
    // box-ordered store takes the reference's decisions, and the ABI returns
    // parcels in container order.  Null when keep_order == 1 (slot = index).
    int* rank = nullptr;
    // box ranges of the sorted store: parcels [box_start[b], box_start[b + 1])
    // of [0, n_box) lie in box b at the last sort
    int* box_start = nullptr;
    int nbox = 0;
    long long n_box = 0;
    // merge / split scratch
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    void* scratch2 = nullptr;
    size_t scratch2_bytes = 0;
    // pairs of the last merge (isma then iclo, container indices, m order),
    // kept on the device and copied when the ABI asks for them
    int* pairs_dev = nullptr;
    long long pairs_cap = 0, n_pairs = 0;
    long long n_parcel_splits = 0, n_parcel_merges = 0, n_big_close = 0;
    bool has_parcels = false;
    // surface fluxes (bndry_fluxes.f90:25-36): binc, hinc are (ny, nx), y
    // fastest, scaled by 2 / dz; hinc = binc + nx * ny
    double* binc = nullptr, *hinc = nullptr;
    bool flux_on = false;
    double flux_dt = 0.0;   // alpha (dz / max|binc|)^(1/3)
    double zdepth = 0.0;

    size_t store_bytes() const {
        return (size_t)(pv.mixed ? PARCEL_BYTES_MIXED : PARCEL_BYTES_PLAIN) * (size_t)cap;
    }
    double* field(int id) const { return fields + (long long)id * P.fsz; }
    double* velog(int c) const { return field(EPIC_FIELD_VELOG_X + c); }
    double* vortg(int c) const { return field(EPIC_FIELD_VORTG_X + c); }
    double* vtend(int c) const { return field(EPIC_FIELD_VTEND_X + c); }
    double* velgrad(int c) const { return field(EPIC_FIELD_VELGRAD_0 + c); }
    double* tbuoyg() const { return field(EPIC_FIELD_TBUOYG); }
    double* dbuoyg() const { return field(EPIC_FIELD_DBUOYG); }
    double* humg() const { return field(EPIC_FIELD_HUMG); }
    double* volg() const { return field(EPIC_FIELD_VOLG); }
    double* w(int k) const { return work + (long long)k * P.fsz; }
    void* get_scratch(size_t bytes);
    void* get_scratch2(size_t bytes);
};

constexpr int N_FIELDS = 21;
constexpr int N_WORK = 14;

// spectral.cu
void spectral_init(Ctx& c);
void spectral_free(Ctx& c);

void vor2vel(Ctx& c);
void vorticity_tendency(Ctx& c);
void diverge_laplace(Ctx& c, double* phi, double* grad[3]);
// dt_cap bounds the step's dt after the reference's checks (the surface-flux
// bound of ls_rk_step; infinite for get_time_step alone)
void time_step_reduce(Ctx& c, double dt_cap = std::numeric_limits<double>::infinity());
void make_phi(Ctx& c, double* phi);

// parcels.cu
// moist = false skips dbuoyg and humg, which nothing in the step reads before
// the next par2grid overwrites them (the RK stages before the last)
void par2grid(Ctx& c, bool reuse, bool store_vectors, bool moist = true);
void vol2grid(Ctx& c, bool reuse);
void grid2par(Ctx& c, bool add);
void g2p_rk_stage(Ctx& c, int stage, bool with_diag);
void rk_substep1_dBdt(Ctx& c);
void apply_vortcor(Ctx& c);
void init_correction(Ctx& c);
void apply_laplace(Ctx& c, bool reuse);
void apply_gradient(Ctx& c, bool reuse);
void parcel_diagnostics(Ctx& c, double* out);
void field_diagnostics(Ctx& c, double* out);
long long parcel_split(Ctx& c);
void periodic_all(Ctx& c);
void reflective_all(Ctx& c);
void finish_parcel_diag(Ctx& c, double* out);

// stage.cu
void scatter_p2g(Ctx& c, bool reuse, bool store, bool moist = true);
void scatter_v2g(Ctx& c, bool reuse);
void fused_stage(Ctx& c, int stage, bool with_diag);
void sort_parcels(Ctx& c);
int box_count(const Params& P);
long long stage_grid_max(const Params& P, long long cap);
void p2g_tail(Ctx& c);
// fixed-point bits of the par2grid sums (the scale of the tail's conversion)
int p2g_fx_bits(const Ctx& c);
// bounds of the step's first par2grid and of the step (StepScalars::pstep)
void p2g_step_bounds(Ctx& c);

// init.cu
void init_state(Ctx& c, const epic_init_spec& s);
void init_from_grids(Ctx& c, const double* vortg, const double* tbuoyg, const double* humg, int* zeta_flags);

// damping.cu
bool damping_on(const epic_cfg& g);
int check_damping_flags(const epic_cfg& g, std::string* msg);
void parcel_damp(Ctx& c);
void set_bndry_fluxes(Ctx& c, const double* bflux, const double* hflux);
double flux_dt_bound(const Ctx& c);
void apply_bndry_fluxes(Ctx& c);

// tune.cu
void autotune(Ctx& c, epic_tuning* out);
// spectral.cu: a forward horizontal FFT of one field into work arrays (timing probe)
void fft_forward_probe(Ctx& c);
// fftxyp2s, lapinv1, fftxys2p of a device field into out (test hook)
void lapinv_probe(Ctx& c, const double* in, double* out);

// merge.cu
// in_step: inside epic_gpu_step, where only the state attributes (and labels,
// container indices) are live at the merge, so parcel_delete moves those
long long parcel_merge(Ctx& c, bool in_step = false);
// parcel_delete of nm distinct container indices (host array; test hook)
void test_delete(Ctx& c, const int* idx, int nm);
size_t merge_scratch_bytes(long long n);
// stage.cu
size_t sort_scratch_bytes(long long n);

// Largest dynamic shared memory a block may opt in to on the current device.
int smem_optin();
// Let `kernel` use up to the device's opt-in maximum of dynamic shared memory
// and check that a launch's `bytes` fit.  The attribute is process-wide, so
// it is always set to that same maximum: contexts on other threads launching
// the kernel with other sizes never see a smaller limit.
template <typename K>
void allow_smem(K kernel, size_t bytes) {
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, kernel));
    int mx = smem_optin() - (int)fa.sharedSizeBytes;   // minus the kernel's static shared memory
    if ((long long)bytes > mx)
        throw CudaError(EPIC_ERR_CONFIG, "grid too large for the shared-memory tiles of this device");
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
}

// api.cu
// rank[i] = i for the n parcels (a store loaded in container order)
void reset_rank(Ctx& c);
// ord[r] = slot of the parcel with container index r, r < n (null rank: none)
void container_order(Ctx& c, int* ord);
void grow_store(Ctx& c, long long need);
void grow_scratch_for_capacity(Ctx& c);
void prof_begin(Ctx& c, const char* name);
void prof_end(Ctx& c, const char* name);
void check_device_error(Ctx& c);
void sync_scalars(Ctx& c);

}  // namespace epic
