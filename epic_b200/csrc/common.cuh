// Common device helpers for the B200 EPIC parcel step.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#define EPIC_DEV __device__ __forceinline__
#define EPIC_HD __host__ __device__ __forceinline__

namespace epic {

// Parcel attribute slots of the structure-of-arrays store.  Each slot is a
// contiguous array of `cap` doubles (attribute k of parcel i at k*cap + i),
// so every per-parcel kernel reads and writes fully coalesced lines.
enum Attr {
    A_X = 0, A_Y, A_Z,                 // position
    A_VX, A_VY, A_VZ,                  // vorticity
    A_B11, A_B12, A_B13, A_B22, A_B23, // shape matrix
    A_VOL, A_BUOY, A_HUM,              // volume, buoyancy, humidity
    A_DX, A_DY, A_DZ,                  // LS-RK delta_pos
    A_DVX, A_DVY, A_DVZ,               // LS-RK delta_vor
    A_DB0,                             // LS-RK delta_b (5)
    A_S0 = A_DB0 + 5,                  // strain (8)
    A_ETA0 = A_S0 + 8,                 // Veta (3)
    A_TAU0 = A_ETA0 + 3,               // Vtau (3)
    N_ATTR = A_TAU0 + 3                // = 39
};
// attributes a parcel carries between steps (moved by delete / split)
constexpr int N_STATE = A_HUM + 1;     // 14

// Velocity gradient component order (fields.f90:52-60).
enum { I_DUDX = 0, I_DUDY, I_DUDZ, I_DVDX, I_DVDY, I_DVDZ, I_DWDX, I_DWDY };

// Run parameters derived like update_parameters (parameters.f90:93-165).
struct Params {
    int nx, ny, nz, nzh;          // nzh = nz + 3 (z = -1 .. nz+1)
    long long fsz;                // nx * ny * nzh
    double lower[3], upper[3], extent[3], extenti[3], dx[3], dxi[3], center[3], hli[3];
    double halo_lower[2];
    double vcell, vcelli, vdomaini, vmin, amax2, lambda_max;
    double glat, lambda_c, q_0, f_cor[3];
    int zeta_zero[2];
    double dzi, hdzi, ap;         // inversion_utils.f90:107-113
};

// Slots held in FP32 by the mixed-precision form: vorticity, B, buoyancy,
// humidity, delta_vor, delta_b, strain, Veta, Vtau.  Position, volume and
// delta_pos stay FP64 in both forms.
EPIC_HD constexpr bool attr_f32(int k) {
    return (k >= A_VX && k <= A_B23) || k == A_BUOY || k == A_HUM || k >= A_DVX;
}
// Byte offset of slot k in units of `cap` in the mixed form (FP32 slots take
// 4 bytes): the prefix sum of the slot sizes in closed form.
EPIC_HD constexpr long long mixed_slot_off(int k) {
    return k <= 3 ? 8LL * k : k <= 11 ? 24 + 4LL * (k - 3) : k <= 12 ? 64 : k <= 14 ? 64 + 4LL * (k - 12)
         : k <= 17 ? 72 + 8LL * (k - 14) : 96 + 4LL * (k - 17);
}
constexpr bool mixed_slot_off_ok() {
    long long o = 0;
    for (int j = 0; j <= N_ATTR; ++j) {
        if (mixed_slot_off(j) != o) return false;
        if (j < N_ATTR) o += attr_f32(j) ? 4 : 8;
    }
    return true;
}
static_assert(mixed_slot_off_ok(), "mixed slot offsets");
constexpr long long PARCEL_BYTES_PLAIN = 8LL * N_ATTR;              // 312
constexpr long long PARCEL_BYTES_MIXED = mixed_slot_off(N_ATTR);    // 184

// View of the parcel store: slot k of parcel i.  get/set convert between the
// slot's storage type and double; typed pointers (d, f) serve the kernels that
// are written for one form.
struct PView {
    double* base;        // start of the store (bytes addressed through off)
    long long cap;
    int mixed;           // 1: FP32 slots as in attr_f32
    EPIC_HD long long off(int k) const { return (mixed ? mixed_slot_off(k) : 8LL * k) * cap; }
    EPIC_HD bool f32(int k) const { return mixed && attr_f32(k); }
    EPIC_HD double* d(int k) const { return reinterpret_cast<double*>(reinterpret_cast<char*>(base) + off(k)); }
    EPIC_HD float* f(int k) const { return reinterpret_cast<float*>(reinterpret_cast<char*>(base) + off(k)); }
    template <class R>
    EPIC_HD R* ptr(int k) const { return reinterpret_cast<R*>(reinterpret_cast<char*>(base) + off(k)); }
    EPIC_HD double get(int k, long long i) const { return f32(k) ? (double)f(k)[i] : d(k)[i]; }
    EPIC_HD void set(int k, long long i, double v) const {
        if (f32(k)) f(k)[i] = (float)v;
        else d(k)[i] = v;
    }
};

// Field index: z fastest with one halo row below, x slowest.
EPIC_HD long long fidx(const Params& p, int iz, int iy, int ix) {
    return ((long long)ix * p.ny + iy) * p.nzh + (iz + 1);
}
EPIC_HD int wrapi(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// Arithmetic policies.  ExactOps forbids FMA contraction so that decisions
// (split test, nearest-parcel distances) round exactly like the oracle's
// -ffp-contract=off build; FastOps lets the compiler contract.
struct ExactOps {
    using T = double;
    static EPIC_DEV double mul(double a, double b) { return __dmul_rn(a, b); }
    static EPIC_DEV double add(double a, double b) { return __dadd_rn(a, b); }
    static EPIC_DEV double sub(double a, double b) { return __dsub_rn(a, b); }
};
struct FastOps {
    using T = double;
    static EPIC_DEV double mul(double a, double b) { return a * b; }
    static EPIC_DEV double add(double a, double b) { return a + b; }
    static EPIC_DEV double sub(double a, double b) { return a - b; }
};
// FP32 arithmetic of the mixed-precision form.
struct F32Ops {
    using T = float;
    static EPIC_DEV float mul(float a, float b) { return a * b; }
    static EPIC_DEV float add(float a, float b) { return a + b; }
    static EPIC_DEV float sub(float a, float b) { return a - b; }
};

// Error word bits written by kernels (read once per step by the host).
enum ErrBits {
    ERRB_B33 = 1u << 0,           // get_B33 division by small number
    ERRB_ZRANGE = 1u << 1,        // interpolation point outside the vertical halo
    ERRB_NO_NEIGHBOUR = 1u << 2,  // merge: no near enough neighbour
    ERRB_CELL = 1u << 3,          // nearest: parcel not in local domain
    ERRB_TREE = 1u << 4,          // resolve_tree first stage error
    ERRB_DT = 1u << 5,            // time step <= 0
    ERRB_NONFINITE = 1u << 6,     // par2grid: a non-finite parcel value
};

EPIC_DEV void set_err(unsigned* err, unsigned bit) { atomicOr(err, bit); }

// Monotone encoding of a non-negative double for atomicMax on 64-bit ints.
EPIC_DEV void atomic_max_nonneg(unsigned long long* addr, double v) {
    atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

}  // namespace epic
