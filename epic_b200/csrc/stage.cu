// Box-decomposed scatter (par2grid, vol2grid), the LS-RK stage kernel, and
// the box ordering of the parcel store.
//
// Ordering: at the start of a step the parcel store is sorted by box of
// BOXX x BOXY x BOXZ cells (cells z fastest inside a box), and the first
// parcel of every box is recorded.  One CTA takes one box; parcels appended
// later (split children) are handled in tail chunks of SCHUNK parcels.
//
// Scatter (parcel_interpl.f90:160-233): every contribution w * v of a support
// point (trilinear weight w of a corner, value v = attribute x point weight
// 1/4 x volume) is a fixed-point integer q = round(w v s_f) at one scale
// s_f = 2^(b - e_f) per field and launch, 2^e_f above the largest |v| of the
// field over all parcels (a bound computed before the scatter).  Grid sums
// are integer sums, exact and therefore independent of the order of the adds:
// par2grid is bitwise reproducible run to run and for any launch shape.  A box
// CTA adds its parcels' contributions into a shared-memory window (the box's
// grid points and WM more on every side) as three 32-bit limbs with integer
// shared atomics, then adds the window to the 64-bit integer grid sums held in
// the field arrays; points outside the window, and tail chunks whose parcels
// do not fit a window, add to the grid sums directly.  The tail kernels
// (parcels.cu) fold the z halos in integers and convert to FP64.
//
// Stage (ls_rk.f90:142-217 + parcel_interpl.f90:405-470): grid2par at the
// support points (support vectors stored by the preceding scatter, from the
// same B, parcel_ellipsoid.f90:216-247), dB/dt, the update of x, w, B and the
// scaling of the accumulators; it also bounds the next par2grid's values.
#include "parcel_ops.cuh"

#include <cub/cub.cuh>
#include <climits>
#include <cstring>

namespace epic {

constexpr int BOXX = 8, BOXY = 4, BOXZ = 4;   // cells per box
constexpr int BOXC = BOXX * BOXY * BOXZ;
constexpr int SCHUNK = 2048;    // parcels per tail chunk
constexpr int ROUND = 4096;     // parcels per fixed-point round
// Window of a box CTA: the box's grid points and WM more on every side
// (parcels that moved up to a cell out of the box since the sort, plus half
// a cell of support-point reach), 13 x 9 x 9 grid points.
constexpr int WM = 2;
constexpr int WCAP = (BOXX + 1 + 2 * WM) * (BOXY + 1 + 2 * WM) * (BOXZ + 1 + 2 * WM);
// Words per limb plane: at least WCAP, and 11 banks apart (WSTRIDE = 11 mod
// 32), so that two lanes adding different limbs of the same grid point hit
// different banks (see LimbOrder).
constexpr int WSTRIDE = ((WCAP + 31 - 11) / 32) * 32 + 11;
constexpr int NLIMB = 3;
constexpr int SB = 2;           // CTAs per SM the scatter kernels are sized for

// Box ranges of the sorted parcel store.
struct Boxes {
    const int* start;   // nbox + 1 first-parcel offsets
    int nbox;           // 0 when the store is not box ordered
    int nby, nbz;       // boxes along y and z
    long long n_box;    // parcels [0, n_box) belong to the box ranges
};

struct Window {
    int gx0, gy0, gz0;   // window origin (grid point; x, y unwrapped)
    int WX, WY, WZ;      // extents
    int ok;
};

// Parcel range and reference cell of this CTA.
struct Range {
    long long r0, r1;
    int ref[3];
    bool box;            // a box of the sorted store (else a tail chunk)
};

// Cell of a position (get_index, fields.f90:165-172).
EPIC_DEV void cell_of(const Params& P, const double* p, int& ci, int& cj, int& ck) {
    ci = (int)floor((p[0] - P.lower[0]) * P.dxi[0]);
    cj = (int)floor((p[1] - P.lower[1]) * P.dxi[1]);
    ck = (int)floor((p[2] - P.lower[2]) * P.dxi[2]);
}

EPIC_DEV Range cta_range(const Params& P, const PView& pv, const Boxes& B, long long n) {
    Range R;
    int b = blockIdx.x;
    if (b < B.nbox) {
        R.r0 = min((long long)B.start[b], B.n_box);
        R.r1 = min((long long)B.start[b + 1], B.n_box);
        int bz = b % B.nbz, r = b / B.nbz;
        int by = r % B.nby, bx = r / B.nby;
        R.ref[0] = bx * BOXX; R.ref[1] = by * BOXY; R.ref[2] = bz * BOXZ;
        R.box = true;
    } else {
        long long t = b - B.nbox;
        R.r0 = B.n_box + t * SCHUNK;
        R.r1 = min(R.r0 + SCHUNK, n);
        R.ref[0] = R.ref[1] = R.ref[2] = 0;
        if (R.r0 < R.r1) {
            double p[3] = {pv.get(A_X, R.r0), pv.get(A_Y, R.r0), pv.get(A_Z, R.r0)};
            cell_of(P, p, R.ref[0], R.ref[1], R.ref[2]);
            R.ref[0] = wrapi(R.ref[0], P.nx);
            R.ref[1] = wrapi(R.ref[1], P.ny);
        }
        R.box = false;
    }
    return R;
}

// Offset of cell c from the reference cell r, periodic, in [-n/2, n - n/2).
EPIC_DEV int rel_periodic(int c, int r, int n) {
    int d = wrapi(c - r, n);
    return d >= n - n / 2 ? d - n : d;
}

// Shared state of a scatter CTA: the cell bounds of a tail chunk (relative
// to its first parcel), the window and the fixed-point scales.
template <int NF>
struct WinShared {
    int mn[3], mx[3];
    Window W;
    double scale[NF];
};

// Window of a box CTA: fixed, the box's grid points +- WM (z clipped to the
// halo rows -1 .. nz + 1).
EPIC_DEV Window box_window(const Params& P, const Range& R) {
    Window W;
    W.gx0 = R.ref[0] - WM;
    W.gy0 = R.ref[1] - WM;
    W.gz0 = max(R.ref[2] - WM, -1);
    W.WX = BOXX + 1 + 2 * WM;
    W.WY = BOXY + 1 + 2 * WM;
    W.WZ = min(R.ref[2] + BOXZ + WM, P.nz + 1) - W.gz0 + 1;
    W.ok = W.WX <= P.nx && W.WY <= P.ny;   // no grid point twice in one window
    return W;
}

// Cell bounds of a tail chunk (one thread per parcel, then a block reduction
// into ws->mn / mx, which thread 0 cleared); the window covers the chunk's
// cells with one cell below and two above (support points and corners).
template <int NF>
EPIC_DEV void tail_bounds(const Params& P, const Range& R, const PView& pv, WinShared<NF>* ws) {
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
    for (long long i = R.r0 + threadIdx.x; i < R.r1; i += blockDim.x) {
        const double p[3] = {pv.get(A_X, i), pv.get(A_Y, i), pv.get(A_Z, i)};
        int c[3];
        cell_of(P, p, c[0], c[1], c[2]);
        const int d[3] = {rel_periodic(c[0], R.ref[0], P.nx), rel_periodic(c[1], R.ref[1], P.ny), c[2] - R.ref[2]};
#pragma unroll
        for (int k = 0; k < 3; ++k) { mn[k] = min(mn[k], d[k]); mx[k] = max(mx[k], d[k]); }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[k] = min(mn[k], __shfl_xor_sync(0xffffffff, mn[k], o));
            mx[k] = max(mx[k], __shfl_xor_sync(0xffffffff, mx[k], o));
        }
    }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; ++k) { atomicMin(&ws->mn[k], mn[k]); atomicMax(&ws->mx[k], mx[k]); }
}

EPIC_DEV Window tail_window(const Params& P, const Range& R, const int* mn, const int* mx) {
    Window W;
    W.gx0 = R.ref[0] + mn[0] - 1;
    W.gy0 = R.ref[1] + mn[1] - 1;
    W.gz0 = max(R.ref[2] + mn[2] - 1, -1);
    W.WX = mx[0] - mn[0] + 4;
    W.WY = mx[1] - mn[1] + 4;
    W.WZ = min(R.ref[2] + mx[2] + 2, P.nz + 1) - W.gz0 + 1;
    W.ok = mn[0] <= mx[0] && W.WX <= P.nx && W.WY <= P.ny && W.WZ > 0 && (long long)W.WX * W.WY * W.WZ <= WCAP;
    return W;
}

struct Fields7 {
    double* f[7];   // vortg x,y,z, dbuoyg, humg, tbuoyg, volg (64-bit integer sums during the scatter)
    int mask;       // bit f set: field f is accumulated (NF = 7)
};
constexpr int ALL_FIELDS = 0x7f;
constexpr int DRY_FIELDS = 0x67;   // without dbuoyg (3) and humg (4)

// Field set of a scatter kernel: NF = 7 (all, masked by Fields7.mask), 5 (the
// dry set: vorticity, tbuoyg, volg) or 1 (one field, vol2grid).
template <int NF>
EPIC_HD constexpr int field_slot(int f) {
    return NF == 5 ? (f < 3 ? f : f + 2) : f;
}
// Slot of field f's bound in StepScalars::pbound (the 7 par2grid fields;
// vol2grid's volume shares the par2grid volume's slot).
template <int NF>
EPIC_HD constexpr int bound_slot(int f) {
    return NF == 1 ? 6 : field_slot<NF>(f);
}
template <int NF>
EPIC_DEV bool field_on(const Fields7& F, int f) {
    return NF != 7 || ((F.mask >> f) & 1);
}

// Arithmetic of the two forms: R is the type of the FP32-able attributes,
// of the gathered values and of the window sums (double: plain, float: mixed).
template <class R> struct Form {
    static constexpr bool mixed = false;
    using Ops = FastOps;
};
template <> struct Form<float> {
    static constexpr bool mixed = true;
    using Ops = F32Ops;
};

// Slot k of parcel i: FP64 slots (position, volume, delta_pos) and R slots.
template <class R>
EPIC_DEV double& a64(const PView& pv, int k, long long i) {
    return reinterpret_cast<double*>(reinterpret_cast<char*>(pv.base) +
                                     (Form<R>::mixed ? mixed_slot_off(k) : 8LL * k) * pv.cap)[i];
}
template <class R>
EPIC_DEV R& aR(const PView& pv, int k, long long i) {
    return reinterpret_cast<R*>(reinterpret_cast<char*>(pv.base) +
                                (Form<R>::mixed ? mixed_slot_off(k) : 8LL * k) * pv.cap)[i];
}

// Fixed-point bits: |w v s_f| <= 2^(b + 2) (merged weights of up to 4 support
// points).  Plain: b = 46, three window limbs (18 + 18 bits unsigned and a
// signed top), 4 x ROUND contributions per grid point per round within 32
// bits each, 2^15 contributions per grid point within the 64-bit grid sums;
// rounding 2^-47 of the field's largest value.  Mixed: b = 34, two limbs
// (19 bits unsigned and a signed top) for 4 x 2048 contributions per round,
// far below FP32 rounding.
template <class R> constexpr int fx_bits() { return Form<R>::mixed ? 34 : 46; }
template <class R> constexpr int win_words() { return Form<R>::mixed ? 2 : NLIMB; }
template <class R, int NF> constexpr size_t win_bytes() { return sizeof(unsigned) * NF * win_words<R>() * WSTRIDE; }
template <class R> constexpr int round_max() { return Form<R>::mixed ? 2048 : ROUND; }

// Scale of field slot k from its bound (largest |value| as ordered bits).
EPIC_DEV double fx_scale(const unsigned long long* pbound, int k, int bits, unsigned* err) {
    const double m = __longlong_as_double((long long)pbound[k]);
    if (!(m <= 1.0e300)) {   // a non-finite parcel value
        set_err(err, ERRB_NONFINITE);
        return 0.0;
    }
    int e = 0;
    if (m > 0.0) frexp(m, &e);   // m < 2^e
    return ldexp(1.0, bits - e);
}

// Rounding of w * vs (|w vs| <= 2^50) to an integer: r = w vs + 1.5 * 2^52
// rounds once; the low 52 bits of r hold 2^51 + q.
constexpr double FX_MAGIC = 6755399441055744.0;   // 1.5 * 2^52
EPIC_DEV long long fx_round(double wt, double vs) {
    const double r = fma(wt, vs, FX_MAGIC);
    return (__double_as_longlong(r) & 0xfffffffffffffll) - (1ll << 51);
}

// The order in which a lane adds the limbs of a contribution.  The two lanes
// of a lane pair take consecutive parcels, usually of one cell, so at every
// corner they add to the same grid point: the odd lane adds its limbs in
// rotated order, and with the limb planes 11 banks apart the pair's atomics
// of one instruction hit different banks instead of the same word.  The
// sums do not depend on the order.
struct LimbOrder {
    int p0, p1, p2;   // plane offsets (words) of the 1st, 2nd and 3rd add
    bool rot;
    EPIC_DEV explicit LimbOrder(int nlimb) {
        rot = (threadIdx.x & 1) != 0;
        if (nlimb == 3) {
            p0 = rot ? WSTRIDE : 0;
            p1 = rot ? 2 * WSTRIDE : WSTRIDE;
            p2 = rot ? 0 : 2 * WSTRIDE;
        } else {
            p0 = rot ? WSTRIDE : 0;
            p1 = rot ? 0 : WSTRIDE;
            p2 = 0;
        }
    }
};

// q = ((m >> 36) - 2^15) * 2^36 + ((m >> 18) & 0x3ffff) * 2^18 + (m & 0x3ffff), m = 2^51 + q
EPIC_DEV void fx_add(unsigned* acc, int w, double wt, double vs, const LimbOrder& o) {
    double r = fma(wt, vs, FX_MAGIC);
    unsigned lo = (unsigned)__double2loint(r), hi = (unsigned)__double2hiint(r);
    const unsigned l0 = lo & 0x3ffffu;
    const unsigned l1 = (lo >> 18) | ((hi & 0xfu) << 14);
    const unsigned l2 = ((hi & 0xfffffu) >> 4) - 32768u;
    atomicAdd(&acc[o.p0 + w], o.rot ? l1 : l0);
    atomicAdd(&acc[o.p1 + w], o.rot ? l2 : l1);
    atomicAdd(&acc[o.p2 + w], o.rot ? l0 : l2);
}
EPIC_DEV long long fx_sum(const unsigned* acc, int w) {
    return (long long)(int)acc[2 * WSTRIDE + w] * (1ll << 36) + (long long)acc[WSTRIDE + w] * (1ll << 18) +
           (long long)acc[w];
}

// Two-limb variant: q = h * 2^19 + l, l = q mod 2^19, h = floor(q / 2^19).
EPIC_DEV void fx2_add(unsigned* acc, int w, double wt, double vs, const LimbOrder& o) {
    double r = fma(wt, vs, FX_MAGIC);
    long long m = __double_as_longlong(r) & 0xfffffffffffffll;   // 2^51 + q
    const unsigned l0 = (unsigned)(m & 0x7ffff);
    const unsigned l1 = (unsigned)((m >> 19) - (1ll << 32));
    atomicAdd(&acc[o.p0 + w], o.rot ? l1 : l0);
    atomicAdd(&acc[o.p1 + w], o.rot ? l0 : l1);
}
EPIC_DEV long long fx2_sum(const unsigned* acc, int w) {
    return (long long)(int)acc[WSTRIDE + w] * (1ll << 19) + (long long)acc[w];
}

// A contribution straight into the 64-bit grid sum of field f at point g.
EPIC_DEV void fx_global(double* f, long long g, double wt, double vs) {
    const long long q = fx_round(wt, vs);
    if (q != 0) atomicAdd(reinterpret_cast<unsigned long long*>(f) + g, (unsigned long long)q);
}

EPIC_DEV int wrap_to(int l, int n) { return ((unsigned)l < (unsigned)n) ? l : wrapi(l, n); }

// Support points of one parcel that fall into the same cell as the point
// before them share their 8 corners: their trilinear weights are summed and
// the corners visited once (sum_p w_p f = (sum_p w_p) f; only the rounding
// order differs from visiting each point).
EPIC_DEV bool same_cell(const Tri& a, const Tri& b) { return a.is == b.is && a.js == b.js && a.ks == b.ks; }
// Whether point p lies in t's cell, and if so adds its trilinear weights to
// t's (the arithmetic of trilinear() followed by add_weights(), without a
// second Tri held in registers).
EPIC_DEV bool merge_into(const Params& P, const double* p, Tri& t) {
    const double x = (p[0] - P.lower[0]) * P.dxi[0];
    const double y = (p[1] - P.lower[1]) * P.dxi[1];
    const double z = (p[2] - P.lower[2]) * P.dxi[2];
    const int is = (int)floor(x), js = (int)floor(y), ks = (int)floor(z);
    if (is != t.is || js != t.js || ks != t.ks) return false;
    const double px = x - (double)is, pxc = 1.0 - px;
    const double py = y - (double)js, pyc = 1.0 - py;
    const double pz = z - (double)ks, pzc = 1.0 - pz;
    const double w00 = pyc * pxc, w10 = pyc * px, w01 = py * pxc, w11 = py * px;
    t.w[0][0][0] += pzc * w00; t.w[0][0][1] += pzc * w10; t.w[0][1][0] += pzc * w01; t.w[0][1][1] += pzc * w11;
    t.w[1][0][0] += pz * w00;  t.w[1][0][1] += pz * w10;  t.w[1][1][0] += pz * w01;  t.w[1][1][1] += pz * w11;
    return true;
}
EPIC_DEV void add_weights(Tri& a, const Tri& b) {
#pragma unroll
    for (int kk = 0; kk < 2; ++kk)
#pragma unroll
        for (int jj = 0; jj < 2; ++jj)
#pragma unroll
            for (int ii = 0; ii < 2; ++ii) a.w[kk][jj][ii] += b.w[kk][jj][ii];
}
EPIC_DEV void support_point(const double* pos, const double* eta, const double* tau, int p, double* pt) {
    const double cp = support_cos(p), sp = support_sin(p);
#pragma unroll
    for (int k = 0; k < 3; ++k) pt[k] = pos[k] + eta[k] * cp + tau[k] * sp;
}
// The points lie on an ellipse in the order 0..3; starting the merge at a
// point whose predecessor (cyclically) is in another cell also merges a run
// that wraps from point 3 to point 0.
EPIC_DEV int merge_start(const Params& P, const double* pos, const double* eta, const double* tau) {
    int c[4][3];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        double pt[3];
        support_point(pos, eta, tau, p, pt);
#pragma unroll
        for (int k = 0; k < 3; ++k) c[p][k] = (int)floor((pt[k] - P.lower[k]) * P.dxi[k]);
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int q = (p + 3) & 3;
        if (c[p][0] != c[q][0] || c[p][1] != c[q][1] || c[p][2] != c[q][2]) return p;
    }
    return 0;
}

// Scatter one support point (or the merged points of one parcel in one cell):
// vs[f] = value x volume x point weight x s_f.
template <int NF, class R>
EPIC_DEV void scatter_tri(const Params& P, const Window& W, unsigned* acc, const Fields7& F, const Tri& t,
                          const double* vs, const LimbOrder& lo, unsigned* err) {
    if (t.ks < -1 || t.ks > P.nz) { set_err(err, ERRB_ZRANGE); return; }
    int lx = wrap_to(t.is - W.gx0, P.nx), ly = wrap_to(t.js - W.gy0, P.ny), lz = t.ks - W.gz0;
    if (W.ok && lx + 1 < W.WX && ly + 1 < W.WY && lz >= 0 && lz + 1 < W.WZ) {
        int base = (lx * W.WY + ly) * W.WZ + lz;
#pragma unroll
        for (int ii = 0; ii < 2; ++ii)
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    int w = base + (ii * W.WY + jj) * W.WZ + kk;
                    if constexpr (Form<R>::mixed) {
                        const double wt = (double)(float)t.w[kk][jj][ii];
#pragma unroll
                        for (int f = 0; f < NF; ++f)
                            if (field_on<NF>(F, f)) fx2_add(acc + f * 2 * WSTRIDE, w, wt, vs[f], lo);
                    } else {
                        const double wt = t.w[kk][jj][ii];
#pragma unroll
                        for (int f = 0; f < NF; ++f)
                            if (field_on<NF>(F, f)) fx_add(acc + f * NLIMB * WSTRIDE, w, wt, vs[f], lo);
                    }
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
                    const double wt = Form<R>::mixed ? (double)(float)t.w[kk][jj][ii] : t.w[kk][jj][ii];
#pragma unroll
                    for (int f = 0; f < NF; ++f)
                        if (field_on<NF>(F, f)) fx_global(F.f[field_slot<NF>(f)], g, wt, vs[f]);
                }
    }
}

template <int NF, class R>
EPIC_DEV void win_zero(unsigned* acc, const Window& W) {
    if (!W.ok) return;
    int n = W.WX * W.WY * W.WZ;
    for (int f = 0; f < NF * win_words<R>(); ++f)
        for (int w = threadIdx.x; w < n; w += blockDim.x) acc[f * WSTRIDE + w] = 0u;
}

// The window's integer sums into the 64-bit grid sums.
template <int NF, class R>
EPIC_DEV void win_flush(const Params& P, const unsigned* acc, const Window& W, const Fields7& F) {
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
            if (!field_on<NF>(F, f)) continue;
            long long q;
            if constexpr (Form<R>::mixed) q = fx2_sum(acc + f * 2 * WSTRIDE, w);
            else q = fx_sum(acc + f * NLIMB * WSTRIDE, w);
            if (q != 0) atomicAdd(reinterpret_cast<unsigned long long*>(F.f[field_slot<NF>(f)]) + g,
                                  (unsigned long long)q);
        }
    }
}

// Contributions of one parcel to the par2grid fields (parcel_interpl.f90:177-230):
// value * point weight (1/4) * volume.
template <class R>
EPIC_DEV void p2g_values(const Params& P, const R* vor, double z, double vol, R buoy, R hum, R* vp) {
    R q_c = hum - (R)P.q_0 * exp((R)(P.lambda_c * (P.lower[2] - z)));
    q_c = fmax((R)0, q_c);
    const R pw = (R)(0.25 * vol);
    vp[0] = pw * vor[0];
    vp[1] = pw * vor[1];
    vp[2] = pw * vor[2];
    vp[3] = pw * buoy;
    vp[4] = pw * hum;
    vp[5] = pw * (buoy + (R)P.glat * q_c);
    vp[6] = pw;
}

template <int NF, class R>
EPIC_DEV void load_values(const Params& P, const PView& pv, long long i, double z, R* vp) {
    if (NF == 1) {
        vp[0] = (R)(0.25 * a64<R>(pv, A_VOL, i));
    } else {
        R vor[3] = {aR<R>(pv, A_VX, i), aR<R>(pv, A_VY, i), aR<R>(pv, A_VZ, i)};
        R v7[7];
        p2g_values<R>(P, vor, z, a64<R>(pv, A_VOL, i), aR<R>(pv, A_BUOY, i), aR<R>(pv, A_HUM, i), v7);
#pragma unroll
        for (int f = 0; f < NF; ++f) vp[f] = v7[field_slot<NF>(f)];
    }
}

// Largest |value| of each scattered field over all parcels (as ordered bits of
// a non-negative double; a NaN counts as +inf), into pbound, which the caller
// cleared: the fixed-point scales of the scatter that follows.  STEP also
// records the step bounds (StepScalars::pstep) for the later stages' scatters.
EPIC_DEV unsigned long long max_bits(double a) { return (unsigned long long)__double_as_longlong(a); }
EPIC_DEV double nan_inf(double a) { return isnan(a) ? INFINITY : a; }
EPIC_DEV double keep_max(double m, double a) { return (a > m || a != a) ? a : m; }
// warp maximum, then one atomic per warp
EPIC_DEV void warp_max_to(unsigned long long* dst, double v) {
    v = nan_inf(v);
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffff, v, o));
    if ((threadIdx.x & 31) == 0 && v > 0.0) atomicMax(dst, max_bits(v));
}
template <int NF, class R, bool STEP>
__global__ void __launch_bounds__(PB) k_p2g_bounds(Params P, PView pv, long long n, unsigned long long* pbound,
                                                   unsigned long long* pstep) {
    double mx[NF], ms[4];
#pragma unroll
    for (int f = 0; f < NF; ++f) mx[f] = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) ms[k] = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        R vp[NF];
        load_values<NF, R>(P, pv, i, a64<R>(pv, A_Z, i), vp);
#pragma unroll
        for (int f = 0; f < NF; ++f) mx[f] = keep_max(mx[f], fabs((double)vp[f]));
        if (STEP) {
            const double pw = 0.25 * a64<R>(pv, A_VOL, i);
            const double b = fabs((double)aR<R>(pv, A_BUOY, i)), h = (double)aR<R>(pv, A_HUM, i);
            ms[0] = keep_max(ms[0], pw * b);
            ms[1] = keep_max(ms[1], pw * fabs(h));
            ms[2] = keep_max(ms[2], pw * (b + P.glat * fmax(h, 0.0)));
            ms[3] = keep_max(ms[3], pw);
        }
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) warp_max_to(&pbound[bound_slot<NF>(f)], mx[f]);
    if (STEP) {
#pragma unroll
        for (int k = 0; k < 4; ++k) warp_max_to(&pstep[k], ms[k]);
    }
}

EPIC_DEV void count_parcel(const Params& P, const double* pos, double vol, int* nparg, int* nsparg, unsigned* err) {
    int ci, cj, ck;
    cell_of(P, pos, ci, cj, ck);
    if (ck < -1 || ck > P.nz) { set_err(err, ERRB_ZRANGE); return; }
    long long g = fidx(P, ck, wrapi(cj, P.ny), wrapi(ci, P.nx));
    atomicAdd(&nparg[g], 1);
    if (vol <= P.vmin) atomicAdd(&nsparg[g], 1);
}

// Support vectors of parcel i: stored ones (reuse) or from B (and stored).
template <class R>
EPIC_DEV void vectors(const PView& pv, long long i, bool reuse, bool store, R* eta, R* tau, unsigned* err) {
    if (reuse) {
#pragma unroll
        for (int k = 0; k < 3; ++k) { eta[k] = aR<R>(pv, A_ETA0 + k, i); tau[k] = aR<R>(pv, A_TAU0 + k, i); }
        return;
    }
    R b[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) b[k] = aR<R>(pv, A_B11 + k, i);
    if constexpr (Form<R>::mixed) support_vectors_f32(b, a64<R>(pv, A_VOL, i), eta, tau, err);
    else support_vectors<FastOps>(b, a64<R>(pv, A_VOL, i), eta, tau, nullptr, err);
    if (store) {
#pragma unroll
        for (int k = 0; k < 3; ++k) { aR<R>(pv, A_ETA0 + k, i) = eta[k]; aR<R>(pv, A_TAU0 + k, i) = tau[k]; }
    }
}

// The support points of parcels [q0, q1) into the window (or the grid sums).
template <int NF, class R, bool VEC = true>
EPIC_DEV void scatter_round(const Params& P, const PView& pv, long long q0, long long q1, const WinShared<NF>* ws,
                            unsigned* acc, const Fields7& F, int* nparg, int* nsparg, bool reuse, bool store,
                            int lg, unsigned* err) {
    const Window W = ws->W;
    // The lanes of a warp take groups of 2^lg consecutive parcels spaced about
    // cnt/32 * 2^lg apart (different cells of the box), so that the addresses
    // of one shared-memory atomic spread over the banks (consecutive parcels
    // of one cell would pile onto few), while a group still shares sectors
    // of the parcel loads.
    const int cnt = (int)(q1 - q0);
    const int U = (cnt + (1 << lg) - 1) >> lg;          // groups
    const int cols = 32 >> lg;                          // groups side by side in a warp
    const int S = (U + cols - 1) / cols;                // groups per column
    const int lane = threadIdx.x & 31, gi = lane >> lg, m = lane & ((1 << lg) - 1);
    const LimbOrder lo(win_words<R>());
    for (int r = threadIdx.x >> 5; r < S; r += blockDim.x >> 5) {
        const int u = gi * S + r;
        const int slot = (u << lg) + m;
        if (u >= U || slot >= cnt) continue;
        long long i = q0 + slot;
        double pos[3] = {a64<R>(pv, A_X, i), a64<R>(pv, A_Y, i), a64<R>(pv, A_Z, i)};
        R eta[3], tau[3];
        // VEC: the support vectors may be recomputed here; else they are stored
        vectors<R>(pv, i, VEC ? reuse : true, store, eta, tau, err);
        double vs[NF];
        {
            R vp[NF];
            load_values<NF, R>(P, pv, i, pos[2], vp);
#pragma unroll
            for (int f = 0; f < NF; ++f) vs[f] = (double)vp[f] * ws->scale[f];
        }
        if (NF != 1 && nparg) count_parcel(P, pos, a64<R>(pv, A_VOL, i), nparg, nsparg, err);
        const double ed[3] = {(double)eta[0], (double)eta[1], (double)eta[2]};
        const double td[3] = {(double)tau[0], (double)tau[1], (double)tau[2]};
        double pt[3];
        const int s0 = merge_start(P, pos, ed, td);
        support_point(pos, ed, td, s0, pt);
        Tri cur = trilinear(P, pt);
        for (int q = 1; q < 4; ++q) {
            support_point(pos, ed, td, (s0 + q) & 3, pt);
            if (!merge_into(P, pt, cur)) {
                scatter_tri<NF, R>(P, W, acc, F, cur, vs, lo, err);
                cur = trilinear(P, pt);
            }
        }
        scatter_tri<NF, R>(P, W, acc, F, cur, vs, lo, err);
    }
}

// Support vectors of every parcel from B (get_points, parcel_ellipsoid.f90:
// 216-260), stored for the scatter that follows: the eigen-solver and the
// scatter run as separate kernels, each with a small instruction footprint.
template <class R>
__global__ void __launch_bounds__(PB, 4) k_vectors(PView pv, long long n, unsigned* err) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        R eta[3], tau[3];
        vectors<R>(pv, i, false, true, eta, tau, err);
    }
}

// par2grid scatter (NF = 7 or 5) and vol2grid (NF = 1).
template <int NF, class R, bool VEC>
// vol2grid (NF = 1) has a small window and few live values: three CTAs per SM
__global__ void __launch_bounds__(PB, NF == 1 ? 3 : SB) k_scatter(Params P, PView pv, long long n, Boxes B, Fields7 F,
                                                    const unsigned long long* pbound, int* nparg, int* nsparg,
                                                    int reuse, int store, int lg, unsigned* err) {
    extern __shared__ __align__(16) unsigned acc[];
    __shared__ WinShared<NF> ws;
    const Range Rg = cta_range(P, pv, B, n);
    if (threadIdx.x == 0) {
        for (int k = 0; k < 3; ++k) { ws.mn[k] = INT_MAX; ws.mx[k] = INT_MIN; }
        for (int f = 0; f < NF; ++f) ws.scale[f] = fx_scale(pbound, bound_slot<NF>(f), fx_bits<R>(), err);
        if (Rg.box) ws.W = box_window(P, Rg);
    }
    __syncthreads();
    if (!Rg.box) {
        tail_bounds<NF>(P, Rg, pv, &ws);
        __syncthreads();
        if (threadIdx.x == 0) ws.W = tail_window(P, Rg, ws.mn, ws.mx);
        __syncthreads();
    }
    for (long long q0 = Rg.r0; q0 < Rg.r1; q0 += round_max<R>()) {
        const long long q1 = min(q0 + round_max<R>(), Rg.r1);
        win_zero<NF, R>(acc, ws.W);
        __syncthreads();
        scatter_round<NF, R, VEC>(P, pv, q0, q1, &ws, acc, F, nparg, nsparg, reuse != 0, store != 0, lg, err);
        __syncthreads();
        win_flush<NF, R>(P, acc, ws.W, F);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Fused stage kernel.
struct FusedArgs {
    int stage, last, lg;
    int recwin;   // gathers from the box's records staged in shared memory (split form)
    double ca, cb;
    // surface fluxes of stage 1 (null: none)
    const double* binc;
    const double* hinc;
    double zdepth;
    // the next par2grid's vorticity bounds (StepScalars::pbound[0..2], cleared
    // by the host), or null
    unsigned long long* vbound;
};

// The 14 gathered fields (velog 3, velgradg 8, vtend 3) of a grid point as
// one record of 16 values (128 bytes plain, 64 bytes mixed): a trilinear
// corner is one record, read with 16-byte loads at constant offsets.
constexpr int GREC = 16;

template <class R>
__global__ void k_pack_gather(GatherFields G, R* pack, long long fsz) {
    constexpr int V = 16 / sizeof(R);   // values per 16-byte word
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < fsz * (GREC / V);
         e += (long long)gridDim.x * blockDim.x) {
        long long g = e / (GREC / V);
        int q = (int)(e - g * (GREC / V));
        R v[V];
#pragma unroll
        for (int j = 0; j < V; ++j) {
            int l = q * V + j;
            v[j] = l < 14 ? (R)G.f[l][g] : (R)0;
        }
        if constexpr (Form<R>::mixed) reinterpret_cast<float4*>(pack)[e] = make_float4(v[0], v[1], v[2], v[3]);
        else reinterpret_cast<double2*>(pack)[e] = make_double2(v[0], v[1]);
    }
}

// Corner x/y indices wrapped into the grid; support points lie within a
// cell or two of the domain, so the modulo is rarely needed.
EPIC_DEV int wrap_near(int i, int n) {
    if (i < 0) i += n;
    else if (i >= n) i -= n;
    return ((unsigned)i < (unsigned)n) ? i : wrapi(i, n);
}

// g[l] += sum over the 8 corners of (w / 4) f_l (interpl.f90:17-56, the
// point weight 1/4 of parcel_interpl.f90:433).  Returns false when the
// point leaves the vertical halo.
template <class R>
EPIC_DEV bool gather_tri(const Params& P, const R* __restrict__ pack, const Tri& t, R* g) {
    if (t.ks < -1 || t.ks > P.nz) return false;
    const int i0 = wrap_near(t.is, P.nx), i1 = wrap_near(t.is + 1, P.nx);
    const int j0 = wrap_near(t.js, P.ny), j1 = wrap_near(t.js + 1, P.ny);
#pragma unroll
    for (int ii = 0; ii < 2; ++ii)
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) {
            const long long a = fidx(P, t.ks, jj ? j1 : j0, ii ? i1 : i0);
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
                const R w = (R)(0.25 * t.w[kk][jj][ii]);
                if constexpr (Form<R>::mixed) {
                    const float4* q = reinterpret_cast<const float4*>(pack + (a + kk) * GREC);
#pragma unroll
                    for (int l4 = 0; l4 < 4; ++l4) {
                        const float4 v = __ldg(q + l4);
                        g[4 * l4] = fmaf(w, v.x, g[4 * l4]);
                        g[4 * l4 + 1] = fmaf(w, v.y, g[4 * l4 + 1]);
                        if (4 * l4 + 2 < 14) g[4 * l4 + 2] = fmaf(w, v.z, g[4 * l4 + 2]);
                        if (4 * l4 + 3 < 14) g[4 * l4 + 3] = fmaf(w, v.w, g[4 * l4 + 3]);
                    }
                } else {
                    const double2* q = reinterpret_cast<const double2*>(pack + (a + kk) * GREC);
#pragma unroll
                    for (int l2 = 0; l2 < 7; ++l2) {
                        const double2 v = __ldg(q + l2);
                        g[2 * l2] = fma(w, v.x, g[2 * l2]);
                        g[2 * l2 + 1] = fma(w, v.y, g[2 * l2 + 1]);
                    }
                }
            }
        }
    return true;
}

// Gather records of the grid points around a box, staged in shared memory by
// the stage kernel: the cells of the box and one cell on every side, so the
// corners of every support point within a cell of the box are on chip.
// Records are stored whole (16 values); the 16-byte words of record r are
// permuted by r (word w at w ^ (r mod 8), plain; w ^ (r mod 4), mixed) so
// that the lanes of a warp, each reading word w of its own record, spread
// over all banks.
constexpr int RWM = 0;   // cells of margin around the box
constexpr int RWX = BOXX + 1 + 2 * RWM, RWY = BOXY + 1 + 2 * RWM, RWZ = BOXZ + 1 + 2 * RWM;
template <class R> constexpr int rec_words() { return (int)(GREC * sizeof(R) / 16); }   // 8 plain, 4 mixed
template <class R> constexpr size_t recwin_bytes() { return sizeof(R) * GREC * RWX * RWY * RWZ; }

struct RecWin {
    int gx0, gy0, gz0, WZ;
    int ok;
};

template <class R>
EPIC_DEV RecWin recwin_load(const Params& P, const Range& Rg, bool box, const R* __restrict__ pack, R* srec) {
    constexpr int V = rec_words<R>();
    RecWin W;
    W.gx0 = Rg.ref[0] - RWM;
    W.gy0 = Rg.ref[1] - RWM;
    W.gz0 = Rg.ref[2] - RWM;
    W.WZ = min(RWZ, P.nz + 2 - W.gz0);
    W.ok = box && RWX <= P.nx && RWY <= P.ny;
    if (!W.ok) return W;
    const int nrec = RWX * RWY * W.WZ;
    const uint4* src = reinterpret_cast<const uint4*>(pack);
    uint4* dst = reinterpret_cast<uint4*>(srec);
    for (int e = threadIdx.x; e < nrec * V; e += blockDim.x) {
        const int r = e / V, w = e - r * V;
        const int z = r % W.WZ, xy = r / W.WZ, y = xy % RWY, x = xy / RWY;
        const long long g = fidx(P, W.gz0 + z, wrap_near(W.gy0 + y, P.ny), wrap_near(W.gx0 + x, P.nx));
        dst[r * V + (w ^ (r & (V - 1)))] = __ldg(src + g * V + w);
    }
    return W;
}

// gather_tri from the staged records when the point's corners are in the
// window, else from global memory; the same sums in the same order.
template <class R>
EPIC_DEV bool gather_tri_win(const Params& P, const R* __restrict__ pack, const R* srec, const RecWin& W,
                             const Tri& t, R* g) {
    constexpr int V = rec_words<R>();
    const int lx = wrap_to(t.is - W.gx0, P.nx), ly = wrap_to(t.js - W.gy0, P.ny), lz = t.ks - W.gz0;
    if (!(W.ok && lx + 1 < RWX && ly + 1 < RWY && lz >= 0 && lz + 1 < W.WZ && t.ks >= -1 && t.ks <= P.nz))
        return gather_tri<R>(P, pack, t, g);
#pragma unroll
    for (int ii = 0; ii < 2; ++ii)
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) {
            const int rb = ((lx + ii) * RWY + ly + jj) * W.WZ + lz;
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
                const int r = rb + kk;
                const R w = (R)(0.25 * t.w[kk][jj][ii]);
                if constexpr (Form<R>::mixed) {
                    const float4* q = reinterpret_cast<const float4*>(srec) + r * V;
#pragma unroll
                    for (int l4 = 0; l4 < 4; ++l4) {
                        const float4 v = q[l4 ^ (r & 3)];
                        g[4 * l4] = fmaf(w, v.x, g[4 * l4]);
                        g[4 * l4 + 1] = fmaf(w, v.y, g[4 * l4 + 1]);
                        if (4 * l4 + 2 < 14) g[4 * l4 + 2] = fmaf(w, v.z, g[4 * l4 + 2]);
                        if (4 * l4 + 3 < 14) g[4 * l4 + 3] = fmaf(w, v.w, g[4 * l4 + 3]);
                    }
                } else {
                    const double2* q = reinterpret_cast<const double2*>(srec) + r * V;
#pragma unroll
                    for (int l2 = 0; l2 < 7; ++l2) {
                        const double2 v = q[l2 ^ (r & 7)];
                        g[2 * l2] = fma(w, v.x, g[2 * l2]);
                        g[2 * l2 + 1] = fma(w, v.y, g[2 * l2 + 1]);
                    }
                }
            }
        }
    return true;
}

// get_dBdt (parcel_ellipsoid.f90:466-507) in the attribute type.
template <class R>
EPIC_DEV void dBdt_r(const R* s, const R* b, R B33, R* o) {
    R dwdz = -(s[I_DUDX] + s[I_DVDY]);
    o[0] = R(2) * (s[I_DUDX] * b[0] + s[I_DUDY] * b[1] + s[I_DUDZ] * b[2]);
    o[1] = s[I_DVDX] * b[0] - dwdz * b[1] + s[I_DVDZ] * b[2] + s[I_DUDY] * b[3] + s[I_DUDZ] * b[4];
    o[2] = s[I_DWDX] * b[0] + s[I_DWDY] * b[1] - s[I_DVDY] * b[2] + s[I_DUDY] * b[4] + s[I_DUDZ] * B33;
    o[3] = R(2) * (s[I_DVDX] * b[1] + s[I_DVDY] * b[3] + s[I_DVDZ] * b[4]);
    o[4] = s[I_DWDX] * b[1] + s[I_DVDX] * b[2] + s[I_DWDY] * b[3] - s[I_DUDX] * b[4] + s[I_DVDZ] * B33;
}


template <bool DIAG, class R, bool VOUT = false>
__global__ void __launch_bounds__(PB, SB) k_stage(Params P, PView pv, long long n, Boxes B, const R* pack,
                                                  FusedArgs S, const StepScalars* sc, double* partials,
                                                  unsigned* err) {
    using Ops = typename Form<R>::Ops;
    extern __shared__ __align__(16) unsigned acc[];
    __shared__ double red[PB / 32][NDIAG];
    constexpr int ND = DIAG ? NDIAG : 1;
    // the diagnostic sums of this thread, in shared memory (registers are
    // the stage kernel's limit)
    __shared__ double dsm[ND][PB];
    // largest |0.25 V w_k| of this thread's advanced parcels (the next
    // par2grid's vorticity bounds)
    __shared__ double vmx[3][PB];
#pragma unroll
    for (int k = 0; k < 3; ++k) vmx[k][threadIdx.x] = 0.0;
#pragma unroll
    for (int k = 0; k < ND; ++k) dsm[k][threadIdx.x] = 0.0;
    double* dacc = &dsm[0][threadIdx.x];
#define DACC(k) dacc[(k) * PB]
    const double dt = sc->dt;
    const Range Rg = cta_range(P, pv, B, n);
    // without the scatter pass, the dynamic shared memory holds the box's gather records
    RecWin RW;
    RW.ok = 0;
    if (S.recwin) {
        RW = recwin_load<R>(P, Rg, blockIdx.x < B.nbox, pack, reinterpret_cast<R*>(acc));
        __syncthreads();
    }
    {
        const long long q0 = Rg.r0, q1 = Rg.r1;
        // grid2par + dB/dt + LS-RK update
        for (long long i = q0 + threadIdx.x; i < q1; i += blockDim.x) {
            // bring the next parcel's attribute lines into L2 (one lane per 128-byte line)
            if ((threadIdx.x & 15) == 0 && i + blockDim.x < q1) {
                const long long j = i + blockDim.x;
#pragma unroll
                for (int k = 0; k < 29; ++k) {
                    const int slot = k < 3 ? A_X + k : k < 6 ? A_ETA0 + (k - 3) : k < 9 ? A_TAU0 + (k - 6)
                                   : k < 14 ? A_B11 + (k - 9) : k == 14 ? A_VOL : k < 18 ? A_VX + (k - 15)
                                   : k < 21 ? A_DX + (k - 18) : k < 24 ? A_DVX + (k - 21) : A_DB0 + (k - 24);
                    if (k >= 18 && S.stage == 1) continue;
                    const void* a = Form<R>::mixed ? (const void*)&aR<R>(pv, slot, j) : (const void*)&a64<R>(pv, slot, j);
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
                }
            }
            double pos[3] = {a64<R>(pv, A_X, i), a64<R>(pv, A_Y, i), a64<R>(pv, A_Z, i)};
            // the attributes of the update are loaded before the gathers, so
            // that their latency overlaps the interpolation
            R b[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) b[k] = aR<R>(pv, A_B11 + k, i);
            const double vol = a64<R>(pv, A_VOL, i);
            R vor[3] = {aR<R>(pv, A_VX, i), aR<R>(pv, A_VY, i), aR<R>(pv, A_VZ, i)};
            // the LS-RK accumulators: the mixed form loads them before the
            // gathers (their latency overlaps the interpolation); the FP64
            // form after them (fewer live registers, no spills)
            double dpo[3] = {0.0, 0.0, 0.0};
            R dvo[3] = {(R)0, (R)0, (R)0}, dbo[5] = {(R)0, (R)0, (R)0, (R)0, (R)0};
            auto load_accumulators = [&]() {
                if (S.stage > 1) {
#pragma unroll
                    for (int k = 0; k < 3; ++k) { dpo[k] = a64<R>(pv, A_DX + k, i); dvo[k] = aR<R>(pv, A_DVX + k, i); }
#pragma unroll
                    for (int k = 0; k < 5; ++k) dbo[k] = aR<R>(pv, A_DB0 + k, i);
                }
            };
            if constexpr (Form<R>::mixed) load_accumulators();
            R g[14];
#pragma unroll
            for (int l = 0; l < 14; ++l) g[l] = (R)0;
            {
                R eta[3], tau[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) { eta[k] = aR<R>(pv, A_ETA0 + k, i); tau[k] = aR<R>(pv, A_TAU0 + k, i); }
                const double ed[3] = {(double)eta[0], (double)eta[1], (double)eta[2]};
                const double td[3] = {(double)tau[0], (double)tau[1], (double)tau[2]};
                double pt[3];
                const int s0 = merge_start(P, pos, ed, td);
                support_point(pos, ed, td, s0, pt);
                Tri cur = trilinear(P, pt);
                bool ok = true;
                for (int q = 1; q < 4; ++q) {
                    support_point(pos, ed, td, (s0 + q) & 3, pt);
                    if (!merge_into(P, pt, cur)) {
                        ok = gather_tri_win<R>(P, pack, reinterpret_cast<const R*>(acc), RW, cur, g) && ok;
                        cur = trilinear(P, pt);
                    }
                }
                ok = gather_tri_win<R>(P, pack, reinterpret_cast<const R*>(acc), RW, cur, g) && ok;
                if (!ok) set_err(err, ERRB_ZRANGE);
            }
            if constexpr (!Form<R>::mixed) load_accumulators();
            double dp[3];
            R dv[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                dp[k] = S.stage > 1 ? dpo[k] + (double)g[k] : (double)g[k];
                dv[k] = S.stage > 1 ? dvo[k] + g[11 + k] : g[11 + k];
            }
            const R* strain = &g[3];
            // B33 from the volume constraint in FP64 (parcel_ellipsoid.f90:383-402)
            double bd[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) bd[k] = (double)b[k];
            const double B33d = get_B33<FastOps>(bd, vol, err);
            if (DIAG) {
                // parcel diagnostics before the update (ls_rk.f90:116, parcel_diagnostics.f90:66-120)
                R U[9], D[3];
                full_matrix<Ops>(b, (R)B33d, U);
                sz_eigenvalues<Ops>(U, D);
                double bu = (double)aR<R>(pv, A_BUOY, i);
                double vx = vor[0], vy = vor[1], vz = vor[2];
                DACC(0) += (dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2]) * vol;
                DACC(1) += (vx * vx + vy * vy + vz * vz) * vol;
                double lam = sqrt((double)D[0] / (double)D[2]);
                DACC(2) += lam;
                DACC(3) += lam * lam;
                DACC(4) += vol;
                DACC(5) += vol * vol;
                if (vol <= P.vmin) DACC(6) += 1.0;
                DACC(7) += vol * (vx * vx);
                DACC(8) += vol * (vy * vy);
                DACC(9) += vol * (vz * vz);
                DACC(10) = fmin(DACC(10), bu);
                DACC(11) = fmax(DACC(11), bu);
            }
            if (DIAG && S.binc) {
                // apply_bndry_fluxes after the diagnostics, before the first
                // substep moves the parcel (ls_rk.f90:113-119)
                double fb, fh;
                if (surface_flux(P, pos, S.binc, S.hinc, S.zdepth, dt, fb, fh)) {
                    aR<R>(pv, A_BUOY, i) = (R)((double)aR<R>(pv, A_BUOY, i) + fb);
                    aR<R>(pv, A_HUM, i) = (R)((double)aR<R>(pv, A_HUM, i) + fh);
                }
            }
            R db[5];
            dBdt_r<R>(strain, b, (R)B33d, db);
            if (S.stage > 1) {
#pragma unroll
                for (int k = 0; k < 5; ++k) db[k] = dbo[k] + db[k];
            }
            const double cdt = S.cb * dt;
            const R cdtr = (R)cdt;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                pos[k] = pos[k] + cdt * dp[k];
                vor[k] = vor[k] + cdtr * dv[k];
            }
#pragma unroll
            for (int k = 0; k < 5; ++k) b[k] = b[k] + cdtr * db[k];
            periodic_bc(P, pos);
            if (S.last) {
                if (pos[2] > P.upper[2]) {
                    pos[2] = 2.0 * P.upper[2] - pos[2];
                    b[2] = -b[2]; b[4] = -b[4];
                } else if (pos[2] < P.lower[2]) {
                    pos[2] = 2.0 * P.lower[2] - pos[2];
                    b[2] = -b[2]; b[4] = -b[4];
                }
            } else {
                const R car = (R)S.ca;
#pragma unroll
                for (int k = 0; k < 3; ++k) { dp[k] = S.ca * dp[k]; dv[k] = car * dv[k]; }
#pragma unroll
                for (int k = 0; k < 5; ++k) db[k] = car * db[k];
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                a64<R>(pv, A_X + k, i) = pos[k];
                aR<R>(pv, A_VX + k, i) = vor[k];
                a64<R>(pv, A_DX + k, i) = dp[k];
                aR<R>(pv, A_DVX + k, i) = dv[k];
            }
            if (S.vbound) {
                // the values p2g_values will scatter, in the same arithmetic
                const R pw = (R)(0.25 * vol);
#pragma unroll
                for (int k = 0; k < 3; ++k) vmx[k][threadIdx.x] = keep_max(vmx[k][threadIdx.x], fabs((double)(pw * vor[k])));
            }
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                aR<R>(pv, A_B11 + k, i) = b[k];
                aR<R>(pv, A_DB0 + k, i) = db[k];
            }
            if (VOUT) {
                // support vectors of the advanced shape for the next par2grid
                R eta[3], tau[3];
                if constexpr (Form<R>::mixed) {
                    support_vectors_f32(b, vol, eta, tau, err);
                } else {
                    double bdn[5] = {(double)b[0], (double)b[1], (double)b[2], (double)b[3], (double)b[4]};
                    support_vectors<FastOps>(bdn, vol, eta, tau, nullptr, err);
                }
#pragma unroll
                for (int k = 0; k < 3; ++k) { aR<R>(pv, A_ETA0 + k, i) = eta[k]; aR<R>(pv, A_TAU0 + k, i) = tau[k]; }
            }
        }
    }
    if (S.vbound) {
#pragma unroll
        for (int k = 0; k < 3; ++k) warp_max_to(&S.vbound[k], vmx[k][threadIdx.x]);
    }
    if (DIAG) {
        int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
        for (int k = 0; k < ND; ++k) {
            double v = DACC(k);
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
#undef DACC
}

// ---------------------------------------------------------------------------
static Fields7 fields7(Ctx& c, bool moist = true) {
    Fields7 F;
    F.f[0] = c.vortg(0); F.f[1] = c.vortg(1); F.f[2] = c.vortg(2);
    F.f[3] = c.dbuoyg(); F.f[4] = c.humg(); F.f[5] = c.tbuoyg(); F.f[6] = c.volg();
    F.mask = moist ? ALL_FIELDS : DRY_FIELDS;
    return F;
}

static Boxes boxes(const Ctx& c) {
    Boxes B;
    bool valid = c.box_start != nullptr && c.n_box > 0;
    B.start = c.box_start;
    B.nbox = valid ? c.nbox : 0;
    B.nby = (c.P.ny + BOXY - 1) / BOXY;
    B.nbz = (c.P.nz + BOXZ - 1) / BOXZ;
    B.n_box = valid ? std::min(c.n_box, c.n) : 0;
    return B;
}

static int sgrid(const Ctx& c, const Boxes& B) {
    long long tail = c.n - B.n_box;
    return (int)std::max<long long>(1, B.nbox + (tail + SCHUNK - 1) / SCHUNK);
}

int box_count(const Params& P) {
    return ((P.nx + BOXX - 1) / BOXX) * ((P.ny + BOXY - 1) / BOXY) * ((P.nz + BOXZ - 1) / BOXZ);
}

long long stage_grid_max(const Params& P, long long cap) {
    return (long long)box_count(P) + (cap + SCHUNK - 1) / SCHUNK + 1;
}

static void zero_p2g_fields(Ctx& c) {
    const Params& P = c.P;
    // the 7 scattered fields are contiguous slots 3..5 and 17..20 of the field block
    CK(cudaMemsetAsync(c.vortg(0), 0, sizeof(double) * 3 * P.fsz, c.stream));
    CK(cudaMemsetAsync(c.tbuoyg(), 0, sizeof(double) * 4 * P.fsz, c.stream));
    CK(cudaMemsetAsync(c.nparg, 0, sizeof(int) * P.fsz, c.stream));
    CK(cudaMemsetAsync(c.nsparg, 0, sizeof(int) * P.fsz, c.stream));
    CK(cudaMemsetAsync(&c.dsc->count, 0, sizeof(long long), c.stream));
}

template <typename K>
static void set_smem(K kernel, size_t bytes) {
    allow_smem(kernel, bytes);
}

// count: par2grid's parcel counts nparg / nsparg (NF = 7 or 5)
template <int NF, class R>
static void launch_scatter(Ctx& c, const Fields7& F, bool reuse, bool store, int lg, bool count) {
    // the fixed-point scales: the largest value of every scattered field,
    // from the kernels that produced the values or from a pass of their own
    if (NF == 1 && c.v2g_bound_ready) {
        CK(cudaMemcpyAsync(&c.dsc->pbound[6], &c.dsc->vbound, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                           c.stream));
    } else if (NF == 1 || !c.p2g_bound_ready) {
        CK(cudaMemsetAsync(c.dsc->pbound, 0, sizeof(c.dsc->pbound), c.stream));
        k_p2g_bounds<NF, R, false><<<pgrid(c.n), PB, 0, c.stream>>>(c.P, c.pv, c.n, c.dsc->pbound, nullptr);
        CKL();
    }
    if (!reuse && store && c.vectors_kernel) {
        k_vectors<R><<<pgrid(c.n), PB, 0, c.stream>>>(c.pv, c.n, &c.dsc->err);
        CKL();
        reuse = true;
    }
    size_t sm = win_bytes<R, NF>();
    Boxes B = boxes(c);
    int* np = count ? c.nparg : nullptr;
    int* nsp = count ? c.nsparg : nullptr;
    auto run = [&](auto kernel) {
        set_smem(kernel, sm);
        kernel<<<sgrid(c, B), PB, sm, c.stream>>>(c.P, c.pv, c.n, B, F, c.dsc->pbound, np, nsp, reuse, store, lg,
                                                   &c.dsc->err);
        CKL();
    };
    if (reuse) run(k_scatter<NF, R, false>);
    else run(k_scatter<NF, R, true>);
}

// par2grid fields: all 7 (moist) or the dry set
template <class R>
static void launch_p2g(Ctx& c, bool moist, bool reuse, bool store, bool count) {
    c.p2g_counted = count;
    if (moist) launch_scatter<7, R>(c, fields7(c, true), reuse, store, c.scatter_lg[1], count);
    else launch_scatter<5, R>(c, fields7(c, false), reuse, store, c.scatter_lg[1], count);
}

void scatter_p2g(Ctx& c, bool reuse, bool store, bool moist) {
    zero_p2g_fields(c);
    if (c.n == 0) return;
    prof_begin(c, "p2g");
    if (c.pv.mixed) launch_p2g<float>(c, moist, reuse, store, true);
    else launch_p2g<double>(c, moist, reuse, store, true);
    prof_end(c, "p2g");
}

void scatter_v2g(Ctx& c, bool reuse) {
    CK(cudaMemsetAsync(c.volg(), 0, sizeof(double) * c.P.fsz, c.stream));
    if (c.n == 0) return;
    Fields7 F;
    F.f[0] = c.volg();
    F.mask = 1;
    prof_begin(c, "v2g");
    if (c.pv.mixed) launch_scatter<1, float>(c, F, reuse, true, c.scatter_lg[0], false);
    else launch_scatter<1, double>(c, F, reuse, true, c.scatter_lg[0], false);
    prof_end(c, "v2g");
}

// The scales of the step's first par2grid and the step bounds (pstep) that
// the later stages' scatters take with their vorticity bounds.
void p2g_step_bounds(Ctx& c) {
    CK(cudaMemsetAsync(c.dsc->pbound, 0, sizeof(c.dsc->pbound) + sizeof(c.dsc->pstep), c.stream));
    if (c.n == 0) return;
    if (c.pv.mixed) k_p2g_bounds<7, float, true><<<pgrid(c.n), PB, 0, c.stream>>>(c.P, c.pv, c.n, c.dsc->pbound, c.dsc->pstep);
    else k_p2g_bounds<7, double, true><<<pgrid(c.n), PB, 0, c.stream>>>(c.P, c.pv, c.n, c.dsc->pbound, c.dsc->pstep);
    CKL();
}

int p2g_fx_bits(const Ctx& c) { return c.pv.mixed ? fx_bits<float>() : fx_bits<double>(); }

template <class R>
static void launch_stage(Ctx& c, const FusedArgs& S, bool with_diag, bool scatter) {
    GatherFields G;
    for (int k = 0; k < 3; ++k) G.f[k] = c.velog(k);
    for (int k = 0; k < 8; ++k) G.f[3 + k] = c.velgrad(k);
    for (int k = 0; k < 3; ++k) G.f[11 + k] = c.vtend(k);
    G.pack = nullptr;
    R* pack = reinterpret_cast<R*>(c.gpack);
    constexpr int V = 16 / sizeof(R);
    k_pack_gather<R><<<pgrid(c.P.fsz * (GREC / V)), PB, 0, c.stream>>>(G, pack, c.P.fsz);
    CKL();
    if (scatter) zero_p2g_fields(c);
    Boxes B = boxes(c);
    int g = sgrid(c, B);
    if (with_diag) {
        c.n_partials = g;
        c.diag_buf = c.stage_partials;
    }
    const bool moist = S.stage + 1 == c.n_stages;
    size_t sm = S.recwin ? recwin_bytes<R>() : 0;
    // the next scatter's scales: vorticity bounds from this kernel, the rest
    // from the step bounds (volume, buoyancy and humidity are those of the
    // step's first par2grid)
    FusedArgs Sk = S;
    Sk.vbound = nullptr;
    const bool fuse_bounds = scatter && c.pstep_valid;
    if (fuse_bounds) {
        CK(cudaMemsetAsync(c.dsc->pbound, 0, 3 * sizeof(unsigned long long), c.stream));
        CK(cudaMemcpyAsync(&c.dsc->pbound[3], c.dsc->pstep, sizeof(c.dsc->pstep), cudaMemcpyDeviceToDevice, c.stream));
        Sk.vbound = c.dsc->pbound;
    }
    auto launch = [&](auto kernel) {
        if (sm) set_smem(kernel, sm);
        prof_begin(c, "stage");
        kernel<<<g, PB, sm, c.stream>>>(c.P, c.pv, c.n, B, pack, Sk, c.dsc, c.stage_partials, &c.dsc->err);
        CKL();
        prof_end(c, "stage");
    };
    // the stage kernel may also compute the support vectors of the advanced
    // shapes, which the scatter then reads
    const bool vout = scatter && c.stage_vectors;
    if (with_diag) vout ? launch(k_stage<true, R, true>) : launch(k_stage<true, R>);
    else vout ? launch(k_stage<false, R, true>) : launch(k_stage<false, R>);
    if (scatter) {
        prof_begin(c, "stage_p2g");
        // the par2grid of stage + 1: dbuoyg and humg only for the last stage;
        // the parcel counts of the intermediate stages are not read (field
        // diagnostics use the step's first par2grid); the last one keeps them
        c.p2g_bound_ready = fuse_bounds;
        launch_p2g<R>(c, moist, vout, true, moist);
        c.p2g_bound_ready = false;
        prof_end(c, "stage_p2g");
    }
}

// One LS-RK stage (grid2par + update), then the next stage's par2grid
// scatter (not after the last stage).
void fused_stage(Ctx& c, int stage, bool with_diag) {
    FusedArgs S;
    S.stage = stage;
    S.last = stage == c.n_stages;
    S.ca = c.ca[stage - 1];
    S.cb = c.cb[stage - 1];
    S.lg = c.scatter_lg[2];
    S.recwin = c.stage_recwin;
    // surface fluxes: inside the stage-1 kernel after its diagnostics, or
    // (no diagnostics) by their own kernel before it
    const bool flux = stage == 1 && c.flux_on;
    if (flux && !with_diag) apply_bndry_fluxes(c);
    S.binc = flux && with_diag ? c.binc : nullptr;
    S.hinc = flux && with_diag ? c.hinc : nullptr;
    S.zdepth = c.zdepth;
    S.vbound = nullptr;
    bool scatter = !S.last;
    if (c.pv.mixed) launch_stage<float>(c, S, with_diag, scatter);
    else launch_stage<double>(c, S, with_diag, scatter);
}

// ---------------------------------------------------------------------------
// Box ordering of the parcel store: key = box (z fastest), then the cell
// inside the box (z fastest).  Only the attributes live at the start of a
// step are moved (state and support vectors).
__global__ void k_sort_keys(Params P, PView pv, long long n, unsigned* key, int* idx) {
    int nby = (P.ny + BOXY - 1) / BOXY, nbz = (P.nz + BOXZ - 1) / BOXZ;
    PLOOP(n) {
        double p[3] = {pv.get(A_X, i), pv.get(A_Y, i), pv.get(A_Z, i)};
        int ci, cj, ck;
        cell_of(P, p, ci, cj, ck);
        ci = min(max(ci, 0), P.nx - 1);
        cj = min(max(cj, 0), P.ny - 1);
        ck = min(max(ck, 0), P.nz - 1);
        unsigned box = (unsigned)(((ci / BOXX) * nby + cj / BOXY) * nbz + ck / BOXZ);
        unsigned local = (unsigned)(((ci % BOXX) * BOXY + cj % BOXY) * BOXZ + ck % BOXZ);
        key[i] = box * (unsigned)BOXC + local;
        idx[i] = (int)i;
    }
}

// First parcel of every box, from the sorted keys.
__global__ void k_box_start(const unsigned* key, long long n, int nbox, int* start) {
    PLOOP(n) {
        int b = (int)(key[i] / BOXC);
        int prev = i > 0 ? (int)(key[i - 1] / BOXC) : -1;
        for (int v = prev + 1; v <= b; ++v) start[v] = (int)i;
        if (i == n - 1)
            for (int v = b + 1; v <= nbox; ++v) start[v] = (int)n;
    }
}

// The 20 live slots of parcel perm[i] into slot i of the other store: all
// loads of a parcel are issued before its stores (the slot types are known at
// compile time, MIXED: the FP32 slots of the mixed form).
template <bool MIXED>
__global__ void k_permute(PView src, PView dst, long long n, const int* perm) {
    constexpr int attrs[20] = {A_X, A_Y, A_Z, A_VX, A_VY, A_VZ, A_B11, A_B12, A_B13, A_B22, A_B23, A_VOL, A_BUOY,
                               A_HUM, A_ETA0, A_ETA0 + 1, A_ETA0 + 2, A_TAU0, A_TAU0 + 1, A_TAU0 + 2};
    PLOOP(n) {
        const long long p = perm[i];
        double v[20];
#pragma unroll
        for (int a = 0; a < 20; ++a)
            v[a] = (MIXED && attr_f32(attrs[a])) ? (double)src.f(attrs[a])[p] : src.d(attrs[a])[p];
#pragma unroll
        for (int a = 0; a < 20; ++a) {
            if (MIXED && attr_f32(attrs[a])) dst.f(attrs[a])[i] = (float)v[a];
            else dst.d(attrs[a])[i] = v[a];
        }
    }
}

// One slot gathered through the permutation into a scratch array.
template <class E>
__global__ void k_gather_slot(const E* src, E* tmp, long long n, const int* perm) {
    PLOOP(n) tmp[i] = src[perm[i]];
}

// Scratch bytes of sort_parcels for n parcels: keys and indices twice, CUB.
size_t sort_scratch_bytes(long long n) {
    size_t cubb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, cubb, (unsigned*)0, (unsigned*)0, (int*)0, (int*)0, (int)n, 0, 32);
    return 4 * ((sizeof(unsigned) * n + 255) & ~(size_t)255) + cubb + 1024;
}

void sort_parcels(Ctx& c) {
    long long n = c.n;
    c.n_box = 0;
    if (n < 2 || c.box_start == nullptr) return;
    size_t cubb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, cubb, (unsigned*)0, (unsigned*)0, (int*)0, (int*)0, (int)n, 0, 32,
                                    c.stream);
    size_t bytes = sort_scratch_bytes(n);
    char* base = reinterpret_cast<char*>(c.get_scratch(bytes));
    auto take = [&](size_t b) { char* p = base; base += (b + 255) & ~(size_t)255; return p; };
    unsigned* k0 = reinterpret_cast<unsigned*>(take(sizeof(unsigned) * n));
    unsigned* k1 = reinterpret_cast<unsigned*>(take(sizeof(unsigned) * n));
    int* i0 = reinterpret_cast<int*>(take(sizeof(int) * n));
    int* i1 = reinterpret_cast<int*>(take(sizeof(int) * n));
    void* tmp = take(cubb);
    k_sort_keys<<<pgrid(n), PB, 0, c.stream>>>(c.P, c.pv, n, k0, i0);
    CKL();
    unsigned long long maxkey = (unsigned long long)c.nbox * BOXC;
    int endbit = 1;
    while ((1ull << endbit) < maxkey) ++endbit;
    CK(cub::DeviceRadixSort::SortPairs(tmp, cubb, k0, k1, i0, i1, (int)n, 0, endbit, c.stream));
    k_box_start<<<pgrid(n), PB, 0, c.stream>>>(k1, n, c.nbox, c.box_start);
    CKL();
    if (c.pv_alt) {
        PView dst{c.pv_alt, c.cap, c.pv.mixed};
        if (c.pv.mixed) k_permute<true><<<pgrid(n), PB, 0, c.stream>>>(c.pv, dst, n, i1);
        else k_permute<false><<<pgrid(n), PB, 0, c.stream>>>(c.pv, dst, n, i1);
        CKL();
        std::swap(c.pv.base, c.pv_alt);
    } else {
        // no second store: slot by slot through the (now free) key arrays k0, k1
        const int live[20] = {A_X, A_Y, A_Z, A_VX, A_VY, A_VZ, A_B11, A_B12, A_B13, A_B22, A_B23, A_VOL, A_BUOY,
                              A_HUM, A_ETA0, A_ETA0 + 1, A_ETA0 + 2, A_TAU0, A_TAU0 + 1, A_TAU0 + 2};
        void* tmp8 = k0;   // k0 and k1 are contiguous: >= 8 n bytes
        for (int a : live) {
            if (c.pv.f32(a)) {
                k_gather_slot<float><<<pgrid(n), PB, 0, c.stream>>>(c.pv.f(a), static_cast<float*>(tmp8), n, i1);
                CKL();
                CK(cudaMemcpyAsync(c.pv.f(a), tmp8, sizeof(float) * n, cudaMemcpyDeviceToDevice, c.stream));
            } else {
                k_gather_slot<double><<<pgrid(n), PB, 0, c.stream>>>(c.pv.d(a), static_cast<double*>(tmp8), n, i1);
                CKL();
                CK(cudaMemcpyAsync(c.pv.d(a), tmp8, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
            }
        }
    }
    if (c.rank) {
        // container indices follow the permutation through the key arrays
        int* tr = reinterpret_cast<int*>(k0);
        k_gather_slot<int><<<pgrid(n), PB, 0, c.stream>>>(c.rank, tr, n, i1);
        CKL();
        CK(cudaMemcpyAsync(c.rank, tr, sizeof(int) * n, cudaMemcpyDeviceToDevice, c.stream));
    }
    if (c.label) {
        // labels and dilutions follow the permutation through the key arrays
        // (free again after k_box_start; k0 and k1 hold >= 8 n bytes)
        long long* tl = reinterpret_cast<long long*>(k0);
        k_gather_slot<long long><<<pgrid(n), PB, 0, c.stream>>>(c.label, tl, n, i1);
        CKL();
        CK(cudaMemcpyAsync(c.label, tl, sizeof(long long) * n, cudaMemcpyDeviceToDevice, c.stream));
        double* td = reinterpret_cast<double*>(k0);
        k_gather_slot<double><<<pgrid(n), PB, 0, c.stream>>>(c.dil, td, n, i1);
        CKL();
        CK(cudaMemcpyAsync(c.dil, td, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
    }
    c.n_box = n;
}

}  // namespace epic
