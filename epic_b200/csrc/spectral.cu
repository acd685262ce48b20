// Spectral part of the step on the device: batched shared-memory FFTs along x
// and y in the reference's Hermitian storage, vertical sine/cosine transforms,
// and the vorticity inversion (vor2vel), vorticity tendency, divergent-flow
// solve (diverge + lapinv1) and the time-step reduction.
//
// Reference semantics:
//   fftxyp2s / fftxys2p  sta3dfft.f90:134-257, forfft / revfft stafft.f90:196-403
//   dst / dct            stafft.f90:410-550
//   diffx / diffy        sta3dfft.f90:301-374 (+ reverse_x/y, mpi_reverse.f90:332-398)
//   vor2vel, vel2vgrad   inversion.f90:25-317
//   vorticity_tendency   inversion.f90:321-404
//   diverge, lapinv1     inversion.f90:410-455, inversion_utils.f90:567-589
//   get_time_step        rk_utils.f90:70-183
#include "ctx.hpp"
#include "eigen.cuh"

#include <climits>
#include <cmath>
#include <vector>
#include <algorithm>
#include <cstring>
#include <initializer_list>
#include <utility>
#include <type_traits>

#include <cooperative_groups.h>

namespace epic {

// ---------------------------------------------------------------------------
// Batched real FFT of lines along x or y, one tile of T lines per CTA.
// Two real lines are packed into one complex line (z = a + i b), transformed
// with a mixed-radix Stockham FFT in shared memory, and separated with the
// conjugate-symmetry identities.  Output uses the stafft Hermitian layout:
//   out[k] = Re X_k / sqrt(n) (k <= n/2),  out[n-k] = Im X_k / sqrt(n).
constexpr int MAXF = 12;

struct FFTBatch {
    const void* in[MAXF];   // element type TI of the kernel
    void* out[MAXF];        // element type TO
    long long es;          // element stride along the transformed axis
    long long row_stride;  // stride between rows of lines
    int nl;                // lines per row (nz + 1, contiguous)
    int T;                 // lines per tile (even)
    int n;
    int nfac;
    int fac[16];
    const double2* tw;
    double scale;
};

EPIC_DEV double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
EPIC_DEV double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
EPIC_DEV double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// Stockham autosort passes on L complex lines of length n held in a / b.
// Returns the buffer holding the result.
EPIC_DEV double2* stockham(double2* a, double2* b, int L, int n, int nfac, const int* fac,
                           const double2* tw) {
    int Ns = 1;
    for (int s = 0; s < nfac; ++s) {
        int p = fac[s];
        int m = n / p;
        int tstep = n / (Ns * p);
        for (int idx = threadIdx.x; idx < L * m; idx += blockDim.x) {
            int l2 = idx / m, j = idx - l2 * m;
            int k = j % Ns;
            const double2* src = a + (long long)l2 * n;
            double2* dst = b + (long long)l2 * n;
            double2 v[5];
            for (int r = 0; r < p; ++r) v[r] = src[j + r * m];
            for (int r = 1; r < p; ++r) v[r] = cmul(v[r], tw[(k * r * tstep) % n]);
            double2 o[5];
            if (p == 2) {
                o[0] = cadd(v[0], v[1]);
                o[1] = csub(v[0], v[1]);
            } else if (p == 4) {
                double2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
                double2 t2 = cadd(v[1], v[3]), d = csub(v[1], v[3]);
                double2 t3 = make_double2(d.y, -d.x);   // -i * d
                o[0] = cadd(t0, t2);
                o[2] = csub(t0, t2);
                o[1] = cadd(t1, t3);
                o[3] = csub(t1, t3);
            } else {
                int step = n / p;
                for (int q = 0; q < p; ++q) {
                    double2 acc = v[0];
                    for (int r = 1; r < p; ++r) acc = cadd(acc, cmul(v[r], tw[((q * r) % p) * step]));
                    o[q] = acc;
                }
            }
            int base = (j / Ns) * Ns * p + k;
            for (int r = 0; r < p; ++r) dst[base + r * Ns] = o[r];
        }
        __syncthreads();
        double2* t = a; a = b; b = t;
        Ns *= p;
    }
    return a;
}

template <bool FWD, class TI, class TO>
__global__ void __launch_bounds__(256) k_fft_lines(FFTBatch B) {
    extern __shared__ double smem[];
    const int n = B.n, T = B.T, L = T / 2;
    double* sx = smem;
    double2* cz = reinterpret_cast<double2*>(sx + (long long)T * n);
    double2* cw = cz + (long long)L * n;
    double2* stw = cw + (long long)L * n;
    const TI* in = static_cast<const TI*>(B.in[blockIdx.z]);
    TO* out = static_cast<TO*>(B.out[blockIdx.z]);
    const int l0 = blockIdx.x * T;
    const long long rowbase = (long long)blockIdx.y * B.row_stride + 1;

    for (int i = threadIdx.x; i < n; i += blockDim.x) stw[i] = B.tw[i];
    for (int idx = threadIdx.x; idx < T * n; idx += blockDim.x) {
        int l = idx % T, e = idx / T;
        int line = l0 + l;
        sx[e * T + l] = (line < B.nl) ? (double)in[rowbase + line + (long long)e * B.es] : 0.0;
    }
    __syncthreads();
    const int h = n / 2;
    if (FWD) {
        for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
            int l2 = idx / n, e = idx - l2 * n;
            cz[idx] = make_double2(sx[e * T + 2 * l2], sx[e * T + 2 * l2 + 1]);
        }
    } else {
        // Hermitian lines a, b -> conj(Xa + i Xb)
        for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
            int l2 = idx / n, k = idx - l2 * n;
            int la = 2 * l2, lb = la + 1;
            double ra, ia, rb, ib;
            if (k == 0 || k == h) {
                ra = sx[k * T + la]; ia = 0.0;
                rb = sx[k * T + lb]; ib = 0.0;
            } else if (k < h) {
                ra = sx[k * T + la]; ia = sx[(n - k) * T + la];
                rb = sx[k * T + lb]; ib = sx[(n - k) * T + lb];
            } else {
                ra = sx[(n - k) * T + la]; ia = -sx[k * T + la];
                rb = sx[(n - k) * T + lb]; ib = -sx[k * T + lb];
            }
            cz[idx] = make_double2(ra - ib, -(ia + rb));
        }
    }
    __syncthreads();
    double2* res = stockham(cz, cw, L, n, B.nfac, B.fac, stw);
    if (FWD) {
        for (int idx = threadIdx.x; idx < L * (h + 1); idx += blockDim.x) {
            int l2 = idx / (h + 1), k = idx - l2 * (h + 1);
            double2 zk = res[(long long)l2 * n + k];
            double2 zn = res[(long long)l2 * n + ((n - k) % n)];
            int la = 2 * l2, lb = la + 1;
            sx[k * T + la] = 0.5 * (zk.x + zn.x);
            sx[k * T + lb] = 0.5 * (zk.y + zn.y);
            if (k > 0 && k < h) {
                sx[(n - k) * T + la] = 0.5 * (zk.y - zn.y);
                sx[(n - k) * T + lb] = 0.5 * (zn.x - zk.x);
            }
        }
    } else {
        for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
            int l2 = idx / n, e = idx - l2 * n;
            double2 z = res[idx];
            sx[e * T + 2 * l2] = z.x;
            sx[e * T + 2 * l2 + 1] = -z.y;
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < T * n; idx += blockDim.x) {
        int l = idx % T, e = idx / T;
        int line = l0 + l;
        if (line < B.nl) out[rowbase + line + (long long)e * B.es] = (TO)(sx[e * T + l] * B.scale);
    }
}

// ---------------------------------------------------------------------------
// 2-D plane FFT: one CTA transforms one (field, z) plane of an n x n grid
// (n = 16 .. 128) held in shared memory as P[ix * S + iy], S = n + 2.  The y
// pass transforms the line pairs (rows 2p, 2p+1) and the x pass the column
// pairs (2q, 2q+1), two real lines packed as one complex line, with the same
// Hermitian storage and 1/sqrt(n) scaling as k_fft_lines.  A complex line of
// length N = N1 * N2 is done by N2 threads of one warp: a radix-N1 DFT in
// registers over n1 (stride N2), the twiddles W_N^(t k1), an exchange through
// the line's own storage, and a radix-N2 DFT in registers; only warp-level
// synchronisation inside a pass.
template <class T>
struct CX {
    T x, y;
};
template <class T> EPIC_DEV CX<T> cx(T a, T b) { CX<T> r; r.x = a; r.y = b; return r; }
template <class T> EPIC_DEV CX<T> operator+(CX<T> a, CX<T> b) { return cx<T>(a.x + b.x, a.y + b.y); }
template <class T> EPIC_DEV CX<T> operator-(CX<T> a, CX<T> b) { return cx<T>(a.x - b.x, a.y - b.y); }
template <class T> EPIC_DEV CX<T> cmulw(CX<T> a, CX<T> w) { return cx<T>(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x); }

// cos(2 pi j / 32) = cos(j pi / 16), j = 0..8, rounded to double
constexpr double K1 = 0.98078528040323043, K2 = 0.92387953251128674, K3 = 0.83146961230254524,
                 K4 = 0.70710678118654757, K5 = 0.55557023301960218, K6 = 0.38268343236508978,
                 K7 = 0.19509032201612825;
EPIC_DEV double w32c(int j) {
    const double c[32] = {1.0, K1, K2, K3, K4, K5, K6, K7, 0.0, -K7, -K6, -K5, -K4, -K3, -K2, -K1,
                          -1.0, -K1, -K2, -K3, -K4, -K5, -K6, -K7, 0.0, K7, K6, K5, K4, K3, K2, K1};
    return c[j & 31];
}
// a * exp(-2 pi i j / 32) with the quarter turns done exactly
template <class T>
EPIC_DEV CX<T> rot32(CX<T> a, int j) {
    j &= 31;
    if (j == 0) return a;
    if (j == 8) return cx<T>(a.y, -a.x);
    if (j == 16) return cx<T>(-a.x, -a.y);
    if (j == 24) return cx<T>(-a.y, a.x);
    return cmulw(a, cx<T>((T)w32c(j), (T)-w32c((j + 24) & 31)));
}

constexpr int bitrev_c(int i, int n) {
    int r = 0;
    for (int b = 1; b < n; b <<= 1) { r = (r << 1) | (i & 1); i >>= 1; }
    return r;
}

// Forward DFT of N <= 32 values in registers (natural order in and out).
template <int N, class T>
EPIC_DEV void fft_reg(CX<T> (&v)[N]) {
#pragma unroll
    for (int half = N / 2; half >= 1; half >>= 1) {
#pragma unroll
        for (int blk = 0; blk < N; blk += 2 * half) {
#pragma unroll
            for (int j = 0; j < half; ++j) {
                CX<T> a = v[blk + j], b = v[blk + j + half];
                v[blk + j] = a + b;
                v[blk + j + half] = rot32(a - b, j * (32 / (2 * half)));
            }
        }
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const int r = bitrev_c(i, N);
        if (r > i) { CX<T> t = v[i]; v[i] = v[r]; v[r] = t; }
    }
}

// a * exp(-2 pi i j / 24), j mod 24 (multiples of 15 degrees), quarter turns exact
constexpr double C15 = 0.96592582628906831, S15 = 0.25881904510252074, C30 = 0.86602540378443865;
EPIC_DEV double w24c(int j) {
    const double c[24] = {1.0, C15, C30, K4, 0.5, S15, 0.0, -S15, -0.5, -K4, -C30, -C15,
                          -1.0, -C15, -C30, -K4, -0.5, -S15, 0.0, S15, 0.5, K4, C30, C15};
    return c[j % 24];
}
template <class T>
EPIC_DEV CX<T> rot24(CX<T> a, int j) {
    j %= 24;
    if (j == 0) return a;
    if (j == 6) return cx<T>(a.y, -a.x);
    if (j == 12) return cx<T>(-a.x, -a.y);
    if (j == 18) return cx<T>(-a.y, a.x);
    return cmulw(a, cx<T>((T)w24c(j), (T)-w24c((j + 18) % 24)));
}

// Forward DFT of N = 3 M values in registers (M = 4 or 8, natural order in
// and out): DFTs of the three decimated subsequences v[3 q + r], twiddles
// exp(-2 pi i r k / N), and radix-3 butterflies.
template <int N, class T>
EPIC_DEV void fft_reg3(CX<T> (&v)[N]) {
    constexpr int M = N / 3;
    static_assert(M * 3 == N && 24 % N == 0, "N = 12 or 24");
    CX<T> u[3][M];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < M; ++q) u[r][q] = v[3 * q + r];
#pragma unroll
    for (int r = 0; r < 3; ++r) fft_reg<M>(u[r]);
#pragma unroll
    for (int r = 1; r < 3; ++r)
#pragma unroll
        for (int k = 1; k < M; ++k) u[r][k] = rot24(u[r][k], (24 / N) * r * k);
    const T h = (T)C30;   // sqrt(3) / 2
#pragma unroll
    for (int k = 0; k < M; ++k) {
        const CX<T> a = u[0][k], s = u[1][k] + u[2][k], d = u[1][k] - u[2][k];
        const CX<T> m = cx<T>(a.x - T(0.5) * s.x, a.y - T(0.5) * s.y);
        const CX<T> rr = cx<T>(h * d.x, h * d.y);
        v[k] = a + s;
        v[k + M] = cx<T>(m.x + rr.y, m.y - rr.x);       // m - i rr
        v[k + 2 * M] = cx<T>(m.x - rr.y, m.y + rr.x);   // m + i rr
    }
}

template <int N, class T>
EPIC_DEV void fft_any(CX<T> (&v)[N]) {
    if constexpr ((N & (N - 1)) == 0) fft_reg<N>(v);
    else fft_reg3<N>(v);
}

template <int N> struct Radix;
template <> struct Radix<48> { static constexpr int N1 = 12, N2 = 4; };
template <> struct Radix<96> { static constexpr int N1 = 24, N2 = 4; };
template <> struct Radix<16> { static constexpr int N1 = 4, N2 = 4; };
template <> struct Radix<32> { static constexpr int N1 = 8, N2 = 4; };
template <> struct Radix<64> { static constexpr int N1 = 8, N2 = 8; };
template <> struct Radix<128> { static constexpr int N1 = 16, N2 = 8; };
template <> struct Radix<256> { static constexpr int N1 = 16, N2 = 16; };
template <> struct Radix<512> { static constexpr int N1 = 32, N2 = 16; };

// Line geometry inside the plane: real element c of line a at P[a0 + c*es],
// of line b at P[a0 + c*es + bo]; complex scratch element c at P[s0 + c*cs].
// A line split over two blocks of rows (the half-plane kernel) puts element
// c at a0 + (c & msk)*es + (c >> sh)*es2 (the scratch likewise with cs).
struct LineGeo {
    int a0, es, bo, s0, cs;
    int msk = -1, sh = 30, es2 = 0;
};

template <int N, bool FWD, class T>
EPIC_DEV void line_fft(T* P, const LineGeo g, int t, const CX<T>* tw, T scale) {
    constexpr int N1 = Radix<N>::N1, N2 = Radix<N>::N2, KPT = N1 / N2, H = N / 2;
    auto EL = [&](int c) { return g.a0 + (c & g.msk) * g.es + (c >> g.sh) * g.es2; };
    // Scratch slot of complex element k, XOR-swizzled within blocks of 8: the
    // transposed reads (k = t * N1 + ...) of the lanes of a quarter warp then
    // fall into 8 different 16-byte bank groups instead of one.
    constexpr int LG1 = N1 >= 32 ? 5 : N1 >= 16 ? 4 : N1 >= 8 ? 3 : N1 >= 4 ? 2 : 1;
    auto SC = [&](int k) -> CX<T>& {
        k ^= (k >> LG1) & 7;
        return *reinterpret_cast<CX<T>*>(P + g.s0 + (k & g.msk) * g.cs + (k >> g.sh) * g.es2);
    };
    CX<T> v[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) {
        const int c = t + N2 * m;
        if (FWD) {
            v[m] = cx<T>(P[EL(c)], P[EL(c) + g.bo]);
        } else {
            // conj(A + i B) from the Hermitian lines a, b
            T ra, ia, rb, ib;
            if (c == 0 || c == H) {
                ra = P[EL(c)]; ia = T(0);
                rb = P[EL(c) + g.bo]; ib = T(0);
            } else if (c < H) {
                ra = P[EL(c)]; ia = P[EL(N - c)];
                rb = P[EL(c) + g.bo]; ib = P[EL(N - c) + g.bo];
            } else {
                ra = P[EL(N - c)]; ia = -P[EL(c)];
                rb = P[EL(N - c) + g.bo]; ib = -P[EL(c) + g.bo];
            }
            v[m] = cx<T>(ra - ib, -(ia + rb));
        }
    }
    fft_any<N1>(v);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmulw(v[k1], tw[t * k1]);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) SC(k1 * N2 + t) = v[k1];
    __syncwarp();
    CX<T> y[KPT][N2];
#pragma unroll
    for (int e = 0; e < KPT; ++e)
#pragma unroll
        for (int t2 = 0; t2 < N2; ++t2) y[e][t2] = SC((t * KPT + e) * N2 + t2);
#pragma unroll
    for (int e = 0; e < KPT; ++e) fft_any<N2>(y[e]);
    __syncwarp();
    if (FWD) {
        // natural order into the scratch, then split into the two real lines
#pragma unroll
        for (int e = 0; e < KPT; ++e)
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) SC(t * KPT + e + N1 * k2) = y[e][k2];
        __syncwarp();
        constexpr int KU = H / N2 + 1;
        CX<T> zk[KU], zn[KU];
#pragma unroll
        for (int j = 0; j < KU; ++j) {
            const int k = t + N2 * j;
            if (k <= H) {
                zk[j] = SC(k);
                zn[j] = SC(k == 0 ? 0 : N - k);
            }
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < KU; ++j) {
            const int k = t + N2 * j;
            if (k <= H) {
                P[EL(k)] = T(0.5) * (zk[j].x + zn[j].x) * scale;
                P[EL(k) + g.bo] = T(0.5) * (zk[j].y + zn[j].y) * scale;
                if (k > 0 && k < H) {
                    P[EL(N - k)] = T(0.5) * (zk[j].y - zn[j].y) * scale;
                    P[EL(N - k) + g.bo] = T(0.5) * (zn[j].x - zk[j].x) * scale;
                }
            }
        }
    } else {
#pragma unroll
        for (int e = 0; e < KPT; ++e)
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) {
                const int k = t * KPT + e + N1 * k2;
                P[EL(k)] = y[e][k2].x * scale;
                P[EL(k) + g.bo] = -y[e][k2].y * scale;
            }
    }
    __syncwarp();
}

struct PlaneBatch {
    const void* in[MAXF];
    void* out[MAXF];
    const double2* tw;   // exp(-2 pi i m / n)
    int ny, nzh;
    double scale;        // 1 / sqrt(n), applied per pass
};

// fftxyp2s (FWD: y then x) / fftxys2p (x then y) of plane z = blockIdx.x of
// field blockIdx.y, rows z = 0 .. nz.
template <int N, bool FWD, class TI, class TO, class TC>
__global__ void __launch_bounds__((N / 2) * Radix<N>::N2) k_fft_plane(PlaneBatch B) {
    constexpr int S = N + 2, N2 = Radix<N>::N2;
    extern __shared__ __align__(16) unsigned char smraw[];
    TC* P = reinterpret_cast<TC*>(smraw);
    __shared__ CX<TC> tw[N];
    const int z = blockIdx.x;
    const TI* in = static_cast<const TI*>(B.in[blockIdx.y]);
    TO* out = static_cast<TO*>(B.out[blockIdx.y]);
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = cx<TC>((TC)B.tw[i].x, (TC)B.tw[i].y);
    // With z fastest in memory every element of the plane is a separate
    // sector: each thread issues U independent loads before it stores any of
    // them, so that a CTA keeps NT * U loads in flight.
    constexpr int NT = (N / 2) * N2, IT = N * N / NT, U = IT < 16 ? IT : 16;
    static_assert(IT * NT == N * N && IT % U == 0, "plane load batches");
    for (int b = 0; b < IT; b += U) {
        TI r[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int idx = threadIdx.x + (b + u) * NT, ix = idx / N, iy = idx - ix * N;
            r[u] = in[((long long)ix * B.ny + iy) * B.nzh + 1 + z];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int idx = threadIdx.x + (b + u) * NT, ix = idx / N, iy = idx - ix * N;
            P[ix * S + iy] = (TC)r[u];
        }
    }
    __syncthreads();
    const int line = threadIdx.x / N2, t = threadIdx.x - line * N2;
    // y lines: rows 2p, 2p+1; x lines: columns 2q, 2q+1 (complex pairs)
    const LineGeo gy = {2 * line * S, 1, S, 2 * line * S, 2};
    const LineGeo gx = {2 * line, S, 1, 2 * line, S};
    const TC scale = (TC)B.scale;
    if (FWD) {
        line_fft<N, true, TC>(P, gy, t, tw, scale);
        __syncthreads();
        line_fft<N, true, TC>(P, gx, t, tw, scale);
    } else {
        line_fft<N, false, TC>(P, gx, t, tw, scale);
        __syncthreads();
        line_fft<N, false, TC>(P, gy, t, tw, scale);
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < IT; ++k) {
        const int idx = threadIdx.x + k * NT, ix = idx / N, iy = idx - ix * N;
        out[((long long)ix * B.ny + iy) * B.nzh + 1 + z] = (TO)P[ix * S + iy];
    }
}

// Compute type of a transform: FP32 when either side is FP32 (mixed form).
template <class TI, class TO>
using TCmp = typename std::conditional<std::is_same<TI, float>::value || std::is_same<TO, float>::value, float,
                                       double>::type;

template <int N, class TI, class TO>
static void launch_plane(Ctx& c, const TI* const* in, TO* const* out, int nf, bool forward) {
    using TC = TCmp<TI, TO>;
    constexpr int S = N + 2;
    PlaneBatch B;
    for (int f = 0; f < nf; ++f) { B.in[f] = in[f]; B.out[f] = out[f]; }
    B.tw = c.px.tw;
    B.ny = c.P.ny;
    B.nzh = c.P.nzh;
    B.scale = 1.0 / std::sqrt((double)N);
    size_t sm = sizeof(TC) * (size_t)N * S;
    dim3 grid(c.P.nz + 1, nf);
    int threads = (N / 2) * Radix<N>::N2;
    prof_begin(c, "fft");
    if (forward) {
        allow_smem(k_fft_plane<N, true, TI, TO, TC>, sm);
        k_fft_plane<N, true, TI, TO, TC><<<grid, threads, sm, c.stream>>>(B);
    } else {
        allow_smem(k_fft_plane<N, false, TI, TO, TC>, sm);
        k_fft_plane<N, false, TI, TO, TC><<<grid, threads, sm, c.stream>>>(B);
    }
    CKL();
    prof_end(c, "fft");
}

// Tiled line FFT along x (axis 0) or y (axis 1) for power-of-two lengths
// n = 16 .. 512.  A CTA holds TL consecutive z-lines (TL a multiple of 16 for
// FP64, of 32 for FP32, chosen per grid by tile_lines_for) of one y (or x)
// index in shared memory as P[l * S + e], S = n + 1, and transforms them as
// TL/2 complex line pairs (lines 2p, 2p+1) with line_fft.  The mappings keep
// every shared access of a warp at its minimum number of wavefronts:
//  * Loads and stores: a warp takes LB consecutive lines x 32/LB elements
//    (LB = 16 for 8-byte words, 32 for 4-byte words), so a global access
//    covers 128-byte runs of z, and with S odd the LB lines fall into LB
//    different banks (bank pairs).
//  * Line pairs: the L = n2 lanes of a pair read L consecutive elements of
//    its lines, so the pairs that share a wavefront are placed at element
//    offsets 2 p S that differ by 32 / (pairs per wavefront) banks
//    (tile_pair); S = n + 1 with n >= 16 a power of two satisfies
//    S = 1 (mod 8), which those offsets need.
//  * Each thread issues its 2 n1 loads in batches before storing any of them.
constexpr int TLMAX = 64;

// Line pair of lane group g (lanes g L .. g L + L - 1) of warp w.
template <int L, int WB>
EPIC_DEV int tile_pair(int w, int g) {
    if (WB == 8) {
        // a wavefront serves a half-warp: its pairs 16 (L = 8) or 8 (L = 4) banks apart
        if (L >= 16) return w * (32 / L) + g;
        if (L == 8) return 8 * (w >> 1) + 2 * (w & 1) + 4 * (g & 1) + (g >> 1);
        return 8 * w + 2 * (g & 3) + (g >> 2);
    }
    // 4-byte words: the pairs of a warp 32 / (32 / L) banks apart for the
    // element reads, and those of each half-warp 16 banks apart for the
    // 8-byte complex scratch
    if (L >= 16) return 16 * (w >> 3) + (w & 7) + 8 * g;
    if (L == 8) return 16 * (w >> 2) + (w & 3) + 4 * (((g & 1) << 1) | (g >> 1));
    return 16 * (w >> 1) + (w & 1) + 2 * (2 * (g & 3) + (g >> 2));
}

template <int N, bool FWD, class TI, class TO, class TC>
__global__ void __launch_bounds__((TLMAX / 2) * Radix<N>::N2) k_fft_tile(FFTBatch B) {
    constexpr int S = N + 1, L = Radix<N>::N2, IT = 2 * Radix<N>::N1, U = IT < 8 ? IT : 8;
    constexpr int WB = sizeof(TC), LB = WB == 8 ? 16 : 32, EB = 32 / LB;
    static_assert(L == 4 || L == 8 || L == 16, "lanes per line pair");
    static_assert(S % 8 == 1, "row stride");
    extern __shared__ __align__(16) unsigned char smraw[];
    TC* P = reinterpret_cast<TC*>(smraw);
    __shared__ CX<TC> tw[N];
    const TI* in = static_cast<const TI*>(B.in[blockIdx.z]);
    TO* out = static_cast<TO*>(B.out[blockIdx.z]);
    const int TL = B.T, l0 = blockIdx.x * TL, lb = TL / LB;
    const long long rowbase = (long long)blockIdx.y * B.row_stride + 1;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = cx<TC>((TC)B.tw[i].x, (TC)B.tw[i].y);
    // Blocks b = w + k nw of LB lines x EB elements: lines LB (b mod lb) +
    // lane mod LB, elements EB (b / lb) + lane / LB.  nw is a multiple of lb
    // (nw / lb = L LB / 64), so a thread keeps its line and steps its element
    // by DE = EB L LB / 64 = L / 2.
    const int l = LB * (w % lb) + lane % LB, e0 = EB * (w / lb) + lane / LB;
    constexpr int DE = L / 2;
    const bool live = l0 + l < B.nl;
    const TI* src = in + rowbase + l0 + l + (long long)e0 * B.es;
    const long long step = (long long)DE * B.es;
    TC* dst = P + l * S + e0;
    for (int k0 = 0; k0 < IT; k0 += U) {
        TI r[U];
#pragma unroll
        for (int u = 0; u < U; ++u) r[u] = live ? src[(k0 + u) * step] : TI(0);
#pragma unroll
        for (int u = 0; u < U; ++u) dst[(k0 + u) * DE] = (TC)r[u];
    }
    __syncthreads();
    const int pair = tile_pair<L, WB>(w, lane / L), t = lane & (L - 1);
    const LineGeo g = {2 * pair * S, 1, S, 2 * pair * S, 2};
    line_fft<N, FWD, TC>(P, g, t, tw, (TC)B.scale);
    __syncthreads();
    if (live) {
        TO* o = out + rowbase + l0 + l + (long long)e0 * B.es;
#pragma unroll 8
        for (int k = 0; k < IT; ++k) o[k * step] = (TO)dst[k * DE];
    }
}

// z-lines per tile: the multiple of 16 (FP64) or 32 (FP32), up to 64, that
// pads nl least, the larger on a tie, with the tile under 100 KB of shared
// memory.
static int tile_lines_for(int nl, int n, size_t elem) {
    const int m = elem == 8 ? 16 : 32;
    int best = m;
    long long best_pad = LLONG_MAX;
    for (int tl = m; tl <= TLMAX; tl += m) {
        if (tl > m && elem * (size_t)tl * (n + 1) > 100 * 1024) break;
        const long long pad = (long long)((nl + tl - 1) / tl) * tl;
        if (pad <= best_pad) { best_pad = pad; best = tl; }
    }
    return best;
}

template <int N, class TI, class TO>
static void launch_tile_axis(Ctx& c, const FFTPlan& pl, int axis, const TI* const* in, TO* const* out,
                             int nf, bool forward) {
    using TC = TCmp<TI, TO>;
    const Params& P = c.P;
    FFTBatch B;
    for (int f = 0; f < nf; ++f) { B.in[f] = in[f]; B.out[f] = out[f]; }
    B.n = N;
    B.tw = pl.tw;
    B.nl = P.nz + 1;
    B.T = tile_lines_for(B.nl, N, sizeof(TC));
    B.scale = 1.0 / std::sqrt((double)N);
    int nrows;
    if (axis == 0) { B.es = (long long)P.ny * P.nzh; B.row_stride = P.nzh; nrows = P.ny; }
    else { B.es = P.nzh; B.row_stride = (long long)P.ny * P.nzh; nrows = P.nx; }
    size_t sm = sizeof(TC) * (size_t)B.T * (N + 1);
    dim3 grid((B.nl + B.T - 1) / B.T, nrows, nf);
    int threads = (B.T / 2) * Radix<N>::N2;
    prof_begin(c, "fft");
    if (forward) {
        allow_smem(k_fft_tile<N, true, TI, TO, TC>, sm);
        k_fft_tile<N, true, TI, TO, TC><<<grid, threads, sm, c.stream>>>(B);
    } else {
        allow_smem(k_fft_tile<N, false, TI, TO, TC>, sm);
        k_fft_tile<N, false, TI, TO, TC><<<grid, threads, sm, c.stream>>>(B);
    }
    CKL();
    prof_end(c, "fft");
}

template <class TI, class TO>
static bool tile_axis(Ctx& c, const FFTPlan& pl, int axis, const TI* const* in, TO* const* out, int nf,
                      bool forward) {
    switch (pl.n) {
        case 16: launch_tile_axis<16>(c, pl, axis, in, out, nf, forward); return true;
        case 48: launch_tile_axis<48>(c, pl, axis, in, out, nf, forward); return true;
        case 96: launch_tile_axis<96>(c, pl, axis, in, out, nf, forward); return true;
        case 32: launch_tile_axis<32>(c, pl, axis, in, out, nf, forward); return true;
        case 64: launch_tile_axis<64>(c, pl, axis, in, out, nf, forward); return true;
        case 128: launch_tile_axis<128>(c, pl, axis, in, out, nf, forward); return true;
        case 256: launch_tile_axis<256>(c, pl, axis, in, out, nf, forward); return true;
        case 512: launch_tile_axis<512>(c, pl, axis, in, out, nf, forward); return true;
        default: return false;
    }
}

// Half-plane 2-D FFT: a cluster of two CTAs per (z plane, field), each with
// half of the plane in shared memory (n/2 rows of n + 2), so that two or
// three planes are in flight per SM.  Forward: CTA r loads the rows
// x in [r n/2, (r+1) n/2), transforms its y lines, then the two CTAs swap
// the off-diagonal quarter blocks through distributed shared memory, after
// which CTA r holds every x of the spectral columns ky in [r n/2, (r+1) n/2)
// -- element (x, ky) at row x mod n/2, column (x / (n/2)) n/2 + ky mod n/2 --
// and transforms its x lines.  Inverse: the same steps in reverse order (the
// swap is its own inverse).
namespace cgr = cooperative_groups;

template <int N, bool FWD, class TI, class TO, class TC>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__((N / 4) * Radix<N>::N2) k_fft_half(PlaneBatch B) {
    constexpr int H = N / 2, S = N + 2, N2 = Radix<N>::N2, NT = (H / 2) * N2;
    constexpr int LH = H == 64 ? 6 : H == 32 ? 5 : H == 16 ? 4 : 3;
    static_assert((1 << LH) == H, "half size");
    extern __shared__ __align__(16) unsigned char smraw[];
    TC* P = reinterpret_cast<TC*>(smraw);
    __shared__ CX<TC> tw[N];
    cgr::cluster_group cl = cgr::this_cluster();
    const int r = (int)cl.block_rank();
    const int z = blockIdx.x >> 1;
    const TI* in = static_cast<const TI*>(B.in[blockIdx.y]);
    TO* out = static_cast<TO*>(B.out[blockIdx.y]);
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = cx<TC>((TC)B.tw[i].x, (TC)B.tw[i].y);
    const int line = threadIdx.x / N2, t = threadIdx.x - line * N2;
    const LineGeo gy = {2 * line * S, 1, S, 2 * line * S, 2};
    LineGeo gx = {2 * line, S, 1, 2 * line, S};
    gx.msk = H - 1;
    gx.sh = LH;
    gx.es2 = H;
    const TC scale = (TC)B.scale;
    auto swap_quarters = [&]() {
        constexpr int PER = H * H / NT;
        cl.sync();   // both CTAs finished the first pass
        const TC* peer = cl.map_shared_rank(P, r ^ 1);
        TC v[PER];
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int idx = threadIdx.x + k * NT;
            const int xl = idx >> LH, c = idx & (H - 1);
            v[k] = peer[xl * S + H * r + c];
        }
        cl.sync();   // both CTAs read their peer's block
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int idx = threadIdx.x + k * NT;
            const int xl = idx >> LH, c = idx & (H - 1);
            P[xl * S + H * (1 - r) + c] = v[k];
        }
        __syncthreads();
    };
    if (FWD) {
        for (int idx = threadIdx.x; idx < H * N; idx += NT) {
            const int xl = idx / N, y = idx - xl * N;
            P[xl * S + y] = (TC)in[((long long)(H * r + xl) * B.ny + y) * B.nzh + 1 + z];
        }
        __syncthreads();
        line_fft<N, true, TC>(P, gy, t, tw, scale);
        swap_quarters();
        line_fft<N, true, TC>(P, gx, t, tw, scale);
        __syncthreads();
        for (int idx = threadIdx.x; idx < N * H; idx += NT) {
            const int x = idx >> LH, c = idx & (H - 1);
            out[((long long)x * B.ny + H * r + c) * B.nzh + 1 + z] = (TO)P[(x & (H - 1)) * S + H * (x >> LH) + c];
        }
    } else {
        for (int idx = threadIdx.x; idx < N * H; idx += NT) {
            const int x = idx >> LH, c = idx & (H - 1);
            P[(x & (H - 1)) * S + H * (x >> LH) + c] = (TC)in[((long long)x * B.ny + H * r + c) * B.nzh + 1 + z];
        }
        __syncthreads();
        line_fft<N, false, TC>(P, gx, t, tw, scale);
        swap_quarters();
        line_fft<N, false, TC>(P, gy, t, tw, scale);
        __syncthreads();
        for (int idx = threadIdx.x; idx < H * N; idx += NT) {
            const int xl = idx / N, y = idx - xl * N;
            out[((long long)(H * r + xl) * B.ny + y) * B.nzh + 1 + z] = (TO)P[xl * S + y];
        }
    }
}

template <int N, class TI, class TO>
static void launch_half(Ctx& c, const TI* const* in, TO* const* out, int nf, bool forward) {
    using TC = TCmp<TI, TO>;
    constexpr int S = N + 2;
    PlaneBatch B;
    for (int f = 0; f < nf; ++f) { B.in[f] = in[f]; B.out[f] = out[f]; }
    B.tw = c.px.tw;
    B.ny = c.P.ny;
    B.nzh = c.P.nzh;
    B.scale = 1.0 / std::sqrt((double)N);
    size_t sm = sizeof(TC) * (size_t)(N / 2) * S;
    dim3 grid(2 * (c.P.nz + 1), nf);
    int threads = (N / 4) * Radix<N>::N2;
    prof_begin(c, "fft");
    if (forward) {
        allow_smem(k_fft_half<N, true, TI, TO, TC>, sm);
        k_fft_half<N, true, TI, TO, TC><<<grid, threads, sm, c.stream>>>(B);
    } else {
        allow_smem(k_fft_half<N, false, TI, TO, TC>, sm);
        k_fft_half<N, false, TI, TO, TC><<<grid, threads, sm, c.stream>>>(B);
    }
    CKL();
    prof_end(c, "fft");
}

// Half-plane cluster kernel sizes: square n x n grids with n = 64, 128.
template <class TI, class TO>
static bool half_fft(Ctx& c, const TI* const* in, TO* const* out, int nf, bool forward) {
    const Params& P = c.P;
    if (P.nx != P.ny) return false;
    switch (P.nx) {
        case 64: launch_half<64>(c, in, out, nf, forward); return true;
        case 128: launch_half<128>(c, in, out, nf, forward); return true;
        default: return false;
    }
}

// Plane kernel sizes: square n x n grids with n = 16, 32, 64, 128.
template <class TI, class TO>
static bool plane_fft(Ctx& c, const TI* const* in, TO* const* out, int nf, bool forward) {
    const Params& P = c.P;
    if (P.nx != P.ny) return false;
    switch (P.nx) {
        case 16: launch_plane<16>(c, in, out, nf, forward); return true;
        case 32: launch_plane<32>(c, in, out, nf, forward); return true;
        case 64: launch_plane<64>(c, in, out, nf, forward); return true;
        case 128: launch_plane<128>(c, in, out, nf, forward); return true;
        default: return false;
    }
}

static void make_plan(FFTPlan& p, int n, cudaStream_t st) {
    p.n = n;
    p.nfac = 0;
    int rem = n;
    for (int f : {4, 2, 3, 5})
        while (rem % f == 0) { p.fac[p.nfac++] = f; rem /= f; }
    if (rem != 1 || n % 2 != 0)
        throw CudaError(EPIC_ERR_CONFIG, "horizontal grid sizes must be even and factor into 2, 3, 5");
    std::vector<double2> tw(n);
    for (int m = 0; m < n; ++m) {
        double a = -2.0 * M_PI * (double)m / (double)n;
        tw[m] = make_double2(std::cos(a), std::sin(a));
    }
    CK(cudaMalloc(&p.tw, sizeof(double2) * n));
    CK(cudaMemcpyAsync(p.tw, tw.data(), sizeof(double2) * n, cudaMemcpyHostToDevice, st));
}

static int tile_lines(int n) {
    int T = 4096 / n;
    T = std::max(2, std::min(32, T));
    return T & ~1;
}

template <class TI, class TO>
static void run_fft_axis(Ctx& c, const FFTPlan& pl, int axis, const TI* const* in,
                         TO* const* out, int nf, bool forward) {
    const Params& P = c.P;
    FFTBatch B;
    for (int f = 0; f < nf; ++f) { B.in[f] = in[f]; B.out[f] = out[f]; }
    B.n = pl.n;
    B.nfac = pl.nfac;
    for (int k = 0; k < 16; ++k) B.fac[k] = pl.fac[k];
    B.tw = pl.tw;
    B.nl = P.nz + 1;
    B.T = tile_lines(pl.n);
    B.scale = 1.0 / std::sqrt((double)pl.n);
    int nrows;
    if (axis == 0) { B.es = (long long)P.ny * P.nzh; B.row_stride = P.nzh; nrows = P.ny; }
    else { B.es = P.nzh; B.row_stride = (long long)P.ny * P.nzh; nrows = P.nx; }
    size_t sm = sizeof(double) * (size_t)B.T * B.n + 2 * sizeof(double2) * (size_t)(B.T / 2) * B.n +
                sizeof(double2) * B.n;
    dim3 grid((B.nl + B.T - 1) / B.T, nrows, nf);
    prof_begin(c, "fft");
    if (forward) {
        allow_smem(k_fft_lines<true, TI, TO>, sm);
        k_fft_lines<true, TI, TO><<<grid, 256, sm, c.stream>>>(B);
        CKL();
    } else {
        allow_smem(k_fft_lines<false, TI, TO>, sm);
        k_fft_lines<false, TI, TO><<<grid, 256, sm, c.stream>>>(B);
        CKL();
    }
    prof_end(c, "fft");
}

// fftxyp2s: y then x (forward); fftxys2p: x then y (reverse).  Only rows
// z = 0 .. nz are read and written.
// The first pass reads TI and writes TO; the second runs in place on TO.
template <class TI, class TO>
void fft_xy(Ctx& c, const TI* const* in, TO* const* out, int nf, bool forward) {
    for (int f0 = 0; f0 < nf; f0 += MAXF) {
        int k = std::min(MAXF, nf - f0);
        if (c.fft_path == 3 && half_fft(c, in + f0, out + f0, k, forward)) continue;
        if ((c.fft_path == 0 || c.fft_path == 3) && plane_fft(c, in + f0, out + f0, k, forward)) continue;
        // per axis: tiled register FFT for powers of two up to 256, else Stockham lines
        auto axis = [&](const FFTPlan& pl, int ax, auto src, TO* const* dst, bool fwd) {
            if (c.fft_path <= 1 && tile_axis(c, pl, ax, src, dst, k, fwd)) return;
            run_fft_axis(c, pl, ax, src, dst, k, fwd);
        };
        const TO* const* oc = const_cast<const TO* const*>(out + f0);
        if (forward) {
            axis(c.py, 1, in + f0, out + f0, true);
            axis(c.px, 0, oc, out + f0, true);
        } else {
            axis(c.px, 0, in + f0, out + f0, false);
            axis(c.py, 1, oc, out + f0, false);
        }
    }
}

// ---------------------------------------------------------------------------
// Vertical (column) kernels.  A CTA holds 32 columns (kx, ky) of nz+1 values
// in shared memory as x[j * 34 + col] (rows 16-byte aligned); matrix-vector
// products with the DST-I / DCT-I matrices keep all 32 lanes busy on
// different columns.
constexpr int CT = 32;
constexpr int CP = 34;

struct ColArgs {
    const double* tab[8];
    const void* in[4];      // element type T of the kernel
    void* out[4];
    const void* mdst;       // (nz+1)^2 matrices in T
    const void* mdct;
    const void* qdst;       // quarter tables in T (even nz), null: full matrices
    const void* qdct;
    int qld_dst, qld_dct;
    int ncol;      // nx * ny
    int nz;
    int nzh;
    double dzi, hdzi;
    double sn;     // sqrt(2 / nz)
};

// Symmetric z transforms (even n = nz, h = n / 2).  The DST-I matrix
// M[k][j] = sn sin(pi k j / n) (rows, columns 1 .. n-1) and the DCT-I matrix
// C[k][j] = sn w_j cos(pi k j / n) (0 .. n, w_0 = w_n = 1/2) satisfy
//   M[k][n-j] = (-1)^(k+1) M[k][j],  M[n-k][j] = (-1)^(j+1) M[k][j],
//   C[k][n-j] = (-1)^k C[k][j],      C[n-k][j] = (-1)^j C[k][j].
// So with S[j] = x[j] + x[n-j], D[j] = x[j] - x[n-j] (j < h), for k < h
//   Y[k]   = E + O + mid,   E, O = sums over even, odd j < h of Q[k][j] V[j],
//   Y[n-k] = O - E + (-1)^(h+1) mid (DST),  E - O + (-1)^h mid (DCT),
// mid = Q[k][h] x[h] and V = S for odd k (DST) / even k (DCT), else D; row h
// is a signed sum of every other x.  A quarter of the multiply-adds of the
// full matrix, from a table Q of (h - j0 + 1) x qld values: rows of the
// S-parity first (padded to 8), then the others (padded to 8).
// KIND 0: DST over rows 1 .. n-1; KIND 1: DCT over rows 0 .. n.  The pairs
// of x are formed in place (x is consumed; rows 0 and n of a DST input and
// row h are kept); ADD accumulates into y.  All threads of the CTA call it.
template <int KIND>
struct ZT {
    static constexpr int j0 = KIND == 0 ? 1 : 0;
    // rows of the two parity blocks below h and their k
    static EPIC_HD int nA(int h) { return KIND == 0 ? h / 2 : (h + 1) / 2; }
    static EPIC_HD int nB(int h) { return KIND == 0 ? (h - 1) / 2 : h / 2; }
    static EPIC_HD int kA(int i) { return KIND == 0 ? 2 * i + 1 : 2 * i; }
    static EPIC_HD int kB(int i) { return KIND == 0 ? 2 * i + 2 : 2 * i + 1; }
    static EPIC_HD int qld(int h) { return 8 * ((nA(h) + 7) / 8 + (nB(h) + 7) / 8); }
};

template <class T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

template <int KIND, bool ADD, class T>
EPIC_DEV void col_ztransform(const T* __restrict__ Q, int qld, T* xs, T* ys, int n, T sn) {
    using Z = ZT<KIND>;
    using V2 = typename Vec2<T>::type;
    constexpr int j0 = Z::j0;
    const int h = n / 2;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
    // row h: a signed sum of every other x (one thread per column)
    T yh = T(0);
    if (tid < CT) {
        if (KIND == 0) {
            for (int j = 1; j < n; j += 2) yh += ((j >> 1) & 1) ? -xs[j * CP + tid] : xs[j * CP + tid];
        } else {
            yh = T(0.5) * (xs[tid] + (((n >> 1) & 1) ? -xs[n * CP + tid] : xs[n * CP + tid]));
            for (int j = 2; j < n; j += 2) yh += ((j >> 1) & 1) ? -xs[j * CP + tid] : xs[j * CP + tid];
        }
        yh *= sn;
    }
    __syncthreads();
    // pairs in place: S[j] at row j, D[j] at row n - j
    const int np = h - j0;
    for (int idx = tid; idx < CT * np; idx += blockDim.x) {
        const int col = idx & (CT - 1), j = j0 + (idx >> 5);
        const T a = xs[j * CP + col], b = xs[(n - j) * CP + col];
        xs[j * CP + col] = a + b;
        xs[(n - j) * CP + col] = a - b;
    }
    __syncthreads();
    if (tid < CT) {
        T* o = ys + h * CP + tid;
        *o = ADD ? *o + yh : yh;
    }
    // octets of rows: 8 rows x 32 columns per warp; a lane owns 2 rows and
    // the columns {2c, 2c+1, 16+2c, 17+2c}, so that each 2-wide load of the
    // 8 lanes of a row group covers 128 contiguous bytes
    const int nA = Z::nA(h), nB = Z::nB(h), oA = (nA + 7) / 8, oB = (nB + 7) / 8;
    const int rl = lane >> 3, cl = lane & 7;
    const int c0 = 2 * cl, c1 = 16 + 2 * cl;
    const T sE = KIND == 0 ? T(-1) : T(1), sO = -sE;
    const T sM = ((h & 1) ^ (KIND == 0 ? 1 : 0)) ? T(-1) : T(1);   // (-1)^(h+1) DST, (-1)^h DCT
    for (int oct = warp; oct < oA + oB; oct += nwarp) {
        const bool blockA = oct < oA;
        const int ib = 8 * (blockA ? oct : oct - oA) + 2 * rl;          // row in its block
        const int iq = blockA ? ib : 8 * oA + ib;                      // row in Q
        const int nrows = blockA ? nA : nB;
        // V rows: S at j (block A), D at n - j (block B)
        const T* v = xs + (blockA ? j0 : n - j0) * CP;
        const int vstep = blockA ? CP : -CP;
        const T* q = Q + iq;
        T e[2][4], o[2][4];
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) { e[r][c] = T(0); o[r][c] = T(0); }
        auto step = [&](T (&acc)[2][4]) {
            const V2 qq = *reinterpret_cast<const V2*>(q);
            const V2 va = *reinterpret_cast<const V2*>(v + c0);
            const V2 vb = *reinterpret_cast<const V2*>(v + c1);
            const T vv[4] = {va.x, va.y, vb.x, vb.y};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                acc[0][c] = fma(qq.x, vv[c], acc[0][c]);
                acc[1][c] = fma(qq.y, vv[c], acc[1][c]);
            }
            q += qld;
            v += vstep;
        };
        int j = j0;
#pragma unroll 2
        for (; j + 1 < h; j += 2) {
            if (j0 & 1) { step(o); step(e); }
            else { step(e); step(o); }
        }
        if (j < h) {
            if (j0 & 1) step(o);
            else step(e);
        }
        // q now points at row j = h: the coefficients of x[h]
        const V2 qm = *reinterpret_cast<const V2*>(Q + (h - j0) * qld + iq);
        const T cm[2] = {qm.x, qm.y};
        const int cols[4] = {c0, c0 + 1, c1, c1 + 1};
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            if (ib + r >= nrows) continue;
            const int k = blockA ? Z::kA(ib + r) : Z::kB(ib + r);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const T mid = cm[r] * xs[h * CP + cols[c]];
                const T y1 = e[r][c] + o[r][c] + mid;
                const T y2 = sE * e[r][c] + sO * o[r][c] + sM * mid;
                T* p1 = ys + k * CP + cols[c];
                T* p2 = ys + (n - k) * CP + cols[c];
                *p1 = ADD ? *p1 + y1 : y1;
                *p2 = ADD ? *p2 + y2 : y2;
            }
        }
    }
}

// Element-wise work over the CTA's columns (256 threads): 8 threads per
// column on consecutive z, so that global accesses run along z and the 16
// lanes of a half-warp (2 columns x 8 rows, row stride CP = 34) hit 16
// different bank pairs; no index division.
static_assert(CT * 8 == 256, "column kernels run 256 threads");
template <class F>
EPIC_DEV void col_each(int nzp, F&& f) {
    const int col = threadIdx.x >> 3;
    for (int j = threadIdx.x & 7; j < nzp; j += 8) f(col, j);
}
template <class T>
EPIC_DEV void col_load(const T* f, T* xs, int c0, const ColArgs& A) {
    const int c = c0 + (threadIdx.x >> 3);
    const bool ok = c < A.ncol;
    const T* src = f + (long long)c * A.nzh + 1;
    col_each(A.nz + 1, [&](int col, int j) { xs[j * CP + col] = ok ? src[j] : T(0); });
}
template <class T>
EPIC_DEV void col_store(T* f, const T* xs, int c0, const ColArgs& A) {
    const int c = c0 + (threadIdx.x >> 3);
    if (c >= A.ncol) return;
    T* dst = f + (long long)c * A.nzh + 1;
    col_each(A.nz + 1, [&](int col, int j) { dst[j] = xs[j * CP + col]; });
}
// table value for (column c, z = j)
EPIC_DEV double tabv(const double* t, int c, int j, const ColArgs& A) {
    return t[(long long)c * A.nzh + 1 + j];
}
// ys[k] = sum_{j=lo..hi} M[k][j] xs[j] for k = lo..hi (M row-major (nz+1)^2),
// all 32 columns of a CTA (256 threads), register tiled: thread (rg, cg)
// computes rows lo + rg + 32 r (r < R) of columns 4 cg .. 4 cg + 3, 20 FMAs
// per 9 loads.  ADD accumulates into ys instead of overwriting.
template <int R, bool ADD, class T>
EPIC_DEV void col_matvec_t(const T* __restrict__ M, int lo, int hi, const T* xs, T* ys, int nz) {
    const int nzp = nz + 1;
    const int cg = threadIdx.x & 7, rg = threadIdx.x >> 3;
    T acc[R][4];
    int krow[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        krow[r] = min(lo + rg + 32 * r, hi) * nzp;
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[r][q] = T(0);
    }
    for (int j = lo; j <= hi; ++j) {
        const T* xr = xs + j * CP + 4 * cg;
        T x0 = xr[0], x1 = xr[1], x2 = xr[2], x3 = xr[3];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            T m = __ldg(M + krow[r] + j);
            acc[r][0] = fma(m, x0, acc[r][0]);
            acc[r][1] = fma(m, x1, acc[r][1]);
            acc[r][2] = fma(m, x2, acc[r][2]);
            acc[r][3] = fma(m, x3, acc[r][3]);
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = lo + rg + 32 * r;
        if (k <= hi) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                T* o = ys + k * CP + 4 * cg + q;
                *o = ADD ? *o + acc[r][q] : acc[r][q];
            }
        }
    }
}

// field_decompose_semi_spectral (inversion_utils.f90:370-401), optionally
// followed by the Hou-Li filter and/or preceded by central_diffz_semi_spectral
// (inversion_utils.f90:460-480).  mode bit 1: filter, bit 2: central diff.
// CTAs per SM the column kernels are held to: up to 5 rows per thread (nz <
// 160) the FP64 columns (70 KB at nz = 128) fit three times and the FP32 ones
// four, at 80 and 64 registers; longer columns fill the shared memory alone.
template <int R, class T>
constexpr int col_min_blocks() { return R > 5 ? 1 : sizeof(T) == 8 ? 3 : 4; }

template <int R, class T>
__global__ void __launch_bounds__(256, col_min_blocks<R, T>()) k_col_decompose(ColArgs A, int mode) {
    extern __shared__ __align__(16) unsigned char smraw[];
    T* sm = reinterpret_cast<T*>(smraw);
    int nzp = A.nz + 1, nz = A.nz;
    T* xs = sm;
    T* ys = sm + nzp * CP;
    int c0 = blockIdx.x * CT;
    const double* phim = A.tab[0];
    const double* phip = A.tab[1];
    const double* filt = A.tab[2];
    col_load(static_cast<const T*>(A.in[blockIdx.y]), xs, c0, A);
    __syncthreads();
    if (mode & 2) {
        for (int idx = threadIdx.x; idx < CT * nzp; idx += blockDim.x) {
            int col = idx % CT, j = idx / CT;
            T v;
            if (j == 0) v = (T)A.dzi * (xs[1 * CP + col] - xs[col]);
            else if (j == nz) v = (T)A.dzi * (xs[nz * CP + col] - xs[(nz - 1) * CP + col]);
            else v = (xs[(j + 1) * CP + col] - xs[(j - 1) * CP + col]) * (T)A.hdzi;
            ys[j * CP + col] = v;
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < CT * nzp; idx += blockDim.x) xs[idx % CT + (idx / CT) * CP] = ys[idx % CT + (idx / CT) * CP];
        __syncthreads();
    }
    // subtract harmonic part (lanes along z: the per-column tables are read coalesced)
    col_each(nzp, [&](int col, int j) {
        if (j < 1 || j > nz - 1) return;
        const int c = min(c0 + col, A.ncol - 1);
        xs[j * CP + col] = xs[j * CP + col] - (xs[col] * (T)tabv(phim, c, j, A) + xs[nz * CP + col] * (T)tabv(phip, c, j, A));
    });
    __syncthreads();
    if (A.qdst) col_ztransform<0, false, T>(static_cast<const T*>(A.qdst), A.qld_dst, xs, ys, nz, (T)A.sn);
    else col_matvec_t<R, false, T>(static_cast<const T*>(A.mdst), 1, nz - 1, xs, ys, nz);
    for (int col = threadIdx.x; col < CT; col += blockDim.x) {
        ys[col] = xs[col];
        ys[nz * CP + col] = xs[nz * CP + col];
    }
    __syncthreads();
    if (mode & 1) {
        col_each(nzp, [&](int col, int j) {
            const int c = min(c0 + col, A.ncol - 1);
            ys[j * CP + col] = (T)tabv(filt, c, j, A) * ys[j * CP + col];
        });
        __syncthreads();
    }
    col_store(static_cast<T*>(A.out[blockIdx.y]), ys, c0, A);
}

// field_combine_semi_spectral (inversion_utils.f90:421-456)
template <int R, class T>
__global__ void __launch_bounds__(256, col_min_blocks<R, T>()) k_col_combine(ColArgs A) {
    extern __shared__ __align__(16) unsigned char smraw[];
    T* sm = reinterpret_cast<T*>(smraw);
    int nzp = A.nz + 1, nz = A.nz;
    T* xs = sm;
    T* ys = sm + nzp * CP;
    int c0 = blockIdx.x * CT;
    const double* phim = A.tab[0];
    const double* phip = A.tab[1];
    col_load(static_cast<const T*>(A.in[blockIdx.y]), xs, c0, A);
    __syncthreads();
    if (A.qdst) col_ztransform<0, false, T>(static_cast<const T*>(A.qdst), A.qld_dst, xs, ys, nz, (T)A.sn);
    else col_matvec_t<R, false, T>(static_cast<const T*>(A.mdst), 1, nz - 1, xs, ys, nz);
    __syncthreads();
    col_each(nzp, [&](int col, int j) {
        const int c = min(c0 + col, A.ncol - 1);
        T v;
        if (j == 0) v = xs[col];
        else if (j == nz) v = xs[nz * CP + col];
        else v = ys[j * CP + col] + xs[col] * (T)tabv(phim, c, j, A) + xs[nz * CP + col] * (T)tabv(phip, c, j, A);
        xs[j * CP + col] = v;
    });
    __syncthreads();
    col_store(static_cast<T*>(A.out[blockIdx.y]), xs, c0, A);
}

// Vertical-velocity solve of vor2vel (inversion.f90:97-150): in[0] = D
// (source) -> out[0] = w (semi-spectral), out[1] = dw/dz part es.
template <int R, class T>
__global__ void __launch_bounds__(256) k_col_wsolve(ColArgs A) {
    extern __shared__ __align__(16) unsigned char smraw[];
    T* sm = reinterpret_cast<T*>(smraw);
    int nzp = A.nz + 1, nz = A.nz;
    T* ds = sm;
    T* as = sm + nzp * CP;
    T* bs = sm + 2 * nzp * CP;
    T* es = sm + 3 * nzp * CP;
    int c0 = blockIdx.x * CT;
    const double* thetam = A.tab[0];
    const double* thetap = A.tab[1];
    const double* dthetam = A.tab[2];
    const double* dthetap = A.tab[3];
    const double* green = A.tab[4];
    const double* rkz = A.tab[5];
    col_load(static_cast<const T*>(A.in[0]), ds, c0, A);
    __syncthreads();
    col_each(nzp, [&](int col, int j) {
        const int c = min(c0 + col, A.ncol - 1);
        const T d0 = ds[col], dn = ds[nz * CP + col];
        if (j >= 1 && j <= nz - 1) bs[j * CP + col] = d0 * (T)tabv(thetam, c, j, A) + dn * (T)tabv(thetap, c, j, A);
        es[j * CP + col] = d0 * (T)tabv(dthetam, c, j, A) + dn * (T)tabv(dthetap, c, j, A);
    });
    __syncthreads();
    col_each(nzp, [&](int col, int j) {
        const int c = min(c0 + col, A.ncol - 1);
        if (j >= 1 && j <= nz - 1) {
            const T g = (T)tabv(green, c, j, A) * ds[j * CP + col];
            ds[j * CP + col] = g;
            as[j * CP + col] = (T)rkz[j] * g;
        } else {
            as[j * CP + col] = T(0);
        }
    });
    __syncthreads();
    // es += DCT(as); then as(1:nz-1) = DST(ds(1:nz-1))
    if (A.qdct) col_ztransform<1, true, T>(static_cast<const T*>(A.qdct), A.qld_dct, as, es, nz, (T)A.sn);
    else col_matvec_t<R, true, T>(static_cast<const T*>(A.mdct), 0, nz, as, es, nz);
    __syncthreads();
    if (A.qdst) col_ztransform<0, false, T>(static_cast<const T*>(A.qdst), A.qld_dst, ds, as, nz, (T)A.sn);
    else col_matvec_t<R, false, T>(static_cast<const T*>(A.mdst), 1, nz - 1, ds, as, nz);
    __syncthreads();
    for (int idx = threadIdx.x; idx < CT * nzp; idx += blockDim.x) {
        int col = idx % CT, j = idx / CT;
        ds[j * CP + col] = (j >= 1 && j <= nz - 1) ? as[j * CP + col] + bs[j * CP + col] : T(0);
    }
    __syncthreads();
    col_store(static_cast<T*>(A.out[0]), ds, c0, A);
    col_store(static_cast<T*>(A.out[1]), es, c0, A);
}

// ---------------------------------------------------------------------------
// Pointwise spectral kernels.  Element (kx, ky, iz), iz = 0 .. nz.
struct SpecArgs {
    const void* in[6];      // element type T of the kernel
    void* out[6];
    const double* k2l2i;
    const double* fdx;
    const double* fdy;
    const void* zbuf;      // (0,0)-column replacement values (2 x (nz+1)), T
    int nx, ny, nz, nzh;
    long long nel;         // nx * ny * (nz + 1)
};

struct SpecIdx {
    long long a;     // address of (kx, ky, iz)
    long long ax;    // address of (nx-kx, ky, iz)
    long long ay;    // address of (kx, ny-ky, iz)
    int kx, ky, iz;
};

EPIC_DEV SpecIdx spec_idx(const SpecArgs& S, long long i) {
    SpecIdx r;
    int nzp = S.nz + 1;
    long long c = i / nzp;
    r.iz = (int)(i - c * nzp);
    r.kx = (int)(c / S.ny);
    r.ky = (int)(c - (long long)r.kx * S.ny);
    int px = r.kx == 0 ? 0 : S.nx - r.kx;
    int py = r.ky == 0 ? 0 : S.ny - r.ky;
    r.a = ((long long)r.kx * S.ny + r.ky) * S.nzh + 1 + r.iz;
    r.ax = ((long long)px * S.ny + r.ky) * S.nzh + 1 + r.iz;
    r.ay = ((long long)r.kx * S.ny + py) * S.nzh + 1 + r.iz;
    return r;
}

// typed views of the kernel's untyped in/out pointers
#define IN(k) static_cast<const T*>(S.in[k])
#define OUT(k) static_cast<T*>(S.out[k])

#define SPEC_LOOP(S) for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (S).nel; \
                          i += (long long)gridDim.x * blockDim.x)

// out0 = Dx(in0) - Dy(in1)  (used for D = B_x - A_y and for the w source
// Dy(A) - Dx(B) with swapped signs via `sign`)
template <class T>
__global__ void k_spec_dxdy(SpecArgs S, double sx, double sy) {
    SPEC_LOOP(S) {
        SpecIdx q = spec_idx(S, i);
        OUT(0)[q.a] = (T)(sx * S.fdx[q.kx]) * IN(0)[q.ax] + (T)(sy * S.fdy[q.ky]) * IN(1)[q.ay];
    }
}

// svor_x = k2l2i (Dx(es) + Dy(ds)); svor_y = k2l2i (Dy(es) - Dx(ds));
// (0,0) column unchanged (inversion.f90:76-87).  in0 = es, in1 = ds.
template <class T>
__global__ void k_spec_project(SpecArgs S) {
    SPEC_LOOP(S) {
        SpecIdx q = spec_idx(S, i);
        if (q.kx == 0 && q.ky == 0) continue;
        T k2 = (T)S.k2l2i[(long long)q.kx * S.ny + q.ky];
        T fx = (T)S.fdx[q.kx], fy = (T)S.fdy[q.ky];
        T ex = fx * IN(0)[q.ax], ey = fy * IN(0)[q.ay];
        T dx = fx * IN(1)[q.ax], dy = fy * IN(1)[q.ay];
        OUT(0)[q.a] = k2 * (ex + dy);
        OUT(1)[q.a] = k2 * (ey - dx);
    }
}

// u = k2l2i (Dx(es) + Dy(cs)), v = k2l2i (Dy(es) - Dx(cs)); (0,0) = ubar, vbar
// (inversion.f90:180-226).  in0 = es, in1 = cs.
template <class T>
__global__ void k_spec_uv(SpecArgs S) {
    SPEC_LOOP(S) {
        SpecIdx q = spec_idx(S, i);
        if (q.kx == 0 && q.ky == 0) {
            OUT(0)[q.a] = static_cast<const T*>(S.zbuf)[q.iz];
            OUT(1)[q.a] = static_cast<const T*>(S.zbuf)[S.nz + 1 + q.iz];
            continue;
        }
        T k2 = (T)S.k2l2i[(long long)q.kx * S.ny + q.ky];
        T fx = (T)S.fdx[q.kx], fy = (T)S.fdy[q.ky];
        T ex = fx * IN(0)[q.ax], ey = fy * IN(0)[q.ay];
        T cx = fx * IN(1)[q.ax], cy = fy * IN(1)[q.ay];
        OUT(0)[q.a] = k2 * (ex + cy);
        OUT(1)[q.a] = k2 * (ey - cx);
    }
}

// velocity gradients (inversion.f90:259-290): in = u, v, w ->
// out = du/dx, du/dy, dw/dx, dv/dy, dw/dy
template <class T>
__global__ void k_spec_grad(SpecArgs S) {
    SPEC_LOOP(S) {
        SpecIdx q = spec_idx(S, i);
        T fx = (T)S.fdx[q.kx], fy = (T)S.fdy[q.ky];
        OUT(0)[q.a] = fx * IN(0)[q.ax];
        OUT(1)[q.a] = fy * IN(0)[q.ay];
        OUT(2)[q.a] = fx * IN(2)[q.ax];
        OUT(3)[q.a] = fy * IN(1)[q.ay];
        OUT(4)[q.a] = fy * IN(2)[q.ay];
    }
}

// vorticity tendency: out_c = Dx(Fx_c) + Dy(Fy_c), in = Fx0, Fy0, Fx1, Fy1, Fx2, Fy2
template <class T>
__global__ void k_spec_divxy(SpecArgs S) {
    SPEC_LOOP(S) {
        SpecIdx q = spec_idx(S, i);
        T fx = (T)S.fdx[q.kx], fy = (T)S.fdy[q.ky];
        for (int c = 0; c < 3; ++c)
            OUT(c)[q.a] = fx * IN(2 * c)[q.ax] + fy * IN(2 * c + 1)[q.ay];
    }
}

// diverge (inversion.f90:431-451): us = Dx(ds), vs = Dy(ds),
// ws = central_diffz_semi_spectral(ds) with ws(0) = ws(nz) = 0.
template <class T>
__global__ void k_spec_lapgrad(SpecArgs S, double hdzi) {
    SPEC_LOOP(S) {
        SpecIdx q = spec_idx(S, i);
        const T* d = IN(0);
        OUT(0)[q.a] = (T)S.fdx[q.kx] * d[q.ax];
        OUT(1)[q.a] = (T)S.fdy[q.ky] * d[q.ay];
        OUT(2)[q.a] = (q.iz == 0 || q.iz == S.nz) ? T(0) : (d[q.a + 1] - d[q.a - 1]) * (T)hdzi;
    }
}

// Mean flow (inversion.f90:158-176), one CTA: zbuf = (ubar, vbar).
template <class T>
__global__ void k_mean_flow(const T* svx, const T* svy, const double* rkzi, const double* gamtop,
                            const double* gambot, const double* mdct, T* zbuf, int nz) {
    extern __shared__ double sm[];
    double* u = sm;
    double* v = sm + nz + 1;
    for (int iz = threadIdx.x; iz <= nz; iz += blockDim.x) {
        bool in = iz >= 1 && iz <= nz - 1;
        u[iz] = in ? -rkzi[iz] * svy[1 + iz] : 0.0;
        v[iz] = in ? rkzi[iz] * svx[1 + iz] : 0.0;
    }
    __syncthreads();
    for (int k = threadIdx.x; k <= nz; k += blockDim.x) {
        const double* row = mdct + (long long)k * (nz + 1);
        double su = 0.0, sv = 0.0;
        for (int j = 0; j <= nz; ++j) { su = fma(row[j], u[j], su); sv = fma(row[j], v[j], sv); }
        zbuf[k] = (T)(su + (double)svy[1 + nz] * gamtop[k] - (double)svy[1] * gambot[k]);
        zbuf[nz + 1 + k] = (T)(sv - (double)svx[1 + nz] * gamtop[k] + (double)svx[1] * gambot[k]);
    }
}

// ---------------------------------------------------------------------------
// Physical-space helpers.  Element (ix, iy, iz) with iz = -1 .. nz+1.
struct PhysArgs {
    const double* in[8];
    double* out[8];
    int mode[8];
    int nf;
    int nx, ny, nz, nzh;
    long long ncol;
};

// z halo rows: mode 0 = linear extrapolation, 1 = anti-symmetry
__global__ void k_halo(PhysArgs A) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= A.ncol * A.nf) return;
    int f = (int)(t / A.ncol);
    long long c = t - (long long)f * A.ncol;
    double* p = A.out[f] + c * A.nzh + 1;
    int nz = A.nz;
    if (A.mode[f] == 0) {
        p[-1] = 2.0 * p[0] - p[1];
        p[nz + 1] = 2.0 * p[nz] - p[nz - 1];
    } else {
        p[-1] = -p[1];
        p[nz + 1] = -p[nz - 1];
    }
}

struct Ptr8 {
    const double* p[8];
};
struct MPtr8 {
    double* p[8];
};

// vel2vgrad tail (inversion.f90:308-312) over all rows incl. the halo rows.
__global__ void k_velgrad_fill(MPtr8 vg, Ptr8 vort, long long fsz) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < fsz;
         i += (long long)gridDim.x * blockDim.x) {
        vg.p[I_DUDZ][i] = vg.p[I_DWDX][i] + vort.p[1][i];
        vg.p[I_DVDX][i] = vg.p[I_DUDY][i] + vort.p[2][i];
        vg.p[I_DVDZ][i] = vg.p[I_DWDY][i] - vort.p[0][i];
    }
}

struct FluxArgs {
    const double* vort[3];
    const double* vel[3];
    const double* b;
    void* f[6];             // work arrays, element type T of the kernel
    double fc[3];
    int nx, ny, nz, nzh;
    long long nel;   // nx * ny * (nz+1)
};

// Flux products of vorticity_tendency (inversion.f90:327-348), rows 0..nz.
template <class T>
__global__ void k_flux(FluxArgs A) {
    int nzp = A.nz + 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < A.nel;
         i += (long long)gridDim.x * blockDim.x) {
        long long c = i / nzp;
        long long a = c * A.nzh + 1 + (i - c * nzp);
        double wx = A.vort[0][a] + A.fc[0], wy = A.vort[1][a] + A.fc[1];
        double b = A.b[a];
        double u = A.vel[0][a], v = A.vel[1][a], w = A.vel[2][a];
        T* const* f = reinterpret_cast<T* const*>(A.f);
        f[0][a] = (T)(wx * u);
        f[1][a] = (T)(wy * u + b);
        f[2][a] = (T)(wx * v - b);
        f[3][a] = (T)(wy * v);
        f[4][a] = (T)(wx * w);
        f[5][a] = (T)(wy * w);
    }
}

// vtend_c(0:nz) = divxy_c + central_diffz((zeta + f_z) u_c), with the zeta
// boundary zeroing (inversion.f90:374-384, inversion_utils.f90:485-510).
template <class T>
__global__ void k_vtend_rows(FluxArgs A, Ptr8 divxy, MPtr8 vt, double dzi, double hdzi, int z0, int z1) {
    int nzp = A.nz + 1, nz = A.nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < A.nel;
         i += (long long)gridDim.x * blockDim.x) {
        long long c = i / nzp;
        int iz = (int)(i - c * nzp);
        long long a = c * A.nzh + 1 + iz;
        const double* wz = A.vort[2];
        double fz = A.fc[2];
        for (int k = 0; k < 3; ++k) {
            const double* u = A.vel[k];
            double dz;
            if (iz == 0) dz = dzi * ((wz[a + 1] + fz) * u[a + 1] - (wz[a] + fz) * u[a]);
            else if (iz == nz) dz = dzi * ((wz[a] + fz) * u[a] - (wz[a - 1] + fz) * u[a - 1]);
            else dz = ((wz[a + 1] + fz) * u[a + 1] - (wz[a - 1] + fz) * u[a - 1]) * hdzi;
            double v = (double)reinterpret_cast<const T*>(divxy.p[k])[a] + dz;
            if (k == 2 && ((iz == 0 && z0) || (iz == nz && z1))) v = 0.0;
            vt.p[k][a] = v;
        }
    }
}

// lapinv1 (inversion_utils.f90:567-589): Thomas solve per (kx, ky) column;
// the (0,0) column is zero (inversion.f90:423-426, inversion_utils.f90:584-587).
// A CTA stages 32 columns of f and of the two tables in shared memory with
// coalesced loads; one warp then solves its 32 columns, one lane each.
template <class T>
EPIC_DEV void cols_load(const T* f, double* xs, int c0, int ncol, int nzp, int nzh) {
    const int c = c0 + (threadIdx.x >> 3);
    const bool ok = c < ncol;
    const T* src = f + (long long)c * nzh + 1;
    col_each(nzp, [&](int col, int j) { xs[j * CP + col] = ok ? (double)src[j] : 0.0; });
}

template <class T>
__global__ void __launch_bounds__(256) k_lapinv(T* fs, const double* etdv, const double* htdv, double ap,
                                               int ncol, int nz, int nzh) {
    extern __shared__ double sm[];
    const int nzp = nz + 1;
    double* f = sm;
    double* e = sm + nzp * CP;
    double* h = sm + 2 * nzp * CP;
    const int c0 = blockIdx.x * CT;
    cols_load(fs, f, c0, ncol, nzp, nzh);
    cols_load(etdv, e, c0, ncol, nzp, nzh);
    cols_load(htdv, h, c0, ncol, nzp, nzh);
    __syncthreads();
    if (threadIdx.x < CT) {
        const int col = threadIdx.x, c = c0 + col;
        if (c == 0) {
            for (int iz = 0; iz <= nz; ++iz) f[iz * CP + col] = 0.0;
        } else if (c < ncol) {
            double prev = f[col] * h[col];
            f[col] = prev;
            for (int iz = 1; iz <= nz - 1; ++iz) {
                prev = (f[iz * CP + col] - ap * prev) * h[iz * CP + col];
                f[iz * CP + col] = prev;
            }
            f[nz * CP + col] = (f[nz * CP + col] - 2.0 * ap * prev) * h[nz * CP + col];
            for (int iz = nz - 1; iz >= 0; --iz) f[iz * CP + col] = e[iz * CP + col] * f[(iz + 1) * CP + col] + f[iz * CP + col];
        }
    }
    __syncthreads();
    const int c = c0 + (threadIdx.x >> 3);
    if (c >= ncol) return;
    T* dst = fs + (long long)c * nzh + 1;
    col_each(nzp, [&](int col, int j) { dst[j] = (T)f[j * CP + col]; });
}

// phi = volg * vcelli - 1 (parcel_correction.f90:158)
__global__ void k_phi(const double* volg, double* phi, double vcelli, long long fsz) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < fsz;
         i += (long long)gridDim.x * blockDim.x)
        phi[i] = volg[i] * vcelli - 1.0;
}

// ---------------------------------------------------------------------------
// get_time_step reductions (rk_utils.f90:96-143)
__global__ void k_timestep_reduce(Params P, Ptr8 vg, const double* b, StepScalars* sc) {
    double gmax = 0.0, dbmax = 0.0;
    long long nel = (long long)P.nx * P.ny * (P.nz + 1);
    int nzp = P.nz + 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nel;
         i += (long long)gridDim.x * blockDim.x) {
        long long c = i / nzp;
        int iz = (int)(i - c * nzp);
        int ix = (int)(c / P.ny), iy = (int)(c - (long long)ix * P.ny);
        long long a = c * P.nzh + 1 + iz;
        double v[8];
#pragma unroll
        for (int l = 0; l < 8; ++l) v[l] = vg.p[l][a];
        double S[9];
        S[0] = v[I_DUDX];
        S[3] = 0.5 * (v[I_DUDY] + v[I_DVDX]);
        S[6] = 0.5 * (v[I_DUDZ] + v[I_DWDX]);
        S[1] = S[3];
        S[4] = v[I_DVDY];
        S[7] = 0.5 * (v[I_DVDZ] + v[I_DWDY]);
        S[2] = S[6];
        S[5] = S[7];
        S[8] = -(v[I_DUDX] + v[I_DVDY]);
        double D[3];
        sz_eigenvalues<FastOps>(S, D);
        gmax = fmax(gmax, fmax(fabs(D[0]), fmax(fabs(D[1]), fabs(D[2]))));
        int ixp = ix + 1 == P.nx ? 0 : ix + 1, ixm = ix == 0 ? P.nx - 1 : ix - 1;
        int iyp = iy + 1 == P.ny ? 0 : iy + 1, iym = iy == 0 ? P.ny - 1 : iy - 1;
        double gx = 0.5 * P.dxi[0] * (b[fidx(P, iz, iy, ixp)] - b[fidx(P, iz, iy, ixm)]);
        double db2 = gx * gx;
        double gy = 0.5 * P.dxi[1] * (b[fidx(P, iz, iyp, ix)] - b[fidx(P, iz, iym, ix)]);
        db2 = db2 + gy * gy;
        double gz = 0.5 * P.dxi[2] * (b[a + 1] - b[a - 1]);
        dbmax = fmax(dbmax, db2 + gz * gz);
    }
    __shared__ double s1[32], s2[32];
    for (int o = 16; o > 0; o >>= 1) {
        gmax = fmax(gmax, __shfl_xor_sync(0xffffffff, gmax, o));
        dbmax = fmax(dbmax, __shfl_xor_sync(0xffffffff, dbmax, o));
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { s1[w] = gmax; s2[w] = dbmax; }
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        gmax = l < nw ? s1[l] : 0.0;
        dbmax = l < nw ? s2[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            gmax = fmax(gmax, __shfl_xor_sync(0xffffffff, gmax, o));
            dbmax = fmax(dbmax, __shfl_xor_sync(0xffffffff, dbmax, o));
        }
        if (l == 0) {
            atomic_max_nonneg(&sc->gmax_bits, gmax);
            atomic_max_nonneg(&sc->bmax_bits, dbmax);
        }
    }
}

// dt = min(alpha / gmax, alpha / bmax) with the reference's guards
// (rk_utils.f90:96-99, 133-182); t is read from the device scalars.
__global__ void k_timestep_final(StepScalars* sc, double alpha, int fixed, double fixed_dt, int precise,
                                 double t_limit, double dt_cap) {
    const double eps = 2.220446049250313e-16;
    double gmax = fmax(eps, __longlong_as_double((long long)sc->gmax_bits));
    double bmax = sqrt(sqrt(__longlong_as_double((long long)sc->bmax_bits)));
    bmax = fmax(eps, bmax);
    double dt = fixed ? fixed_dt : fmin(alpha / gmax, alpha / bmax);
    if (precise && (sc->t + dt > t_limit)) dt = t_limit - sc->t;
    if (!(dt > 0.0)) sc->err |= ERRB_DT;
    sc->dt = fmin(dt, dt_cap);
}

// ---------------------------------------------------------------------------
// Host orchestration

static int nblocks(long long n, int bs = 256) {
    long long b = (n + bs - 1) / bs;
    return (int)std::min<long long>(b, 148LL * 64);
}

// Work arrays of the spectral part in the form's type T (the mixed form's
// are FP32, packed at k * fsz floats of the work block).
template <class T>
static T* wk(Ctx& c, int k) { return reinterpret_cast<T*>(c.work) + (long long)k * c.P.fsz; }

template <class T>
static ColArgs col_args(Ctx& c) {
    ColArgs A;
    std::memset(&A, 0, sizeof(A));
    if (std::is_same<T, float>::value) {
        A.mdst = c.T.mdst32; A.mdct = c.T.mdct32; A.qdst = c.T.qdst32; A.qdct = c.T.qdct32;
    } else {
        A.mdst = c.T.mdst; A.mdct = c.T.mdct; A.qdst = c.T.qdst; A.qdct = c.T.qdct;
    }
    A.qld_dst = c.T.qld_dst;
    A.qld_dct = c.T.qld_dct;
    A.sn = std::sqrt(2.0 / (double)c.P.nz);
    A.ncol = c.P.nx * c.P.ny;
    A.nz = c.P.nz;
    A.nzh = c.P.nzh;
    A.dzi = c.P.dzi;
    A.hdzi = c.P.hdzi;
    return A;
}

static SpecArgs spec_args(Ctx& c) {
    SpecArgs S;
    std::memset(&S, 0, sizeof(S));
    S.k2l2i = c.T.k2l2i;
    S.fdx = c.T.fdx;
    S.fdy = c.T.fdy;
    S.nx = c.P.nx; S.ny = c.P.ny; S.nz = c.P.nz; S.nzh = c.P.nzh;
    S.nel = (long long)c.P.nx * c.P.ny * (c.P.nz + 1);
    return S;
}

static void halo(Ctx& c, std::initializer_list<std::pair<double*, int>> list) {
    PhysArgs A;
    std::memset(&A, 0, sizeof(A));
    int f = 0;
    for (auto& e : list) { A.out[f] = e.first; A.mode[f] = e.second; ++f; }
    A.nf = f;
    A.nx = c.P.nx; A.ny = c.P.ny; A.nz = c.P.nz; A.nzh = c.P.nzh;
    A.ncol = (long long)c.P.nx * c.P.ny;
    long long tot = A.ncol * f;
    k_halo<<<(int)((tot + 255) / 256), 256, 0, c.stream>>>(A);
    CKL();
}

template <class T = double>
static size_t col_smem(const Ctx& c, int arrays) { return sizeof(T) * (size_t)arrays * (c.P.nz + 1) * CP; }

// Rows per thread of the tiled column matvec: ceil((nz + 1) / 32), nz <= 511.
static int col_rows(const Params& P) {
    int R = (P.nz + 1 + 31) / 32;
    if (R > 16) throw CudaError(EPIC_ERR_CONFIG, "nz larger than 511 is not supported");
    return R;
}

// Calls f(std::integral_constant<int, R'>{}) with R' >= R.
template <typename F>
static void with_rows(int R, F&& f) {
    switch (R) {
        case 1: f(std::integral_constant<int, 1>{}); break;
        case 2: f(std::integral_constant<int, 2>{}); break;
        case 3: f(std::integral_constant<int, 3>{}); break;
        case 4: f(std::integral_constant<int, 4>{}); break;
        case 5: f(std::integral_constant<int, 5>{}); break;
        case 6: f(std::integral_constant<int, 6>{}); break;
        case 7: f(std::integral_constant<int, 7>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        case 9: f(std::integral_constant<int, 9>{}); break;
        case 10: f(std::integral_constant<int, 10>{}); break;
        case 11: case 12: f(std::integral_constant<int, 12>{}); break;
        default: f(std::integral_constant<int, 16>{}); break;
    }
}

template <class T>
static void col_decompose(Ctx& c, const T* const* in, T* const* out, int nf, int mode) {
    ColArgs A = col_args<T>(c);
    A.tab[0] = c.T.phim; A.tab[1] = c.T.phip; A.tab[2] = c.T.filt;
    for (int f = 0; f < nf; ++f) { A.in[f] = in[f]; A.out[f] = out[f]; }
    size_t sm = col_smem<T>(c, 2);
    with_rows(col_rows(c.P), [&](auto R) {
        allow_smem(k_col_decompose<R, T>, sm);
        k_col_decompose<R, T><<<dim3((A.ncol + CT - 1) / CT, nf), 256, sm, c.stream>>>(A, mode);
        CKL();
    });
}

template <class T>
static void col_combine(Ctx& c, const T* const* in, T* const* out, int nf) {
    ColArgs A = col_args<T>(c);
    A.tab[0] = c.T.phim; A.tab[1] = c.T.phip;
    for (int f = 0; f < nf; ++f) { A.in[f] = in[f]; A.out[f] = out[f]; }
    size_t sm = col_smem<T>(c, 2);
    with_rows(col_rows(c.P), [&](auto R) {
        allow_smem(k_col_combine<R, T>, sm);
        k_col_combine<R, T><<<dim3((A.ncol + CT - 1) / CT, nf), 256, sm, c.stream>>>(A);
        CKL();
    });
}

template <class T>
static void vor2vel_t(Ctx& c) {
    const Params& P = c.P;
    SpecArgs S = spec_args(c);
    int sb = nblocks(S.nel);
    T* sv[3] = {wk<T>(c, 0), wk<T>(c, 1), wk<T>(c, 2)};
    T *ds = wk<T>(c, 3), *es = wk<T>(c, 4), *cs = wk<T>(c, 5);
    // decompose and filter (inversion.f90:36-40)
    {
        const double* in[3] = {c.vortg(0), c.vortg(1), c.vortg(2)};
        fft_xy(c, in, sv, 3, true);
        col_decompose<T>(c, sv, sv, 3, 1);
    }
    // solenoidal projection (inversion.f90:43-87)
    S.in[0] = sv[1]; S.in[1] = sv[0]; S.out[0] = ds;
    k_spec_dxdy<T><<<sb, 256, 0, c.stream>>>(S, 1.0, -1.0);
    CKL();
    {
        const T* in[1] = {sv[2]};
        T* out[1] = {cs};
        col_combine<T>(c, in, out, 1);
        const T* in2[1] = {cs};
        T* out2[1] = {es};
        col_decompose<T>(c, in2, out2, 1, 2);
    }
    S.in[0] = es; S.in[1] = ds; S.out[0] = sv[0]; S.out[1] = sv[1];
    k_spec_project<T><<<sb, 256, 0, c.stream>>>(S);
    CKL();
    // vorticity in physical space (inversion.f90:91-93); halo rows keep the
    // par2grid extrapolation, as in the reference
    // (combine(svor_z) is cs from above: svor_z is unchanged since)
    {
        T* tmp[2] = {wk<T>(c, 10), wk<T>(c, 11)};
        col_combine<T>(c, sv, tmp, 2);
        const T* inv[3] = {tmp[0], tmp[1], cs};
        double* outv[3] = {c.vortg(0), c.vortg(1), c.vortg(2)};
        fft_xy(c, inv, outv, 3, false);
    }
    // vertical velocity (inversion.f90:97-150)
    S.in[0] = sv[1]; S.in[1] = sv[0]; S.out[0] = ds;
    k_spec_dxdy<T><<<sb, 256, 0, c.stream>>>(S, -1.0, 1.0);
    CKL();
    {
        ColArgs A = col_args<T>(c);
        A.tab[0] = c.T.thetam; A.tab[1] = c.T.thetap; A.tab[2] = c.T.dthetam; A.tab[3] = c.T.dthetap;
        A.tab[4] = c.T.green; A.tab[5] = c.T.rkz;
        A.in[0] = ds;
        A.out[0] = wk<T>(c, 9);
        A.out[1] = es;
        size_t sm = col_smem<T>(c, 4);
        with_rows(col_rows(c.P), [&](auto R) {
            allow_smem(k_col_wsolve<R, T>, sm);
            k_col_wsolve<R, T><<<(A.ncol + CT - 1) / CT, 256, sm, c.stream>>>(A);
            CKL();
        });
        // cs = combine(svor_z) still holds (inversion.f90:150)
    }
    // mean flow (inversion.f90:158-176)
    T* zbuf = wk<T>(c, 13);   // first 2 (nz+1) entries used as scratch
    k_mean_flow<T><<<1, 256, 2 * sizeof(double) * (P.nz + 1), c.stream>>>(
        sv[0], sv[1], c.T.rkzi, c.T.gamtop, c.T.gambot, c.T.mdct, zbuf, P.nz);
    CKL();
    // u, v (inversion.f90:180-226)
    S.in[0] = es; S.in[1] = cs; S.out[0] = wk<T>(c, 7); S.out[1] = wk<T>(c, 8); S.zbuf = zbuf;
    k_spec_uv<T><<<sb, 256, 0, c.stream>>>(S);
    CKL();
    // velocity gradients (inversion.f90:259-300)
    S.in[0] = wk<T>(c, 7); S.in[1] = wk<T>(c, 8); S.in[2] = wk<T>(c, 9);
    S.out[0] = wk<T>(c, 10); S.out[1] = wk<T>(c, 11); S.out[2] = wk<T>(c, 12); S.out[3] = wk<T>(c, 3);
    S.out[4] = wk<T>(c, 6);
    k_spec_grad<T><<<sb, 256, 0, c.stream>>>(S);
    CKL();
    {
        const T* in[8] = {wk<T>(c, 7), wk<T>(c, 8), wk<T>(c, 9), wk<T>(c, 10), wk<T>(c, 11), wk<T>(c, 12),
                          wk<T>(c, 3), wk<T>(c, 6)};
        double* out[8] = {c.velog(0), c.velog(1), c.velog(2), c.velgrad(I_DUDX), c.velgrad(I_DUDY),
                          c.velgrad(I_DWDX), c.velgrad(I_DVDY), c.velgrad(I_DWDY)};
        fft_xy(c, in, out, 8, false);
    }
    halo(c, {{c.velgrad(I_DUDX), 0}, {c.velgrad(I_DUDY), 0}, {c.velgrad(I_DWDX), 1},
             {c.velgrad(I_DVDY), 0}, {c.velgrad(I_DWDY), 1},
             {c.velog(0), 0}, {c.velog(1), 0}, {c.velog(2), 1}});
    MPtr8 vg;
    Ptr8 vo;
    for (int k = 0; k < 8; ++k) vg.p[k] = c.velgrad(k);
    for (int k = 0; k < 3; ++k) vo.p[k] = c.vortg(k);
    k_velgrad_fill<<<nblocks(P.fsz), 256, 0, c.stream>>>(vg, vo, P.fsz);
    CKL();
}

template <class T>
static void vorticity_tendency_t(Ctx& c) {
    const Params& P = c.P;
    FluxArgs F;
    std::memset(&F, 0, sizeof(F));
    for (int k = 0; k < 3; ++k) { F.vort[k] = c.vortg(k); F.vel[k] = c.velog(k); F.fc[k] = P.f_cor[k]; }
    F.b = c.tbuoyg();
    for (int k = 0; k < 6; ++k) F.f[k] = wk<T>(c, k);
    F.nx = P.nx; F.ny = P.ny; F.nz = P.nz; F.nzh = P.nzh;
    F.nel = (long long)P.nx * P.ny * (P.nz + 1);
    int nb = nblocks(F.nel);
    k_flux<T><<<nb, 256, 0, c.stream>>>(F);
    CKL();
    T* fl[6] = {wk<T>(c, 0), wk<T>(c, 1), wk<T>(c, 2), wk<T>(c, 3), wk<T>(c, 4), wk<T>(c, 5)};
    fft_xy(c, fl, fl, 6, true);
    SpecArgs S = spec_args(c);
    for (int k = 0; k < 6; ++k) S.in[k] = wk<T>(c, k);
    S.out[0] = wk<T>(c, 6); S.out[1] = wk<T>(c, 7); S.out[2] = wk<T>(c, 8);
    k_spec_divxy<T><<<nblocks(S.nel), 256, 0, c.stream>>>(S);
    CKL();
    T* dv[3] = {wk<T>(c, 6), wk<T>(c, 7), wk<T>(c, 8)};
    fft_xy(c, dv, dv, 3, false);
    Ptr8 d;
    MPtr8 vt;
    for (int k = 0; k < 3; ++k) { d.p[k] = reinterpret_cast<const double*>(wk<T>(c, 6 + k)); vt.p[k] = c.vtend(k); }
    k_vtend_rows<T><<<nb, 256, 0, c.stream>>>(F, d, vt, P.dzi, P.hdzi, P.zeta_zero[0], P.zeta_zero[1]);
    CKL();
    halo(c, {{c.vtend(0), 0}, {c.vtend(1), 0}, {c.vtend(2), 0}});
}

// phi -> grad = gradient of the solution of Lap(psi) = phi (diverge,
// inversion.f90:410-455), grad halo rows extrapolated (parcel_correction.f90:163-165)
template <class T>
static void diverge_laplace_t(Ctx& c, double* phi, double* grad[3]) {
    const Params& P = c.P;
    T* ds = wk<T>(c, 0);
    const double* in[1] = {phi};
    T* out[1] = {ds};
    fft_xy(c, in, out, 1, true);
    int ncol = P.nx * P.ny;
    size_t lsm = col_smem<double>(c, 3);
    allow_smem(k_lapinv<T>, lsm);
    k_lapinv<T><<<(ncol + CT - 1) / CT, 256, lsm, c.stream>>>(ds, c.T.etdv, c.T.htdv, P.ap, ncol, P.nz, P.nzh);
    CKL();
    SpecArgs S = spec_args(c);
    S.in[0] = ds;
    S.out[0] = wk<T>(c, 1); S.out[1] = wk<T>(c, 2); S.out[2] = wk<T>(c, 3);
    k_spec_lapgrad<T><<<nblocks(S.nel), 256, 0, c.stream>>>(S, P.hdzi);
    CKL();
    const T* gi[3] = {wk<T>(c, 1), wk<T>(c, 2), wk<T>(c, 3)};
    fft_xy(c, gi, grad, 3, false);
    halo(c, {{grad[0], 0}, {grad[1], 0}, {grad[2], 0}});
}

// fftxyp2s, lapinv1, fftxys2p of a device field (rows 0 .. nz) into out:
// the transforms and the tridiagonal solve of diverge (test hook).
template <class T>
static void lapinv_probe_t(Ctx& c, const double* in, double* out) {
    const Params& P = c.P;
    T* ds = wk<T>(c, 0);
    const double* fin[1] = {in};
    T* fs[1] = {ds};
    fft_xy(c, fin, fs, 1, true);
    int ncol = P.nx * P.ny;
    size_t lsm = col_smem<double>(c, 3);
    allow_smem(k_lapinv<T>, lsm);
    k_lapinv<T><<<(ncol + CT - 1) / CT, 256, lsm, c.stream>>>(ds, c.T.etdv, c.T.htdv, P.ap, ncol, P.nz, P.nzh);
    CKL();
    const T* gin[1] = {ds};
    double* gout[1] = {out};
    fft_xy(c, gin, gout, 1, false);
}
void lapinv_probe(Ctx& c, const double* in, double* out) {
    if (c.pv.mixed) lapinv_probe_t<float>(c, in, out);
    else lapinv_probe_t<double>(c, in, out);
}

void fft_forward_probe(Ctx& c) {
    const double* in[3] = {c.tbuoyg(), c.velog(0), c.velog(1)};
    if (c.pv.mixed) {
        float* out[3] = {wk<float>(c, 0), wk<float>(c, 1), wk<float>(c, 2)};
        fft_xy(c, in, out, 3, true);
    } else {
        double* out[3] = {wk<double>(c, 0), wk<double>(c, 1), wk<double>(c, 2)};
        fft_xy(c, in, out, 3, true);
    }
}

// Dispatch by form: the mixed form's spectral temporaries and arithmetic are
// FP32 (the physical fields stay FP64; lapinv solves in FP64).
void vor2vel(Ctx& c) {
    if (c.pv.mixed && !c.spectral_fp64) vor2vel_t<float>(c);
    else vor2vel_t<double>(c);
}
void vorticity_tendency(Ctx& c) {
    if (c.pv.mixed && !c.spectral_fp64) vorticity_tendency_t<float>(c);
    else vorticity_tendency_t<double>(c);
}
void diverge_laplace(Ctx& c, double* phi, double* grad[3]) {
    if (c.pv.mixed && !c.spectral_fp64) diverge_laplace_t<float>(c, phi, grad);
    else diverge_laplace_t<double>(c, phi, grad);
}

void make_phi(Ctx& c, double* phi) {
    k_phi<<<nblocks(c.P.fsz), 256, 0, c.stream>>>(c.volg(), phi, c.P.vcelli, c.P.fsz);
    CKL();
}

void time_step_reduce(Ctx& c, double dt_cap) {
    CK(cudaMemsetAsync(&c.dsc->gmax_bits, 0, 2 * sizeof(unsigned long long), c.stream));
    Ptr8 vg;
    for (int k = 0; k < 8; ++k) vg.p[k] = c.velgrad(k);
    long long nel = (long long)c.P.nx * c.P.ny * (c.P.nz + 1);
    k_timestep_reduce<<<nblocks(nel), 256, 0, c.stream>>>(c.P, vg, c.tbuoyg(), c.dsc);
    CKL();
    const epic_cfg& g = c.cfg;
    k_timestep_final<<<1, 1, 0, c.stream>>>(c.dsc, g.alpha, g.use_fixed_dt, g.fixed_dt, g.precise_stop, g.t_limit,
                                            dt_cap);
    CKL();
}

// ---------------------------------------------------------------------------
// Tables (sta3dfft.f90:52-109, inversion_utils.f90:79-351), computed on the
// host in FP64 and uploaded once.
static double ipow(double x, int n) {
    double r = 1.0, b = x;
    while (n > 0) {
        if (n & 1) r *= b;
        b *= b;
        n >>= 1;
    }
    return r;
}

void spectral_init(Ctx& c) {
    const Params& P = c.P;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    cudaStream_t st = c.stream;
    make_plan(c.px, nx, st);
    make_plan(c.py, ny, st);
    const double pi = M_PI;
    // wavenumbers (sta2dfft.f90:63-67, sta3dfft.f90:88-104, deriv1d.f90:12-33)
    std::vector<double> hrkx(nx + 1), hrky(ny + 1), rkx(nx, 0.0), rky(ny, 0.0), rkz(nz + 1, 0.0), rkzi(nz + 1, 0.0);
    for (int k = 1; k <= nx; ++k) hrkx[k] = (pi / P.extent[0]) * (double)k;
    for (int k = 1; k <= ny; ++k) hrky[k] = (pi / P.extent[1]) * (double)k;
    int nwx = nx / 2, nwy = ny / 2;
    for (int k = 1; k <= nwx - 1; ++k) rkx[k] = rkx[nx - k] = hrkx[2 * k];
    rkx[nwx] = hrkx[nx];
    for (int k = 1; k <= nwy - 1; ++k) rky[k] = rky[ny - k] = hrky[2 * k];
    rky[nwy] = hrky[ny];
    for (int i = 1; i <= nz; ++i) rkz[i] = (pi / P.extent[2]) * (double)i;
    for (int i = 1; i <= nz - 1; ++i) rkzi[i] = 1.0 / rkz[i];
    // derivative factors (sta3dfft.f90:318-335)
    std::vector<double> fdx(nx, 0.0), fdy(ny, 0.0);
    for (int kx = 1; kx < nx; ++kx) {
        int dk = std::min(2 * kx, 2 * (nx - kx));
        fdx[kx] = (kx >= nwx + 1 ? 1.0 : -1.0) * hrkx[dk];
    }
    fdx[nwx] = 0.0;
    for (int ky = 1; ky < ny; ++ky) {
        int dk = std::min(2 * ky, 2 * (ny - ky));
        fdy[ky] = (ky >= nwy + 1 ? 1.0 : -1.0) * hrky[dk];
    }
    fdy[nwy] = 0.0;
    // k2l2, k2l2i (inversion_utils.f90:115-127)
    std::vector<double> k2l2((size_t)nx * ny), k2l2i((size_t)nx * ny);
    for (int kx = 0; kx < nx; ++kx)
        for (int ky = 0; ky < ny; ++ky) k2l2[(size_t)kx * ny + ky] = rkx[kx] * rkx[kx] + rky[ky] * rky[ky];
    k2l2[0] = 1.0;
    for (size_t h = 0; h < k2l2.size(); ++h) k2l2i[h] = 1.0 / k2l2[h];
    k2l2[0] = 0.0;
    k2l2i[0] = 0.0;
    // filter (inversion_utils.f90:129-150)
    double kxmaxi = 1.0 / *std::max_element(rkx.begin(), rkx.end());
    double kymaxi = 1.0 / *std::max_element(rky.begin(), rky.end());
    double kzmaxi = 1.0 / *std::max_element(rkz.begin(), rkz.end());
    std::vector<double> skx(nx), sky(ny), skz(nz + 1);
    for (int k = 0; k < nx; ++k) skx[k] = -36.0 * ipow(kxmaxi * rkx[k], 36);
    for (int k = 0; k < ny; ++k) sky[k] = -36.0 * ipow(kymaxi * rky[k], 36);
    for (int k = 0; k <= nz; ++k) skz[k] = -36.0 * ipow(kzmaxi * rkz[k], 36);

    const size_t fsz = (size_t)P.fsz;
    std::vector<double> filt(fsz, 0.0), green(fsz, 0.0), phim(fsz, 0.0), phip(fsz, 0.0), thm(fsz, 0.0),
        thp(fsz, 0.0), dthm(fsz, 0.0), dthp(fsz, 0.0), etdv(fsz, 0.0), htdv(fsz, 0.0);
    auto S = [&](int iz, int ky, int kx) { return ((size_t)kx * ny + ky) * P.nzh + 1 + iz; };
    std::vector<double> zm(nz + 1), zp(nz + 1);
    for (int iz = 0; iz <= nz; ++iz) {
        double z = P.lower[2] + P.dx[2] * (double)iz;
        zm[iz] = P.upper[2] - z;
        zp[iz] = z - P.lower[2];
    }
    const double dzisq = P.dxi[2] * P.dxi[2];
    for (int kx = 0; kx < nx; ++kx)
        for (int ky = 0; ky < ny; ++ky) {
            size_t h = (size_t)kx * ny + ky;
            double f0 = std::exp(skx[kx] + sky[ky]);
            filt[S(0, ky, kx)] = f0;
            filt[S(nz, ky, kx)] = f0;
            for (int kz = 1; kz <= nz - 1; ++kz) filt[S(kz, ky, kx)] = f0 * std::exp(skz[kz]);
            for (int kz = 1; kz <= nz; ++kz) green[S(kz, ky, kx)] = -1.0 / (k2l2[h] + rkz[kz] * rkz[kz]);
            green[S(0, ky, kx)] = -k2l2i[h];
            if (kx == 0 && ky == 0) {
                for (int iz = 0; iz <= nz; ++iz) {
                    filt[S(iz, 0, 0)] = 1.0;
                    phim[S(iz, 0, 0)] = zm[iz] / P.extent[2];
                    phip[S(iz, 0, 0)] = zp[iz] / P.extent[2];
                }
            } else {
                // set_hyperbolic_functions (inversion_utils.f90:257-351)
                double kl = std::sqrt(k2l2[h]);
                double fac = kl * P.extent[2];
                double ef = std::exp(-fac);
                double div = 1.0 / (1.0 - ef * ef);
                double k2ifac = 0.5 * k2l2i[h];
                for (int iz = 0; iz <= nz; ++iz) {
                    double Lm = kl * zm[iz], Lp = kl * zp[iz];
                    double ep = std::exp(-Lp), em = std::exp(-Lm);
                    size_t s = S(iz, ky, kx);
                    double pm = div * (ep - ef * em), pp = div * (em - ef * ep);
                    double dpm = -kl * div * (ep + ef * em), dpp = kl * div * (em + ef * ep);
                    phim[s] = pm;
                    phip[s] = pp;
                    double Q = div * (1.0 + ef * ef), R = div * 2.0 * ef;
                    thm[s] = k2ifac * (R * Lm * pp - Q * Lp * pm);
                    thp[s] = k2ifac * (R * Lp * pm - Q * Lm * pp);
                    dthm[s] = -k2ifac * ((Q * Lp - 1.0) * dpm - R * Lm * dpp);
                    dthp[s] = -k2ifac * ((Q * Lm - 1.0) * dpp - R * Lp * dpm);
                }
            }
            // tridiagonal coefficients (inversion_utils.f90:230-250)
            double a0 = -2.0 * dzisq - k2l2[h];
            double ap = dzisq;
            htdv[S(0, ky, kx)] = 1.0 / a0;
            etdv[S(0, ky, kx)] = -2.0 * ap * htdv[S(0, ky, kx)];
            for (int iz = 1; iz <= nz - 1; ++iz) {
                htdv[S(iz, ky, kx)] = 1.0 / (a0 + ap * etdv[S(iz - 1, ky, kx)]);
                etdv[S(iz, ky, kx)] = -ap * htdv[S(iz, ky, kx)];
            }
            if (kx == 0 && ky == 0) etdv[S(nz - 1, 0, 0)] = 0.0;
            htdv[S(nz, ky, kx)] = 1.0 / (a0 + 2.0 * ap * etdv[S(nz - 1, ky, kx)]);
            if (kx == 0 && ky == 0)
                for (int iz = 0; iz <= nz; ++iz) { htdv[S(iz, 0, 0)] = 0.0; etdv[S(iz, 0, 0)] = 0.0; }
        }
    std::vector<double> gamtop(nz + 1), gambot(nz + 1);
    for (int iz = 0; iz <= nz; ++iz) {
        double p00 = zp[iz] / P.extent[2];
        gamtop[iz] = 0.5 * P.extent[2] * (p00 * p00 - 1.0 / 3.0);
    }
    for (int iz = 0; iz <= nz; ++iz) gambot[iz] = gamtop[nz - iz];
    // z-transform matrices: DST-I and DCT-I with factor sqrt(2/nz)
    std::vector<double> mdst((size_t)(nz + 1) * (nz + 1), 0.0), mdct((size_t)(nz + 1) * (nz + 1), 0.0);
    double sn = std::sqrt(2.0 / (double)nz);
    for (int k = 0; k <= nz; ++k)
        for (int j = 0; j <= nz; ++j) {
            long m = ((long)j * k) % (2 * nz);
            double ang = pi * (double)m / (double)nz;
            if (k >= 1 && k <= nz - 1 && j >= 1 && j <= nz - 1) mdst[(size_t)k * (nz + 1) + j] = sn * std::sin(ang);
            double w = (j == 0 || j == nz) ? 0.5 : 1.0;
            mdct[(size_t)k * (nz + 1) + j] = sn * w * std::cos(ang);
        }
    auto up = [&](double** dst, const std::vector<double>& v) {
        CK(cudaMalloc(dst, sizeof(double) * v.size()));
        CK(cudaMemcpyAsync(*dst, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice, st));
    };
    up(&c.T.k2l2i, k2l2i); up(&c.T.fdx, fdx); up(&c.T.fdy, fdy);
    up(&c.T.filt, filt); up(&c.T.green, green); up(&c.T.phim, phim); up(&c.T.phip, phip);
    up(&c.T.thetam, thm); up(&c.T.thetap, thp); up(&c.T.dthetam, dthm); up(&c.T.dthetap, dthp);
    up(&c.T.etdv, etdv); up(&c.T.htdv, htdv);
    up(&c.T.rkz, rkz); up(&c.T.rkzi, rkzi); up(&c.T.gamtop, gamtop); up(&c.T.gambot, gambot);
    up(&c.T.mdst, mdst); up(&c.T.mdct, mdct);
    std::vector<float> mdst32(mdst.begin(), mdst.end()), mdct32(mdct.begin(), mdct.end());
    CK(cudaMalloc(&c.T.mdst32, sizeof(float) * mdst32.size()));
    CK(cudaMalloc(&c.T.mdct32, sizeof(float) * mdct32.size()));
    CK(cudaMemcpyAsync(c.T.mdst32, mdst32.data(), sizeof(float) * mdst32.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c.T.mdct32, mdct32.data(), sizeof(float) * mdct32.size(), cudaMemcpyHostToDevice, st));
    // quarter tables of the symmetric transforms (col_ztransform), even nz
    if (nz % 2 == 0 && nz >= 4) {
        auto quarter = [&](auto Z, const std::vector<double>& m, double** qd, float** qf, int* qld) {
            using ZK = decltype(Z);
            const int h = nz / 2, j0 = ZK::j0, nA = ZK::nA(h), nB = ZK::nB(h), offB = 8 * ((nA + 7) / 8);
            *qld = ZK::qld(h);
            std::vector<double> q((size_t)(h - j0 + 1) * *qld, 0.0);
            for (int j = j0; j <= h; ++j) {
                for (int i = 0; i < nA; ++i) q[(size_t)(j - j0) * *qld + i] = m[(size_t)ZK::kA(i) * (nz + 1) + j];
                for (int i = 0; i < nB; ++i) q[(size_t)(j - j0) * *qld + offB + i] = m[(size_t)ZK::kB(i) * (nz + 1) + j];
            }
            up(qd, q);
            std::vector<float> q32(q.begin(), q.end());
            CK(cudaMalloc(qf, sizeof(float) * q32.size()));
            CK(cudaMemcpyAsync(*qf, q32.data(), sizeof(float) * q32.size(), cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
        };
        quarter(ZT<0>{}, mdst, &c.T.qdst, &c.T.qdst32, &c.T.qld_dst);
        quarter(ZT<1>{}, mdct, &c.T.qdct, &c.T.qdct32, &c.T.qld_dct);
    }
    CK(cudaStreamSynchronize(st));
}

void spectral_free(Ctx& c) {
    double** all[] = {&c.T.k2l2i, &c.T.fdx, &c.T.fdy, &c.T.filt, &c.T.green, &c.T.phim, &c.T.phip,
                      &c.T.thetam, &c.T.thetap, &c.T.dthetam, &c.T.dthetap, &c.T.etdv, &c.T.htdv,
                      &c.T.rkz, &c.T.rkzi, &c.T.gamtop, &c.T.gambot, &c.T.mdst, &c.T.mdct};
    for (auto p : all) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    if (c.T.mdst32) cudaFree(c.T.mdst32);
    if (c.T.mdct32) cudaFree(c.T.mdct32);
    c.T.mdst32 = c.T.mdct32 = nullptr;
    for (double** p : {&c.T.qdst, &c.T.qdct}) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    for (float** p : {&c.T.qdst32, &c.T.qdct32}) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    if (c.px.tw) cudaFree(c.px.tw);
    if (c.py.tw) cudaFree(c.py.tw);
    c.px.tw = c.py.tw = nullptr;
}

}  // namespace epic
