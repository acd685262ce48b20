// ORACLE -- test infrastructure only.
//
// CPU FP64 restatement of the reference EPIC 3-D parcel step (EPIC 0.14.3),
// used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as
// the checker.  Nothing in the product (epic_b200/) may include or link it.
//
// Parity pinning: the eigen-solver is pinned against the reference's golden
// vectors unit-tests/3d/{B,D,V}.asc (test_scherzinger_2.f90:47, atol 1e-12);
// the spectral inversion against the reference's analytic unit tests
// (test_mpi_vor2vel.f90, test_mpi_vel2vgrad.f90, test_mpi_diffx/diffy,
// test_mpi_fft*, test_mpi_dst); interpolation against test_mpi_trilinear /
// test_mpi_grid2par; merging against the test_mpi_nearest_* constellations.
// The full step has no reference golden vector (the reference cannot be built
// here: no Fortran compiler, MPI or NetCDF), so end-to-end parity is pinned
// only through these component tests.
//
// Every function cites the reference file:line it restates.  Fortran
// evaluation order (left to right) is kept in the arithmetic so that results
// agree to rounding; Fortran intrinsic semantics are kept where they matter
// for decisions: nint = round half away from zero, int = truncate, floor,
// maxloc = first maximum.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <vector>
#include <complex>
#include <string>
#include <stdexcept>
#include <algorithm>

namespace oracle {

// constants.f90:7-46
static const double zero = 0.0, one = 1.0, two = 2.0, three = 3.0, four = 4.0, five = 5.0;
static const double pi = std::acos(-1.0);
static const double twopi = 2.0 * pi;
static const double fpi = 1.0 / pi;
static const double fpi4 = pi / 4.0;
static const double fpi6 = pi / 6.0;
static const double f12 = 0.5, f13 = 1.0 / 3.0, f14 = 0.25, f23 = 2.0 / 3.0, f32 = 1.5, f34 = 0.75;

struct OracleError : std::runtime_error {
    int code;
    OracleError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Fortran NINT: round half away from zero.
inline int fnint(double x) { return (int)std::lround(x); }
// Fortran INT: truncate toward zero.
inline int fint(double x) { return (int)x; }
inline int ffloor(double x) { return (int)std::floor(x); }

// Integer power by repeated squaring, as gfortran evaluates x**n for an
// integer literal n (used for the Hou-Li filter exponent 36,
// inversion_utils.f90:129-135).
inline double powi(double x, int n) {
    double r = 1.0, b = x;
    while (n > 0) {
        if (n & 1) r *= b;
        b *= b;
        n >>= 1;
    }
    return r;
}

// ---------------------------------------------------------------------------
// linalg.f90:9-71
inline double signum(double v) {
    double s = std::copysign(1.0, v);
    if (v == 0.0) s = 0.0;
    return s;
}
inline void cross(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
// Column-major 3x3: A[i + 3*j] = A(i+1, j+1).
#define M3(A, i, j) (A)[(i) + 3 * (j)]
inline double trace3(const double* A) { return M3(A, 0, 0) + M3(A, 1, 1) + M3(A, 2, 2); }
inline double determinant3(const double* A) {
    return M3(A, 0, 0) * (M3(A, 1, 1) * M3(A, 2, 2) - M3(A, 1, 2) * M3(A, 1, 2))
         - M3(A, 0, 1) * (M3(A, 0, 1) * M3(A, 2, 2) - M3(A, 0, 2) * M3(A, 1, 2))
         + M3(A, 0, 2) * (M3(A, 0, 1) * M3(A, 1, 2) - M3(A, 0, 2) * M3(A, 1, 1));
}
inline void dsymm(const double* A, const double* B, double* C) {
    M3(C, 0, 0) = M3(A, 0, 0) * M3(B, 0, 0) + M3(A, 0, 1) * M3(B, 0, 1) + M3(A, 0, 2) * M3(B, 0, 2);
    M3(C, 0, 1) = M3(A, 0, 0) * M3(B, 0, 1) + M3(A, 0, 1) * M3(B, 1, 1) + M3(A, 0, 2) * M3(B, 1, 2);
    M3(C, 0, 2) = M3(A, 0, 0) * M3(B, 0, 2) + M3(A, 0, 1) * M3(B, 1, 2) + M3(A, 0, 2) * M3(B, 2, 2);
    M3(C, 1, 0) = M3(A, 0, 1) * M3(B, 0, 0) + M3(A, 1, 1) * M3(B, 0, 1) + M3(A, 1, 2) * M3(B, 0, 2);
    M3(C, 1, 1) = M3(A, 0, 1) * M3(B, 0, 1) + M3(A, 1, 1) * M3(B, 1, 1) + M3(A, 1, 2) * M3(B, 1, 2);
    M3(C, 1, 2) = M3(A, 0, 1) * M3(B, 0, 2) + M3(A, 1, 1) * M3(B, 1, 2) + M3(A, 1, 2) * M3(B, 2, 2);
    M3(C, 2, 0) = M3(A, 0, 2) * M3(B, 0, 0) + M3(A, 1, 2) * M3(B, 0, 1) + M3(A, 2, 2) * M3(B, 0, 2);
    M3(C, 2, 1) = M3(A, 0, 2) * M3(B, 0, 1) + M3(A, 1, 2) * M3(B, 1, 1) + M3(A, 2, 2) * M3(B, 1, 2);
    M3(C, 2, 2) = M3(A, 0, 2) * M3(B, 0, 2) + M3(A, 1, 2) * M3(B, 1, 2) + M3(A, 2, 2) * M3(B, 2, 2);
}
// norm2 of a 3-vector, evaluated as sqrt of the sum of squares.  gfortran's
// norm2 uses a scaled sum; both agree to within an ulp.
inline double norm2v(const double* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// ---------------------------------------------------------------------------
// scherzinger.f90:16 -- atol is the single-precision literal 1.0e-12.
static const double scherzinger_atol = (double)1.0e-12f;

// scherzinger.f90:151-227 (evaluate_eigenvalues).  A (column-major, symmetric)
// is overwritten by its deviator; r receives s1, s2 in columns 0, 1.
inline void evaluate_eigenvalues(double* A, double* r, double* eta, double* D) {
    double AA[9];
    double tr = trace3(A);
    double tmp = f13 * tr;
    M3(A, 0, 0) -= tmp; M3(A, 1, 1) -= tmp; M3(A, 2, 2) -= tmp;
    dsymm(A, A, AA);
    double j2 = f12 * trace3(AA);
    double j3 = determinant3(A);
    double smp = f12 * j3 * std::pow(three / j2, f32);
    smp = std::min(std::max(-one, smp), one);
    double alpha = f13 * std::acos(smp);
    if (alpha > fpi6) alpha = alpha + f23 * pi;
    eta[0] = two * std::sqrt(f13 * j2) * std::cos(alpha);
    // eq 19: r columns
    M3(r, 0, 0) = M3(A, 0, 0) - eta[0]; M3(r, 1, 0) = M3(A, 1, 0);          M3(r, 2, 0) = M3(A, 2, 0);
    M3(r, 0, 1) = M3(A, 0, 1);          M3(r, 1, 1) = M3(A, 1, 1) - eta[0]; M3(r, 2, 1) = M3(A, 2, 1);
    M3(r, 0, 2) = M3(A, 0, 2);          M3(r, 1, 2) = M3(A, 1, 2);          M3(r, 2, 2) = M3(A, 2, 2) - eta[0];
    double rlen[3] = {norm2v(&r[0]), norm2v(&r[3]), norm2v(&r[6])};
    int i = 0;
    if (rlen[1] > rlen[i]) i = 1;
    if (rlen[2] > rlen[i]) i = 2;
    double s1[3] = {r[3 * i] / rlen[i], r[3 * i + 1] / rlen[i], r[3 * i + 2] / rlen[i]};
    if (i == 1) { r[3] = r[0]; r[4] = r[1]; r[5] = r[2]; }
    else if (i == 2) { r[6] = r[0]; r[7] = r[1]; r[8] = r[2]; }
    r[0] = s1[0]; r[1] = s1[1]; r[2] = s1[2];
    tmp = dot3(&r[0], &r[3]);
    smp = dot3(&r[0], &r[6]);
    for (int k = 0; k < 3; ++k) {
        r[3 + k] = r[3 + k] - tmp * r[k];
        r[6 + k] = r[6 + k] - smp * r[k];
    }
    rlen[0] = norm2v(&r[0]); rlen[1] = norm2v(&r[3]); rlen[2] = norm2v(&r[6]);
    i = (rlen[2] > rlen[1]) ? 2 : 1;
    double s2[3] = {r[3 * i] / rlen[i], r[3 * i + 1] / rlen[i], r[3 * i + 2] / rlen[i]};
    r[3] = s2[0]; r[4] = s2[1]; r[5] = s2[2];
    // eq 22: AA(:,1:2) = matmul(A, r(:,1:2))
    double Ar[6];
    for (int c = 0; c < 2; ++c)
        for (int row = 0; row < 3; ++row)
            Ar[row + 3 * c] = M3(A, row, 0) * r[0 + 3 * c] + M3(A, row, 1) * r[1 + 3 * c] + M3(A, row, 2) * r[2 + 3 * c];
    double s1As1 = dot3(&r[0], &Ar[0]);
    double s2As1 = dot3(&r[3], &Ar[0]);
    double s1As2 = s2As1;
    double s2As2 = dot3(&r[3], &Ar[3]);
    tmp = s1As1 - s2As2;
    smp = s1As1 + s2As2;
    eta[1] = f12 * smp - f12 * signum(tmp) * std::sqrt(tmp * tmp + four * s1As2 * s2As1);
    eta[2] = smp - eta[1];
    for (int k = 0; k < 3; ++k) D[k] = eta[k] + f13 * tr;
}

// scherzinger.f90:234-257 (sort_eigenvalues)
inline void sort_eigenvalues(double* D) {
    double t;
    if (D[1] > D[0]) { t = D[0]; D[0] = D[1]; D[1] = t; }
    if (D[2] > D[1]) { t = D[1]; D[1] = D[2]; D[2] = t; }
    if (D[1] > D[0]) { t = D[0]; D[0] = D[1]; D[1] = t; }
}

// scherzinger.f90:127-147 (scherzinger_eigenvalues)
inline void scherzinger_eigenvalues(double* A, double* D) {
    double tmp = std::fabs(M3(A, 0, 1)) + std::fabs(M3(A, 0, 2)) + std::fabs(M3(A, 1, 2));
    if (tmp < scherzinger_atol) {
        D[0] = M3(A, 0, 0); D[1] = M3(A, 1, 1); D[2] = M3(A, 2, 2);
    } else {
        double r[9], eta[3];
        evaluate_eigenvalues(A, r, eta, D);
    }
    sort_eigenvalues(D);
}

inline void swap_cols(double* V, int a, int b) {
    for (int k = 0; k < 3; ++k) std::swap(V[3 * a + k], V[3 * b + k]);
}

// scherzinger.f90:31-118 (scherzinger_diagonalise).  V column j belongs to D[j].
inline void scherzinger_diagonalise(double* A, double* D, double* V) {
    double tmp = std::fabs(M3(A, 0, 1)) + std::fabs(M3(A, 0, 2)) + std::fabs(M3(A, 1, 2));
    if (tmp < scherzinger_atol) {
        for (int k = 0; k < 9; ++k) V[k] = 0.0;
        V[0] = V[4] = V[8] = 1.0;
        D[0] = M3(A, 0, 0); D[1] = M3(A, 1, 1); D[2] = M3(A, 2, 2);
        // sort_descending (scherzinger.f90:261-290)
        double t;
        if (D[1] > D[0]) { t = D[0]; D[0] = D[1]; D[1] = t; swap_cols(V, 0, 1); }
        if (D[2] > D[1]) { t = D[1]; D[1] = D[2]; D[2] = t; swap_cols(V, 1, 2); }
        if (D[1] > D[0]) { t = D[0]; D[0] = D[1]; D[1] = t; swap_cols(V, 0, 1); }
        return;
    }
    double r[9], eta[3];
    evaluate_eigenvalues(A, r, eta, D);
    M3(A, 0, 0) -= eta[1]; M3(A, 1, 1) -= eta[1]; M3(A, 2, 2) -= eta[1];
    cross(&r[0], &r[3], &V[0]);
    double Ar[6];
    for (int c = 0; c < 2; ++c)
        for (int row = 0; row < 3; ++row)
            Ar[row + 3 * c] = M3(A, row, 0) * r[0 + 3 * c] + M3(A, row, 1) * r[1 + 3 * c] + M3(A, row, 2) * r[2 + 3 * c];
    for (int k = 0; k < 6; ++k) r[k] = Ar[k];
    double rlen[3] = {norm2v(&r[0]), norm2v(&r[3]), norm2v(&r[6])};
    int i = (rlen[1] > rlen[0]) ? 1 : 0;
    for (int k = 0; k < 3; ++k) V[6 + k] = r[3 * i + k] / rlen[i];
    cross(&V[6], &V[0], &V[3]);
    cross(&V[0], &V[3], &V[6]);
    rlen[0] = norm2v(&V[0]); rlen[1] = norm2v(&V[3]); rlen[2] = norm2v(&V[6]);
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 3; ++k) V[3 * c + k] = V[3 * c + k] / rlen[c];
    double t;
    if (D[1] > D[0]) { t = D[0]; D[0] = D[1]; D[1] = t; swap_cols(V, 0, 1); }
    if (D[2] > D[1]) { t = D[1]; D[1] = D[2]; D[2] = t; swap_cols(V, 1, 2); }
    if (D[1] > D[0]) { t = D[0]; D[0] = D[1]; D[1] = t; swap_cols(V, 0, 1); }
}

// ---------------------------------------------------------------------------
// Spectral transforms.  The reference's stafft (src/fft/stafft.f90) is a
// mixed-radix real FFT whose output is in "Hermitian form"
// (stafft.f90:55-59): for X_k = sum_j x_j exp(-2 pi i j k / n),
//   out[k]   = Re X_k / sqrt(n)   (k = 0 .. n/2)
//   out[n-k] = Im X_k / sqrt(n)   (k = 1 .. (n-1)/2)
// (normalisation stafft.f90:279; the sign of the sine slots follows from the
// derivative rule of deriv1d.f90:60-86 and sta3dfft.f90:301-337).  revfft is
// its exact inverse (stafft.f90:296-403).  dst / dct (stafft.f90:410-550)
// are the self-inverse DST-I / DCT-I with factor sqrt(2/n).  This oracle
// computes the same transforms with its own complex mixed-radix FFT.
struct CFFT {
    int n = 0;
    std::vector<std::complex<double>> w;   // exp(-2 pi i k / n)
    std::vector<int> factors;
    void init(int n_) {
        n = n_;
        w.resize(n);
        for (int k = 0; k < n; ++k) w[k] = std::polar(1.0, -twopi * (double)k / (double)n);
        factors.clear();
        int rem = n;
        for (int p : {4, 2, 3, 5}) while (rem % p == 0) { factors.push_back(p); rem /= p; }
        for (int p = 7; rem > 1; ++p) while (rem % p == 0) { factors.push_back(p); rem /= p; }
    }
    // Recursive decimation in time with one scratch buffer of n elements:
    // out[kk] = sum_j in[j*stride] * W_len^(j*kk), W_len = exp(-2 pi i / len).
    void rec(const std::complex<double>* in, std::complex<double>* out, int len, int stride,
             size_t fi, int wstep, std::complex<double>* scratch) const {
        if (len == 1) { out[0] = in[0]; return; }
        int p = factors[fi];
        int m = len / p;
        for (int r = 0; r < p; ++r) rec(in + r * stride, out + r * m, m, stride * p, fi + 1, wstep * p, scratch);
        for (int kk = 0; kk < len; ++kk) {
            int k = kk % m;
            std::complex<double> s = out[k];
            for (int r = 1; r < p; ++r) {
                long e = ((long)r * kk) % len;
                s += out[(size_t)r * m + k] * w[(size_t)(e * wstep)];
            }
            scratch[kk] = s;
        }
        for (int kk = 0; kk < len; ++kk) out[kk] = scratch[kk];
    }
    void forward(const std::complex<double>* in, std::complex<double>* out) const {
        thread_local std::vector<std::complex<double>> scratch;
        if ((int)scratch.size() < n) scratch.resize(n);
        rec(in, out, n, 1, 0, 1, scratch.data());
    }
};

// Real transform of one line with the stafft conventions.
struct RealFFT {
    int n = 0;
    CFFT c;
    void init(int n_) { n = n_; c.init(n_); }
    // forfft (stafft.f90:196-287)
    void forfft(double* x) const {
        thread_local std::vector<std::complex<double>> a, b;
        if ((int)a.size() < n) { a.resize(n); b.resize(n); }
        for (int j = 0; j < n; ++j) a[j] = x[j];
        c.forward(a.data(), b.data());
        double s = one / std::sqrt((double)n);
        x[0] = b[0].real() * s;
        for (int k = 1; 2 * k < n; ++k) {
            x[k] = b[k].real() * s;
            x[n - k] = b[k].imag() * s;
        }
        if (n % 2 == 0) x[n / 2] = b[n / 2].real() * s;
    }
    // revfft (stafft.f90:296-403)
    void revfft(double* x) const {
        thread_local std::vector<std::complex<double>> a, b;
        if ((int)a.size() < n) { a.resize(n); b.resize(n); }
        double rn = std::sqrt((double)n);
        a[0] = x[0] * rn;
        for (int k = 1; 2 * k < n; ++k) {
            a[k] = std::complex<double>(x[k], x[n - k]) * rn;
            a[n - k] = std::conj(a[k]);
        }
        if (n % 2 == 0) a[n / 2] = x[n / 2] * rn;
        // inverse DFT: x_j = (1/n) sum_k a_k exp(+2 pi i jk/n) = conj(FFT(conj(a)))/n
        for (int k = 0; k < n; ++k) a[k] = std::conj(a[k]);
        c.forward(a.data(), b.data());
        for (int j = 0; j < n; ++j) x[j] = b[j].real() / (double)n;
    }
};

// DST-I / DCT-I of length n (stafft.f90:410-550) through a complex FFT of
// length 2n of the odd / even extension.
struct TrigTransform {
    int n = 0;
    CFFT c2;
    void init(int n_) { n = n_; c2.init(2 * n_); }
    // dst(1, n, x(1:n)): x[0..n-1] holds x(1..n); x(n) is ignored on input and
    // zero on output.
    void dst(double* x) const {
        thread_local std::vector<std::complex<double>> a, b;
        if ((int)a.size() < 2 * n) { a.resize(2 * n); b.resize(2 * n); }
        std::fill(a.begin(), a.begin() + 2 * n, std::complex<double>(0.0));
        for (int j = 1; j < n; ++j) { a[j] = x[j - 1]; a[2 * n - j] = -x[j - 1]; }
        c2.forward(a.data(), b.data());
        double s = std::sqrt(two / (double)n);
        for (int k = 1; k < n; ++k) x[k - 1] = -s * b[k].imag() * f12;
        x[n - 1] = zero;
    }
    // dct(1, n, x(0:n))
    void dct(double* x) const {
        thread_local std::vector<std::complex<double>> a, b;
        if ((int)a.size() < 2 * n) { a.resize(2 * n); b.resize(2 * n); }
        for (int j = 0; j <= n; ++j) a[j] = x[j];
        for (int j = 1; j < n; ++j) a[2 * n - j] = x[j];
        c2.forward(a.data(), b.data());
        double s = std::sqrt(two / (double)n);
        for (int k = 0; k <= n; ++k) x[k] = s * b[k].real() * f12;
    }
};

}  // namespace oracle
