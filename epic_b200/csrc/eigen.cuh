// Analytic 3x3 symmetric eigen decomposition after Scherzinger & Dohrmann
// (2008), following the reference's scherzinger.f90:31-290 step for step so
// that eigenvalues and eigenvectors agree with the FP64 oracle to rounding.
// Matrices are column-major A[i + 3*j]; eigenvector j is V[3*j .. 3*j+2].
#pragma once
#include "common.cuh"

#include <type_traits>

namespace epic {

// scherzinger.f90:16 -- the single-precision literal 1.0e-12
#define EPIC_SCHERZINGER_ATOL ((double)1.0e-12f)

template <class O, class T = typename O::T>
EPIC_DEV T dot3(const T* a, const T* b) {
    return O::add(O::add(O::mul(a[0], b[0]), O::mul(a[1], b[1])), O::mul(a[2], b[2]));
}
template <class O, class T = typename O::T>
EPIC_DEV T nrm3(const T* a) { return sqrt(dot3<O>(a, a)); }

template <class O, class T = typename O::T>
EPIC_DEV void cross3(const T* a, const T* b, T* c) {
    c[0] = O::sub(O::mul(a[1], b[2]), O::mul(a[2], b[1]));
    c[1] = O::sub(O::mul(a[2], b[0]), O::mul(a[0], b[2]));
    c[2] = O::sub(O::mul(a[0], b[1]), O::mul(a[1], b[0]));
}

EPIC_DEV float rsq(float v) { return rsqrtf(v); }
EPIC_DEV double rsq(double v) { return rsqrt(v); }

template <class T>
EPIC_DEV T signum_d(T v) { return v == T(0) ? T(0) : copysign(T(1), v); }

// evaluate_eigenvalues (scherzinger.f90:151-227); A becomes its deviator,
// r receives s1, s2 (columns 0, 1) and t3 (column 2).
template <class O, class T = typename O::T>
EPIC_DEV void sz_evaluate(T* A, T* r, T* eta, T* D) {
    const T f13 = T(1.0 / 3.0);
    T tr = O::add(O::add(A[0], A[4]), A[8]);
    T tmp = O::mul(f13, tr);
    A[0] = O::sub(A[0], tmp); A[4] = O::sub(A[4], tmp); A[8] = O::sub(A[8], tmp);
    // j2 = 1/2 trace(A A) with dsymm's evaluation (linalg.f90:57-71)
    T a11 = A[0], a12 = A[3], a13 = A[6], a22 = A[4], a23 = A[7], a33 = A[8];
    T c11 = O::add(O::add(O::mul(a11, a11), O::mul(a12, a12)), O::mul(a13, a13));
    T c22 = O::add(O::add(O::mul(a12, a12), O::mul(a22, a22)), O::mul(a23, a23));
    T c33 = O::add(O::add(O::mul(a13, a13), O::mul(a23, a23)), O::mul(a33, a33));
    T j2 = O::mul(T(0.5), O::add(O::add(c11, c22), c33));
    // determinant (linalg.f90:43-52)
    T j3 = O::add(O::sub(O::mul(a11, O::sub(O::mul(a22, a33), O::mul(a23, a23))),
                              O::mul(a12, O::sub(O::mul(a12, a33), O::mul(a13, a23)))),
                       O::mul(a13, O::sub(O::mul(a12, a23), O::mul(a13, a22))));
    const double pi = 3.141592653589793;
    T cal;   // cos(alpha)
    T smp;
    if constexpr (std::is_same<O, FastOps>::value) {
        // (3/j2)^1.5 as q sqrt(q); cos(acos(s) / 3 [+ 2 pi / 3]) as the root
        // of the triple-angle cubic 4 y^3 - 3 y = s next to an FP32 estimate,
        // refined by Newton in FP64 (|y| >= cos(pi/6), so 12 y^2 - 3 >= 6)
        const double q = 3.0 / j2;
        smp = 0.5 * j3 * (q * sqrt(q));
        smp = fmin(fmax(-1.0, smp), 1.0);
        float af = acosf((float)smp) * (1.0f / 3.0f);
        if (af > (float)(pi / 6.0)) af += (float)(2.0 * pi / 3.0);
        double y = (double)cosf(af);
        // chord steps with the derivative at the FP32 estimate (relative
        // change of f' ~ 1e-7 per step: three steps reach FP64 rounding)
        const double idf = 1.0 / (12.0 * y * y - 3.0);
#pragma unroll
        for (int it = 0; it < 3; ++it) y = y - (y * (4.0 * y * y - 3.0) - smp) * idf;
        cal = y;
    } else if constexpr (std::is_same<O, F32Ops>::value) {
        // the FP32 form: (3/j2)^1.5 as q sqrt(q), single-precision acos / cos
        const float q = 3.0f / j2;
        smp = 0.5f * j3 * (q * sqrtf(q));
        smp = fminf(fmaxf(-1.0f, smp), 1.0f);
        float alpha = acosf(smp) * (1.0f / 3.0f);
        if (alpha > (float)(pi / 6.0)) alpha += (float)(2.0 * pi / 3.0);
        cal = cosf(alpha);
    } else {
        smp = O::mul(O::mul(T(0.5), j3), pow(T(3) / j2, T(1.5)));
        smp = fmin(fmax(T(-1), smp), T(1));
        T alpha = O::mul(f13, acos(smp));
        if (alpha > T(pi / 6.0)) alpha = O::add(alpha, O::mul(T(2.0 / 3.0), T(pi)));
        cal = cos(alpha);
    }
    eta[0] = O::mul(O::mul(T(2), sqrt(O::mul(f13, j2))), cal);
    r[0] = O::sub(A[0], eta[0]); r[1] = A[1];                 r[2] = A[2];
    r[3] = A[3];                 r[4] = O::sub(A[4], eta[0]); r[5] = A[5];
    r[6] = A[6];                 r[7] = A[7];                 r[8] = O::sub(A[8], eta[0]);
    int i = 0;
    T s1[3];
    if constexpr (std::is_same<O, FastOps>::value || std::is_same<O, F32Ops>::value) {
        // the longest column by squared norms, normalised by a reciprocal square root
        const T q0 = dot3<O>(&r[0], &r[0]), q1 = dot3<O>(&r[3], &r[3]), q2 = dot3<O>(&r[6], &r[6]);
        T qm = q0;
        if (q1 > qm) { i = 1; qm = q1; }
        if (q2 > qm) { i = 2; qm = q2; }
        const T ir = rsq(qm);
#pragma unroll
        for (int k = 0; k < 3; ++k) s1[k] = (i == 0 ? r[k] : i == 1 ? r[3 + k] : r[6 + k]) * ir;
    } else {
        T rl0 = nrm3<O>(&r[0]), rl1 = nrm3<O>(&r[3]), rl2 = nrm3<O>(&r[6]);
        T rm = rl0;
        if (rl1 > rm) { i = 1; rm = rl1; }
        if (rl2 > rm) { i = 2; rm = rl2; }
        // column i of r, selected without a run-time array index (keeps r in registers)
#pragma unroll
        for (int k = 0; k < 3; ++k) s1[k] = (i == 0 ? r[k] : i == 1 ? r[3 + k] : r[6 + k]) / rm;
    }
    if (i == 1) { r[3] = r[0]; r[4] = r[1]; r[5] = r[2]; }
    else if (i == 2) { r[6] = r[0]; r[7] = r[1]; r[8] = r[2]; }
    r[0] = s1[0]; r[1] = s1[1]; r[2] = s1[2];
    tmp = dot3<O>(&r[0], &r[3]);
    smp = dot3<O>(&r[0], &r[6]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r[3 + k] = O::sub(r[3 + k], O::mul(tmp, r[k]));
        r[6 + k] = O::sub(r[6 + k], O::mul(smp, r[k]));
    }
    T s2[3];
    if constexpr (std::is_same<O, FastOps>::value || std::is_same<O, F32Ops>::value) {
        const T q1 = dot3<O>(&r[3], &r[3]), q2 = dot3<O>(&r[6], &r[6]);
        const int j = (q2 > q1) ? 2 : 1;
        const T ir = rsq(j == 2 ? q2 : q1);
#pragma unroll
        for (int k = 0; k < 3; ++k) s2[k] = (j == 2 ? r[6 + k] : r[3 + k]) * ir;
    } else {
        T rl1 = nrm3<O>(&r[3]);
        T rl2 = nrm3<O>(&r[6]);
        int j = (rl2 > rl1) ? 2 : 1;
        T rj = (j == 2) ? rl2 : rl1;
#pragma unroll
        for (int k = 0; k < 3; ++k) s2[k] = (j == 2 ? r[6 + k] : r[3 + k]) / rj;
    }
    r[3] = s2[0]; r[4] = s2[1]; r[5] = s2[2];
    T Ar[6];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int row = 0; row < 3; ++row)
            Ar[row + 3 * c] = O::add(O::add(O::mul(A[row], r[3 * c]), O::mul(A[row + 3], r[3 * c + 1])),
                                     O::mul(A[row + 6], r[3 * c + 2]));
    T s1As1 = dot3<O>(&r[0], &Ar[0]);
    T s2As1 = dot3<O>(&r[3], &Ar[0]);
    T s1As2 = s2As1;
    T s2As2 = dot3<O>(&r[3], &Ar[3]);
    tmp = O::sub(s1As1, s2As2);
    smp = O::add(s1As1, s2As2);
    T disc = O::add(O::mul(tmp, tmp), O::mul(O::mul(T(4), s1As2), s2As1));
    eta[1] = O::sub(O::mul(T(0.5), smp), O::mul(O::mul(T(0.5), signum_d(tmp)), sqrt(disc)));
    eta[2] = O::sub(smp, eta[1]);
    T t3 = O::mul(f13, tr);
    D[0] = O::add(eta[0], t3); D[1] = O::add(eta[1], t3); D[2] = O::add(eta[2], t3);
}

template <class T>
EPIC_DEV void swapd(T& a, T& b) { T t = a; a = b; b = t; }

// scherzinger_eigenvalues (scherzinger.f90:127-147) + sort_eigenvalues
template <class O, class T = typename O::T>
EPIC_DEV void sz_eigenvalues(T* A, T* D) {
    T off = fabs(A[3]) + fabs(A[6]) + fabs(A[7]);
    if (off < T(EPIC_SCHERZINGER_ATOL)) {
        D[0] = A[0]; D[1] = A[4]; D[2] = A[8];
    } else {
        T r[9], eta[3];
        sz_evaluate<O>(A, r, eta, D);
    }
    if (D[1] > D[0]) swapd(D[0], D[1]);
    if (D[2] > D[1]) swapd(D[1], D[2]);
    if (D[1] > D[0]) swapd(D[0], D[1]);
}

template <class T>
EPIC_DEV void swapcol(T* V, int a, int b) {
#pragma unroll
    for (int k = 0; k < 3; ++k) swapd(V[3 * a + k], V[3 * b + k]);
}

// scherzinger_diagonalise (scherzinger.f90:31-118)
template <class O, class T = typename O::T>
EPIC_DEV void sz_diagonalise(T* A, T* D, T* V) {
    T off = fabs(A[3]) + fabs(A[6]) + fabs(A[7]);
    if (off < T(EPIC_SCHERZINGER_ATOL)) {
#pragma unroll
        for (int k = 0; k < 9; ++k) V[k] = T(0);
        V[0] = V[4] = V[8] = T(1);
        D[0] = A[0]; D[1] = A[4]; D[2] = A[8];
    } else {
        T r[9], eta[3];
        sz_evaluate<O>(A, r, eta, D);
        A[0] = O::sub(A[0], eta[1]); A[4] = O::sub(A[4], eta[1]); A[8] = O::sub(A[8], eta[1]);
        cross3<O>(&r[0], &r[3], &V[0]);
        T Ar[6];
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int row = 0; row < 3; ++row)
                Ar[row + 3 * c] = O::add(O::add(O::mul(A[row], r[3 * c]), O::mul(A[row + 3], r[3 * c + 1])),
                                         O::mul(A[row + 6], r[3 * c + 2]));
        if constexpr (std::is_same<O, FastOps>::value || std::is_same<O, F32Ops>::value) {
            // normalisations by reciprocal square roots
            const T q0 = dot3<O>(&Ar[0], &Ar[0]), q1 = dot3<O>(&Ar[3], &Ar[3]);
            const int i = (q1 > q0) ? 1 : 0;
            const T il = rsq(i ? q1 : q0);
#pragma unroll
            for (int k = 0; k < 3; ++k) V[6 + k] = (i ? Ar[3 + k] : Ar[k]) * il;
            cross3<O>(&V[6], &V[0], &V[3]);
            cross3<O>(&V[0], &V[3], &V[6]);
            const T n0 = rsq(dot3<O>(&V[0], &V[0])), n1 = rsq(dot3<O>(&V[3], &V[3]));
            const T n2 = rsq(dot3<O>(&V[6], &V[6]));
#pragma unroll
            for (int k = 0; k < 3; ++k) { V[k] *= n0; V[3 + k] *= n1; V[6 + k] *= n2; }
        } else {
            T l0 = nrm3<O>(&Ar[0]), l1 = nrm3<O>(&Ar[3]);
            int i = (l1 > l0) ? 1 : 0;
            T li = i ? l1 : l0;
#pragma unroll
            for (int k = 0; k < 3; ++k) V[6 + k] = (i ? Ar[3 + k] : Ar[k]) / li;
            cross3<O>(&V[6], &V[0], &V[3]);
            cross3<O>(&V[0], &V[3], &V[6]);
            T n0 = nrm3<O>(&V[0]), n1 = nrm3<O>(&V[3]), n2 = nrm3<O>(&V[6]);
#pragma unroll
            for (int k = 0; k < 3; ++k) { V[k] /= n0; V[3 + k] /= n1; V[6 + k] /= n2; }
        }
    }
    if (D[1] > D[0]) { swapd(D[0], D[1]); swapcol(V, 0, 1); }
    if (D[2] > D[1]) { swapd(D[1], D[2]); swapcol(V, 1, 2); }
    if (D[1] > D[0]) { swapd(D[0], D[1]); swapcol(V, 0, 1); }
}

// get_abc (parcel_ellipsoid.f90:409-415)
EPIC_DEV double get_abc(double volume) {
    const double fpi = 1.0 / 3.141592653589793;
    return 0.75 * volume * fpi;
}

// get_B33 (parcel_ellipsoid.f90:383-402); sets ERRB_B33 on a small divisor.
template <class O>
EPIC_DEV double get_B33(const double* b, double vol, unsigned* err) {
    double abc = get_abc(vol);
    double den = O::sub(O::mul(b[0], b[3]), O::mul(b[1], b[1]));
    if (fabs(den) <= 2.220446049250313e-16) set_err(err, ERRB_B33);
    double num = O::sub(O::add(O::sub(O::mul(abc, abc), O::mul(b[2], O::sub(O::mul(b[1], b[4]), O::mul(b[2], b[3])))),
                               O::mul(b[0], O::mul(b[4], b[4]))),
                        O::mul(O::mul(b[1], b[2]), b[4]));
    return num / den;
}

template <class O, class T = typename O::T>
EPIC_DEV void full_matrix(const T* b, T B33, T* U) {
    U[0] = b[0]; U[3] = b[1]; U[6] = b[2];
    U[1] = b[1]; U[4] = b[3]; U[7] = b[4];
    U[2] = b[2]; U[5] = b[4]; U[8] = B33;
}

// Support-point vectors (parcel_ellipsoid.f90:216-247):
// Veta = sqrt|a2 - c2| rho v1, Vtau = sqrt|b2 - c2| rho v2.
template <class O>
EPIC_DEV void support_vectors(const double* b, double vol, double* Veta, double* Vtau, double* Dout,
                              unsigned* err) {
    double U[9], D[3], V[9];
    full_matrix<O>(b, get_B33<O>(b, vol, err), U);
    sz_diagonalise<O>(U, D, V);
    const double rho = 0.6324555320336759;   // sqrt(2/5)
    double se = sqrt(fabs(D[0] - D[2])) * rho;
    double st = sqrt(fabs(D[1] - D[2])) * rho;
#pragma unroll
    for (int k = 0; k < 3; ++k) { Veta[k] = se * V[k]; Vtau[k] = st * V[3 + k]; }
    if (Dout) { Dout[0] = D[0]; Dout[1] = D[1]; Dout[2] = D[2]; }
}

// Mixed form: B in FP32, B33 recovered in FP64 (get_B33), the eigen-
// decomposition and the support vectors in FP32.
EPIC_DEV void support_vectors_f32(const float* b, double vol, float* Veta, float* Vtau, unsigned* err) {
    double bd[5] = {b[0], b[1], b[2], b[3], b[4]};
    float U[9], D[3], V[9];
    full_matrix<F32Ops>(b, (float)get_B33<FastOps>(bd, vol, err), U);
    sz_diagonalise<F32Ops>(U, D, V);
    const float rho = 0.6324555320336759f;   // sqrt(2/5)
    float se = sqrtf(fabsf(D[0] - D[2])) * rho;
    float st = sqrtf(fabsf(D[1] - D[2])) * rho;
#pragma unroll
    for (int k = 0; k < 3; ++k) { Veta[k] = se * V[k]; Vtau[k] = st * V[3 + k]; }
}

// cos/sin of theta_j = (2j-1) pi / 4 evaluated in FP64 from the double
// arguments j * (pi/4) (parcel_ellipsoid.f90:30-34), as the reference's
// compile-time constants are.
EPIC_DEV double support_cos(int j) {
    return j == 0 ? 0.7071067811865476 : j == 1 ? -0.7071067811865475 : j == 2 ? -0.7071067811865477
                                                                              : 0.7071067811865474;
}
EPIC_DEV double support_sin(int j) {
    return j == 0 ? 0.7071067811865475 : j == 1 ? 0.7071067811865476 : j == 2 ? -0.7071067811865475
                                                                             : -0.7071067811865477;
}

}  // namespace epic
