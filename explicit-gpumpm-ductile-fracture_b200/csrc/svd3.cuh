// 3x3 SVD by Givens bidiagonalisation and implicit-shift QR sweeps, the
// algorithm of the reference's __GEIGEN__::math::qr_svd (QRSVD.hpp:224-322,
// givens.hpp:11-210), written register-resident: every rotation acts on
// compile-time row/column pairs so nothing spills to local memory.
//
// Matrices are row-major R[9] (element (r,c) at 3r+c).  F = U diag(S) V^T.
#pragma once
#include <cfloat>
#include <cuda_runtime.h>

namespace gmpm {

template <typename R> struct SvdEps;
template <> struct SvdEps<float> {
    // numeric_limits<float>::epsilon() * 128
    __device__ static constexpr float value() { return 1.1920928955078125e-07f * 128.0f; }
};
template <> struct SvdEps<double> {
    __device__ static constexpr double value() { return 2.220446049250313e-16 * 128.0; }
};

__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_r(double x) { return 1.0 / sqrt(x); }

// Quotients: in FP32 the reciprocal-based __fdividef (within 2 ulp for the
// normal-range divisors met here: singular values, stress norms, material
// constants), in FP64 IEEE division as in the oracle.  An IEEE FP32 division
// is a multi-instruction sequence with a slow-path branch; the SVD and return
// map take about a dozen per particle.
__device__ __forceinline__ float div_r(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double div_r(double a, double b) { return a / b; }

// Conventional Givens: [c -s; s c][a; b] = [*; 0]  (givens.hpp:48-59)
template <typename R>
__device__ __forceinline__ void givens_conventional(R a, R b, R& c, R& s) {
    const R d = a * a + b * b;
    c = R(1);
    s = R(0);
    if (d != R(0)) {
        const R t = rsqrt_r(d);
        c = a * t;
        s = -b * t;
    }
}
// Unconventional Givens: [c -s; s c][a; b] = [0; *]  (givens.hpp:62-73)
template <typename R>
__device__ __forceinline__ void givens_unconventional(R a, R b, R& c, R& s) {
    const R d = a * a + b * b;
    c = R(0);
    s = R(1);
    if (d != R(0)) {
        const R t = rsqrt_r(d);
        s = a * t;
        c = b * t;
    }
}
// A <- G^T A on rows I,K
template <int I, int K, typename R>
__device__ __forceinline__ void rot_rows(R* A, R c, R s) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const R t1 = A[3 * I + j], t2 = A[3 * K + j];
        A[3 * I + j] = c * t1 - s * t2;
        A[3 * K + j] = s * t1 + c * t2;
    }
}
// A <- A G on columns I,K
template <int I, int K, typename R>
__device__ __forceinline__ void rot_cols(R* A, R c, R s) {
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const R t1 = A[3 * r + I], t2 = A[3 * r + K];
        A[3 * r + I] = c * t1 - s * t2;
        A[3 * r + K] = s * t1 + c * t2;
    }
}
template <int I, int K, typename R>
__device__ __forceinline__ void swap_cols(R* A) {
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const R t = A[3 * r + I];
        A[3 * r + I] = A[3 * r + K];
        A[3 * r + K] = t;
    }
}
template <int J, typename R>
__device__ __forceinline__ void negate_col(R* A) {
#pragma unroll
    for (int r = 0; r < 3; ++r) A[3 * r + J] = -A[3 * r + J];
}
template <typename R>
__device__ __forceinline__ void swap_r(R& a, R& b) {
    const R t = a;
    a = b;
    b = t;
}

// zero_chasing (givens.hpp:140-176)
template <typename R>
__device__ __forceinline__ void zero_chasing(R* H, R* U, R* V) {
    R c1, s1, c2, s2, c3, s3;
    givens_conventional(H[0], H[3], c1, s1);
    if (H[3] != R(0))
        givens_conventional(H[0] * H[1] + H[3] * H[4], H[0] * H[2] + H[3] * H[5], c2, s2);
    else
        givens_conventional(H[1], H[2], c2, s2);
    rot_rows<0, 1>(H, c1, s1);
    rot_cols<1, 2>(H, c2, s2);
    rot_cols<1, 2>(V, c2, s2);
    givens_conventional(H[4], H[7], c3, s3);
    rot_rows<1, 2>(H, c3, s3);
    rot_cols<0, 1>(U, c1, s1);
    rot_cols<1, 2>(U, c3, s3);
}

// qr_svd2x2 on the 2x2 block at (T,T) of B (QRSVD.hpp:25-97) followed by the
// accumulation of process<T> (QRSVD.hpp:201-222).
template <int T, typename R>
__device__ __forceinline__ void process_block(const R* B, R* U, R* S, R* V) {
    constexpr int other = (T == 1) ? 0 : 2;
    S[other] = B[4 * other];
    const R a00 = B[3 * T + T], a01 = B[3 * T + T + 1], a10 = B[3 * (T + 1) + T], a11 = B[3 * (T + 1) + T + 1];
    // polar decomposition
    R uc, us;
    {
        const R x0 = a00 + a11, x1 = a10 - a01;
        const R d2 = x0 * x0 + x1 * x1;
        if (sizeof(R) == 4 && d2 >= R(FLT_MIN)) {
            // FP32: one reciprocal square root for both quotients
            const R id = rsqrt_r(d2);
            uc = x0 * id;
            us = -x1 * id;
        } else if (d2 != R(0)) {
            const R d = sqrt(d2);
            uc = x0 / d;
            us = -x1 / d;
        } else {
            uc = R(1);
            us = R(0);
        }
    }
    // S_sym = G^T A
    const R s00 = uc * a00 - us * a10, s01 = uc * a01 - us * a11;
    const R s11 = us * a01 + uc * a11;
    R cosine, sine, S0, S1;
    const R x = s00, y = s01, z = s11;
    const R y2 = y * y;
    if (y2 == R(0)) {
        cosine = R(1);
        sine = R(0);
        S0 = x;
        S1 = z;
    } else {
        const R tau = R(0.5) * (x - z);
        const R w = sqrt(tau * tau + y2);
        const R t = div_r(y, (tau > R(0)) ? (tau + w) : (tau - w));
        cosine = rsqrt_r(t * t + R(1));
        sine = -t * cosine;
        const R c2 = cosine * cosine, csy2 = R(2) * cosine * sine * y, s2 = sine * sine;
        S0 = c2 * x - csy2 + s2 * z;
        S1 = s2 * x + csy2 + c2 * z;
    }
    R vc, vs;
    if (S0 < S1) {
        swap_r(S0, S1);
        vc = -sine;
        vs = cosine;
    } else {
        vc = cosine;
        vs = sine;
    }
    // U *= V (rotation composition)
    const R nuc = uc * vc - us * vs, nus = us * vc + uc * vs;
    S[T] = S0;
    S[T + 1] = S1;
    rot_cols<T, T + 1>(U, nuc, nus);
    rot_cols<T, T + 1>(V, vc, vs);
}

template <int J, typename R>
__device__ __forceinline__ void flip_sign(R* U, R* S) {
    S[J] = -S[J];
    negate_col<J>(U);
}

// sort_sigma<0> (QRSVD.hpp:121-155)
template <typename R>
__device__ __forceinline__ void sort_sigma0(R* U, R* S, R* V) {
    if (fabs(S[1]) >= fabs(S[2])) {
        if (S[1] < R(0)) {
            flip_sign<1>(U, S);
            flip_sign<2>(U, S);
        }
        return;
    }
    if (S[2] < R(0)) {
        flip_sign<1>(U, S);
        flip_sign<2>(U, S);
    }
    swap_r(S[1], S[2]);
    swap_cols<1, 2>(U);
    swap_cols<1, 2>(V);
    if (S[1] > S[0]) {
        swap_r(S[0], S[1]);
        swap_cols<0, 1>(U);
        swap_cols<0, 1>(V);
    } else {
        negate_col<2>(U);
        negate_col<2>(V);
    }
}
// sort_sigma<1> (QRSVD.hpp:157-198)
template <typename R>
__device__ __forceinline__ void sort_sigma1(R* U, R* S, R* V) {
    if (fabs(S[0]) >= S[1]) {
        if (S[0] < R(0)) {
            flip_sign<0>(U, S);
            flip_sign<2>(U, S);
        }
        return;
    }
    swap_r(S[0], S[1]);
    swap_cols<0, 1>(U);
    swap_cols<0, 1>(V);
    if (fabs(S[1]) < fabs(S[2])) {
        swap_r(S[1], S[2]);
        swap_cols<1, 2>(U);
        swap_cols<1, 2>(V);
    } else {
        negate_col<1>(U);
        negate_col<1>(V);
    }
    if (S[1] < R(0)) {
        flip_sign<1>(U, S);
        flip_sign<2>(U, S);
    }
}

// Returns false when the sweep limit was hit (the reference loops unbounded).
template <typename R>
__device__ __forceinline__ bool svd3(const R* A, R* U, R* S, R* V, int max_sweeps = 64) {
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        U[q] = (q % 4 == 0) ? R(1) : R(0);
        V[q] = (q % 4 == 0) ? R(1) : R(0);
    }
    R B[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) B[q] = A[q];
    // upper_bidiagonalize (givens.hpp:187-203)
    {
        R c, s;
        givens_conventional(B[3], B[6], c, s);
        rot_rows<1, 2>(B, c, s);
        rot_cols<1, 2>(U, c, s);
        zero_chasing(B, U, V);
    }
    R a0 = B[0], a1 = B[4], a2 = B[8], b0 = B[1], b1 = B[5];
    R g0 = a0 * b0, g1 = a1 * b1;
    const R eta = SvdEps<R>::value();
    const R tol = eta * fmax(R(0.5) * sqrt(a0 * a0 + a1 * a1 + a2 * a2 + b0 * b0 + b1 * b1), R(1));
    int sweeps = 0;
    bool ok = true;
    while (fabs(a0) > tol && fabs(a1) > tol && fabs(a2) > tol && fabs(b0) > tol && fabs(b1) > tol) {
        if (sweeps >= max_sweeps) {
            ok = false;
            break;
        }
        // wilkinson_shift (QRSVD.hpp:99-107)
        const R wa1 = a1 * a1 + b0 * b0, wa2 = a2 * a2 + b1 * b1;
        const R d = R(0.5) * (wa1 - wa2);
        const R bs = g1 * g1;
        const R mu = wa2 - copysign(div_r(bs, fabs(d) + sqrt(d * d + bs)), d);
        R c, s;
        givens_conventional(a0 * a0 - mu, g0, c, s);
        rot_cols<0, 1>(B, c, s);
        rot_cols<0, 1>(V, c, s);
        zero_chasing(B, U, V);
        a0 = B[0];
        a1 = B[4];
        a2 = B[8];
        b0 = B[1];
        b1 = B[5];
        g0 = a0 * b0;
        g1 = a1 * b1;
        ++sweeps;
    }
    if (!ok || fabs(b1) <= tol) {
        process_block<0>(B, U, S, V);
        sort_sigma0(U, S, V);
    } else if (fabs(b0) <= tol) {
        process_block<1>(B, U, S, V);
        sort_sigma1(U, S, V);
    } else if (fabs(a1) <= tol) {
        R c, s;
        givens_unconventional(B[5], B[8], c, s);
        rot_rows<1, 2>(B, c, s);
        rot_cols<1, 2>(U, c, s);
        process_block<0>(B, U, S, V);
        sort_sigma0(U, S, V);
    } else if (fabs(a2) <= tol) {
        R c, s;
        givens_conventional(B[4], B[5], c, s);
        rot_cols<1, 2>(B, c, s);
        rot_cols<1, 2>(V, c, s);
        givens_conventional(B[0], B[2], c, s);
        rot_cols<0, 2>(B, c, s);
        rot_cols<0, 2>(V, c, s);
        process_block<0>(B, U, S, V);
        sort_sigma0(U, S, V);
    } else {  // fabs(a0) <= tol
        R c, s;
        givens_unconventional(B[1], B[4], c, s);
        rot_rows<0, 1>(B, c, s);
        rot_cols<0, 1>(U, c, s);
        givens_unconventional(B[2], B[8], c, s);
        rot_rows<0, 2>(B, c, s);
        rot_cols<0, 2>(U, c, s);
        process_block<1>(B, U, S, V);
        sort_sigma1(U, S, V);
    }
    return ok;
}

}  // namespace gmpm
