// ORACLE — test infrastructure only, never the product.
//
// FP64 CPU restatement of the explicit APIC-MPM substep of
// KemengHuang/Explicit-GPUMPM-Ductile-Fracture.  Each function cites the
// reference file:line it restates (paths relative to the reference root).
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
// reference arm load this library.
//
// Canonicalisations (the reference's own choices are nondeterministic):
//   * particle order: stable sort by (page key << 6 | cell, previous slot)
//     instead of atomicAdd order (Particle_kernal.cu:167-241);
//   * page/block ids: ascending page key instead of hash/atomicAdd order
//     (Transformer_kernal.cu:49-114);
//   * P2G sums: per-page 6x6x6 tiles accumulated in sorted particle order,
//     then each grid page sums the 8 overlapping tiles in slot order 0..7.
//
// Substep order (an exact reordering of ExplicitTimeIntegrator::integrate,
// ExplicitTimeIntegrator.cu:881-994): the constitutive update applyVonMises
// that the reference runs at the start of substep n+1 is run at the end of
// G2P of substep n (it reads only G2P's outputs), plus once at scene creation.
//
// Phase field: the default (explicit) mode replaces the reference's implicit
// Jacobi-PCG solve (ExplicitTimeIntegrator.cu:909-972) with an explicit update
// of the same discrete operator (lumped mass M_L = sum V w, reaction diagonal
// sum V w (1/dt + M FP), stiffness K = sum 4 L0^2 V grad w grad w^T):
//     c_new_i = (M_L,i (c_i/dt + M) - M (K c~)_i) / (M_L,i/dt + M sum V w FP)
// where (K c~)_i = sum_p grad w_ip . q_p and q_p = 4 L0^2 V_p grad c_p, with
// grad c_p gathered in the previous G2P from the previous grid's c_new.
// The increment c_new - c_grid replaces channel 7 exactly as
// update_grid_phase does (ExplicitTimeIntegrator.cu:632-642).
#include "gmpm_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// SPGrid bit arithmetic
// ---------------------------------------------------------------------------

// Masks of SPGridMask::Cal_Masks (SPGridMask.cpp:76-129): struct_size 6,
// element_size 2 (constructor SPGridMask.h:5-8 ignores its arguments);
// element bits 2..7 (z 2-3, y 4-5, x 6-7), page bits Morton from bit 12.
void spgrid_masks(uint64_t m[3]) {
    const uint64_t struct_size = 6, element_size = 2;
    const unsigned block_bits = 6;
    const unsigned zb = block_bits / 3 + (block_bits % 3 > 0);
    const unsigned yb = block_bits / 3 + (block_bits % 3 > 1);
    const unsigned xb = block_bits / 3;
    const uint64_t ez = ((1ull << zb) - 1) << element_size;
    const uint64_t ey = ((1ull << yb) - 1) << (element_size + zb);
    const uint64_t ex = ((1ull << xb) - 1) << (element_size + zb + yb);
    const unsigned sh = 3 - struct_size % 3;
    const uint64_t pz = (0x9249249249249249ull << sh) & 0xfffffffffffff000ull;
    const uint64_t py = (0x2492492492492492ull << sh) & 0xfffffffffffff000ull;
    const uint64_t px = (0x4924924924924924ull << sh) & 0xfffffffffffff000ull;
    m[0] = px | ex;
    m[1] = py | ey;
    m[2] = pz | ez;
}

// Bit_Spread (SPGridMask.cpp:4-73): deposit consecutive data bits into the
// set bits of mask, low to high.
uint64_t bit_spread(uint64_t mask, uint64_t data) {
    uint64_t result = 0;
    for (int b = 0; b < 64; ++b) {
        const uint64_t bit = 1ull << b;
        if (mask & bit)
            result |= data & bit;
        else
            data <<= 1;
    }
    return result;
}

// Bit_Pack_Mine (TimeIntegrator.cu:26-45): gather the data bits at the set
// bits of mask into consecutive low bits.
int64_t bit_pack(uint64_t mask, uint64_t data) {
    uint64_t r = 0;
    int pos = 0;
    for (int b = 0; b < 64; ++b)
        if (mask & (1ull << b)) r |= ((data >> b) & 1ull) << pos++;
    return (int64_t)(int)r;
}

// Packed_Add (Transformer_kernal.cu:6-13).
uint64_t packed_add(const uint64_t m[3], uint64_t i, uint64_t j) {
    const uint64_t all = m[0] | m[1] | m[2];
    const uint64_t x = ((i | ~m[0]) + (j & m[0])) & m[0];
    const uint64_t y = ((i | ~m[1]) + (j & m[1])) & m[1];
    const uint64_t z = ((i | ~m[2]) + (j & m[2])) & m[2];
    const uint64_t w = ((i | all) + (j & ~all)) & ~all;
    return x | y | z | w;
}

struct Masks {
    uint64_t m[3];
    Masks() { spgrid_masks(m); }
};
const Masks& masks() {
    static Masks M;
    return M;
}

// SPGrid offset of node (i,j,k) (SPGridMask::Linear_Offset, SPGridMask.cpp:84-87).
uint64_t linear_offset(int i, int j, int k) {
    const uint64_t* m = masks().m;
    return bit_spread(m[0], (uint64_t)(int64_t)i) | bit_spread(m[1], (uint64_t)(int64_t)j) |
           bit_spread(m[2], (uint64_t)(int64_t)k);
}

// Page key of block (bx,by,bz) = offset >> 12 of its first node.
uint32_t page_key(int bx, int by, int bz) { return (uint32_t)(linear_offset(4 * bx, 4 * by, 4 * bz) >> 12); }

void page_coords(uint32_t key, int* bx, int* by, int* bz) {
    const uint64_t off = (uint64_t)key << 12;
    const uint64_t* m = masks().m;
    *bx = (int)(bit_pack(m[0], off) >> 2);
    *by = (int)(bit_pack(m[1], off) >> 2);
    *bz = (int)(bit_pack(m[2], off) >> 2);
}

// ---------------------------------------------------------------------------
// 3x3 SVD: restatement of __GEIGEN__::math::qr_svd (QRSVD.hpp:224-322) and
// the Givens machinery of givens.hpp:11-210, on a plain row-major array.
// ---------------------------------------------------------------------------

struct M3 {
    double a[3][3];
    double& operator()(int i, int j) { return a[i][j]; }
    double operator()(int i, int j) const { return a[i][j]; }
    void identity() {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) a[i][j] = (i == j) ? 1.0 : 0.0;
    }
};

struct M2 {
    double a[2][2];
};

// GivensRotation (givens.hpp:11-120).
struct Givens {
    int i, k;
    double c, s;
    Givens(int ii, int kk) : i(ii), k(kk), c(1.0), s(0.0) {}
    Givens(double a, double b, int ii, int kk) : i(ii), k(kk) { conventional(a, b); }
    // [c -s; s c] [a; b] = [*; 0]   (givens.hpp:48-59)
    void conventional(double a, double b) {
        const double d = a * a + b * b;
        c = 1.0;
        s = 0.0;
        if (d != 0.0) {
            const double t = 1.0 / std::sqrt(d);
            c = a * t;
            s = -b * t;
        }
    }
    // [c -s; s c] [a; b] = [0; *]   (givens.hpp:62-73)
    void unconventional(double a, double b) {
        const double d = a * a + b * b;
        c = 0.0;
        s = 1.0;
        if (d != 0.0) {
            const double t = 1.0 / std::sqrt(d);
            s = a * t;
            c = b * t;
        }
    }
    // A <- G^T A on rows i,k   (givens.hpp:89-101)
    void rows(M3& A) const {
        for (int j = 0; j < 3; ++j) {
            const double t1 = A(i, j), t2 = A(k, j);
            A(i, j) = c * t1 - s * t2;
            A(k, j) = s * t1 + c * t2;
        }
    }
    void rows2(M2& A) const {
        for (int j = 0; j < 2; ++j) {
            const double t1 = A.a[i][j], t2 = A.a[k][j];
            A.a[i][j] = c * t1 - s * t2;
            A.a[k][j] = s * t1 + c * t2;
        }
    }
    // A <- A G on columns i,k   (givens.hpp:104-114)
    void cols(M3& A) const {
        for (int r = 0; r < 3; ++r) {
            const double t1 = A(r, i), t2 = A(r, k);
            A(r, i) = c * t1 - s * t2;
            A(r, k) = s * t1 + c * t2;
        }
    }
    // composition (givens.hpp:117-123)
    void compose(const Givens& R) {
        const double nc = c * R.c - s * R.s;
        const double ns = s * R.c + c * R.s;
        c = nc;
        s = ns;
    }
};

// zero_chasing (givens.hpp:140-176).
void zero_chasing(M3& H, M3& U, M3& V) {
    Givens r1(H(0, 0), H(1, 0), 0, 1);
    Givens r2(1, 2);
    if (H(1, 0) != 0.0)
        r2.conventional(H(0, 0) * H(0, 1) + H(1, 0) * H(1, 1), H(0, 0) * H(0, 2) + H(1, 0) * H(1, 2));
    else
        r2.conventional(H(0, 1), H(0, 2));
    r1.rows(H);
    r2.cols(H);
    r2.cols(V);
    Givens r3(H(1, 1), H(2, 1), 1, 2);
    r3.rows(H);
    r1.cols(U);
    r3.cols(U);
}

// upper_bidiagonalize (givens.hpp:187-203).
void upper_bidiagonalize(M3& H, M3& U, M3& V) {
    U.identity();
    V.identity();
    Givens r(H(1, 0), H(2, 0), 1, 2);
    r.rows(H);
    r.cols(U);
    zero_chasing(H, U, V);
}

// polar_decomposition (QRSVD.hpp:25-45).
void polar2(const M2& A, M2& S, Givens& R) {
    S = A;
    const double x0 = A.a[0][0] + A.a[1][1], x1 = A.a[1][0] - A.a[0][1];
    const double d = std::sqrt(x0 * x0 + x1 * x1);
    if (d != 0.0) {
        R.c = x0 / d;
        R.s = -x1 / d;
    } else {
        R.c = 1.0;
        R.s = 0.0;
    }
    R.rows2(S);
}

// qr_svd2x2 (QRSVD.hpp:47-97).
void qr_svd2x2(const M2& A, double S[2], Givens& U, Givens& V) {
    M2 Ss;
    polar2(A, Ss, U);
    double cosine, sine;
    const double x = Ss.a[0][0], y = Ss.a[0][1], z = Ss.a[1][1];
    const double y2 = y * y;
    if (y2 == 0.0) {
        cosine = 1.0;
        sine = 0.0;
        S[0] = x;
        S[1] = z;
    } else {
        const double tau = 0.5 * (x - z);
        const double w = std::sqrt(tau * tau + y2);
        double t;
        if (tau > 0.0)
            t = y / (tau + w);
        else
            t = y / (tau - w);
        cosine = 1.0 / std::sqrt(t * t + 1.0);
        sine = -t * cosine;
        const double c2 = cosine * cosine;
        const double csy2 = 2.0 * cosine * sine * y;
        const double s2 = sine * sine;
        S[0] = c2 * x - csy2 + s2 * z;
        S[1] = s2 * x + csy2 + c2 * z;
    }
    if (S[0] < S[1]) {
        std::swap(S[0], S[1]);
        V.c = -sine;
        V.s = cosine;
    } else {
        V.c = cosine;
        V.s = sine;
    }
    U.compose(V);
}

// wilkinson_shift (QRSVD.hpp:99-107).
double wilkinson_shift(double a1, double b1, double a2) {
    const double d = 0.5 * (a1 - a2);
    const double bs = b1 * b1;
    return a2 - std::copysign(bs / (std::fabs(d) + std::sqrt(d * d + bs)), d);
}

void flip_sign(int j, M3& U, double S[3]) {  // QRSVD.hpp:109-115
    S[j] = -S[j];
    for (int r = 0; r < 3; ++r) U(r, j) = -U(r, j);
}
void swap_cols(M3& A, int a, int b) {
    for (int r = 0; r < 3; ++r) std::swap(A(r, a), A(r, b));
}
void negate_col(M3& A, int j) {
    for (int r = 0; r < 3; ++r) A(r, j) = -A(r, j);
}

// sort_sigma<0> / sort_sigma<1> (QRSVD.hpp:117-199).
void sort_sigma(int t, M3& U, double S[3], M3& V) {
    if (t == 0) {
        if (std::fabs(S[1]) >= std::fabs(S[2])) {
            if (S[1] < 0) {
                flip_sign(1, U, S);
                flip_sign(2, U, S);
            }
            return;
        }
        if (S[2] < 0) {
            flip_sign(1, U, S);
            flip_sign(2, U, S);
        }
        std::swap(S[1], S[2]);
        swap_cols(U, 1, 2);
        swap_cols(V, 1, 2);
        if (S[1] > S[0]) {
            std::swap(S[0], S[1]);
            swap_cols(U, 0, 1);
            swap_cols(V, 0, 1);
        } else {
            negate_col(U, 2);
            negate_col(V, 2);
        }
    } else {
        if (std::fabs(S[0]) >= S[1]) {
            if (S[0] < 0) {
                flip_sign(0, U, S);
                flip_sign(2, U, S);
            }
            return;
        }
        std::swap(S[0], S[1]);
        swap_cols(U, 0, 1);
        swap_cols(V, 0, 1);
        if (std::fabs(S[1]) < std::fabs(S[2])) {
            std::swap(S[1], S[2]);
            swap_cols(U, 1, 2);
            swap_cols(V, 1, 2);
        } else {
            negate_col(U, 1);
            negate_col(V, 1);
        }
        if (S[1] < 0) {
            flip_sign(1, U, S);
            flip_sign(2, U, S);
        }
    }
}

// process<t> (QRSVD.hpp:201-222).
void process(int t, M3& B, M3& U, double S[3], M3& V) {
    Givens u(0, 1), v(0, 1);
    const int other = (t == 1) ? 0 : 2;
    S[other] = B(other, other);
    M2 Bt;
    Bt.a[0][0] = B(t, t);
    Bt.a[0][1] = B(t, t + 1);
    Bt.a[1][0] = B(t + 1, t);
    Bt.a[1][1] = B(t + 1, t + 1);
    double S2[2];
    qr_svd2x2(Bt, S2, u, v);
    S[t] = S2[0];
    S[t + 1] = S2[1];
    u.i += t;
    u.k += t;
    v.i += t;
    v.k += t;
    u.cols(U);
    v.cols(V);
}

// qr_svd (QRSVD.hpp:224-322).  Returns the number of implicit-shift sweeps.
int qr_svd(const M3& A, double S[3], M3& U, M3& V) {
    U.identity();
    V.identity();
    M3 B = A;
    upper_bidiagonalize(B, U, V);
    Givens r(0, 1);
    double al[3] = {B(0, 0), B(1, 1), B(2, 2)};
    double be[2] = {B(0, 1), B(1, 2)};
    double ga[2] = {al[0] * be[0], al[1] * be[1]};
    const double eta = 2.220446049250313e-16 * 128.0;  // numeric_limits<double>::epsilon()*128
    const double tol =
        eta * std::max(0.5 * std::sqrt(al[0] * al[0] + al[1] * al[1] + al[2] * al[2] + be[0] * be[0] + be[1] * be[1]),
                       1.0);
    int sweeps = 0;
    while (std::fabs(al[0]) > tol && std::fabs(al[1]) > tol && std::fabs(al[2]) > tol && std::fabs(be[0]) > tol &&
           std::fabs(be[1]) > tol) {
        const double mu = wilkinson_shift(al[1] * al[1] + be[0] * be[0], ga[1], al[2] * al[2] + be[1] * be[1]);
        r.conventional(al[0] * al[0] - mu, ga[0]);
        r.cols(B);
        r.cols(V);
        zero_chasing(B, U, V);
        al[0] = B(0, 0);
        al[1] = B(1, 1);
        al[2] = B(2, 2);
        be[0] = B(0, 1);
        be[1] = B(1, 2);
        ga[0] = al[0] * be[0];
        ga[1] = al[1] * be[1];
        ++sweeps;
    }
    if (std::fabs(be[1]) <= tol) {
        process(0, B, U, S, V);
        sort_sigma(0, U, S, V);
    } else if (std::fabs(be[0]) <= tol) {
        process(1, B, U, S, V);
        sort_sigma(1, U, S, V);
    } else if (std::fabs(al[1]) <= tol) {
        Givens r1(1, 2);
        r1.unconventional(B(1, 2), B(2, 2));
        r1.rows(B);
        r1.cols(U);
        process(0, B, U, S, V);
        sort_sigma(0, U, S, V);
    } else if (std::fabs(al[2]) <= tol) {
        Givens r1(1, 2);
        r1.conventional(B(1, 1), B(1, 2));
        r1.cols(B);
        r1.cols(V);
        Givens r2(0, 2);
        r2.conventional(B(0, 0), B(0, 2));
        r2.cols(B);
        r2.cols(V);
        process(0, B, U, S, V);
        sort_sigma(0, U, S, V);
    } else if (std::fabs(al[0]) <= tol) {
        Givens r1(0, 1);
        r1.unconventional(B(0, 1), B(1, 1));
        r1.rows(B);
        r1.cols(U);
        Givens r2(0, 2);
        r2.unconventional(B(0, 2), B(2, 2));
        r2.rows(B);
        r2.cols(U);
        process(1, B, U, S, V);
        sort_sigma(1, U, S, V);
    }
    return sweeps;
}

// ---------------------------------------------------------------------------
// Constitutive update: restatement of applyVonMises
// (ExplicitTimeIntegrator.cu:132-370), R (:64-68) and Inverse (:71-129).
// ---------------------------------------------------------------------------

// Gauss-Jordan with full pivot search as in Inverse (ExplicitTimeIntegrator.cu:71-129),
// row-major 3x3.
void gauss_jordan_inverse(const double* in, double* mat) {
    for (int i = 0; i < 9; ++i) mat[i] = in[i];
    int swapR[3], swapC[3];
    int pivot[3] = {0, 0, 0};
    for (int i = 0; i < 3; ++i) {
        int pr = 0, pc = 0;
        double maxv = 0;
        for (int j = 0; j < 3; ++j)
            if (pivot[j] != 1)
                for (int k = 0; k < 3; ++k)
                    if (pivot[k] == 0 && mat[j * 3 + k] > maxv) {
                        maxv = mat[j * 3 + k];
                        pr = j;
                        pc = k;
                    }
        if (pr != pc)
            for (int j = 0; j < 3; ++j) std::swap(mat[pr * 3 + j], mat[pc * 3 + j]);
        swapC[i] = pc;
        swapR[i] = pr;
        ++pivot[i];
        const double inv = 1.0 / mat[pc * 3 + pc];
        mat[pc * 3 + pc] = 1;
        for (int j = 0; j < 3; ++j) mat[pc * 3 + j] *= inv;
        for (int j = 0; j < 3; ++j)
            if (j != pc) {
                const double ratio = mat[j * 3 + pc];
                mat[j * 3 + pc] = 0.0;
                for (int k = 0; k < 3; ++k) mat[j * 3 + k] -= mat[pc * 3 + k] * ratio;
            }
    }
    for (int i = 0; i < 3; ++i)
        if (swapR[i] != swapC[i])
            for (int j = 0; j < 3; ++j) std::swap(mat[j * 3 + swapC[i]], mat[j * 3 + swapR[i]]);
}

// Constants that the reference's FP64 build rounds through float:
//   parameter1 = 2.f / 3.f                    (ExplicitTimeIntegrator.cu:190)
//   sqrt(2.f / 3.f) inside R()                (ExplicitTimeIntegrator.cu:67)
const double kP23 = (double)(2.0f / 3.0f);
const double kSqrtP23 = std::sqrt((double)(2.0f / 3.0f));
const double kSqrtP23f = (double)std::sqrt(2.0f / 3.0f);

// Lame parameters (Materials.cpp:4-13).
void lame(double E, double nu, double* lambda, double* mu, double* kappa) {
    *lambda = E * nu / ((1 + nu) * (1 - 2 * nu));
    *mu = E / (2 * (1 + nu));
    *kappa = E / (3 * (1 - 2 * nu));
}

struct MatConsts {
    double lambda, mu, kappa;
    double D[9];  // inverse of the isotropic stiffness C
    const gmpm_material* m;
    void init(const gmpm_material* mat) {
        m = mat;
        lame(mat->youngs_modulus, mat->poisson_ratio, &lambda, &mu, &kappa);
        double C[9] = {2 * mu + lambda, lambda, lambda, lambda, 2 * mu + lambda, lambda, lambda, lambda,
                       2 * mu + lambda};
        gauss_jordan_inverse(C, D);
    }
};

// R(alpha): reference exponential law (ExplicitTimeIntegrator.cu:64-68) or linear.
double hardening_R(const gmpm_material* m, double alpha) {
    if (m->hardening_law == GMPM_HARDENING_LINEAR) return m->yield_stress + m->hardening * alpha;
    return kSqrtP23f * m->yield_stress - (kSqrtP23f * m->yield_stress - m->yield_stress) / std::exp(m->hardening * alpha);
}

struct VMOut {
    double F[9];
    double g, alpha, psi, FP, contrib[9], vol;
};

// applyVonMises for one particle.  F col-major (r + 3c).  Returns false if the
// SVD sweep count was unusual (never in practice).
void von_mises(const MatConsts& mc, double V0, const double* Fin, double g, double alpha, double c, double psi,
               VMOut& o) {
    const gmpm_material* m = mc.m;
    double F[9];
    for (int i = 0; i < 9; ++i) F[i] = Fin[i];
    // msvd(F[0], F[3], F[6], ...) passes F row by row (ExplicitTimeIntegrator.cu:144).
    M3 A, Um, Vm;
    for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc) A(r, cc) = F[r + 3 * cc];
    double S[3];
    qr_svd(A, S, Um, Vm);
    double U[9], V[9];
    for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc) {
            U[r + 3 * cc] = Um(r, cc);
            V[r + 3 * cc] = Vm(r, cc);
        }
    const double lambda = mc.lambda, mu = mc.mu, kappa = mc.kappa;
    const double C0 = 2 * mu + lambda, C1 = lambda;
    double eps[3];
    for (int k = 0; k < 3; ++k) eps[k] = (S[k] > 0.0) ? std::log(S[k]) : 0.0;
    double tau_tr[3];
    tau_tr[0] = C0 * eps[0] + C1 * eps[1] + C1 * eps[2];
    tau_tr[1] = C1 * eps[0] + C0 * eps[1] + C1 * eps[2];
    tau_tr[2] = C1 * eps[0] + C1 * eps[1] + C0 * eps[2];
    const double tau_tr_F = std::sqrt(tau_tr[0] * tau_tr[0] + tau_tr[1] * tau_tr[1] + tau_tr[2] * tau_tr[2]);
    const double tau_tr_sum = tau_tr[0] + tau_tr[1] + tau_tr[2];
    const double divider = tau_tr_sum / 3.0;
    double tau_dev_tr[3];
    for (int k = 0; k < 3; ++k) tau_dev_tr[k] = g * (tau_tr[k] - divider);
    const double y = tau_tr_F - g * hardening_R(m, alpha) * kSqrtP23;
    double alpha_out = alpha;
    if (y >= 1e-12) {  // ExplicitTimeIntegrator.cu:197-280
        double dlambda = 0.0;
        const double bss = kP23 * g * tau_tr_sum;
        if (bss > 0.0) dlambda = y / bss;
        if (dlambda > m->dlambda_cap) dlambda = m->dlambda_cap;
        if (alpha < m->alpha_cap) {
            alpha += kSqrtP23 * dlambda;
            alpha_out = alpha;
        }
        if (alpha > m->alpha_cap) alpha_out = m->alpha_cap;
        const double tn = std::sqrt(tau_dev_tr[0] * tau_dev_tr[0] + tau_dev_tr[1] * tau_dev_tr[1] +
                                    tau_dev_tr[2] * tau_dev_tr[2]);
        // ExplicitTimeIntegrator.cu:242 divides by |tau_dev|.  The yield test
        // uses the full trial stress, so a purely hydrostatic trial state can
        // yield with tau_dev = 0: there is no deviator to scale, and the factor
        // is taken as 0 where the reference would produce 0 * inf = NaN.
        const double taudiv = tn > 0.0 ? (1.0 / tn) * kP23 * g * tau_tr_sum * dlambda : 0.0;
        double tau_nn[3];
        const double p2 = (1.0 / 3.0) * tau_tr_sum;
        for (int k = 0; k < 3; ++k) tau_nn[k] = (tau_dev_tr[k] - tau_dev_tr[k] * taudiv) + p2;
        const double* D = mc.D;
        double en[3];
        en[0] = D[0] * tau_nn[0] + D[1] * tau_nn[1] + D[2] * tau_nn[2];
        en[1] = D[3] * tau_nn[0] + D[4] * tau_nn[1] + D[5] * tau_nn[2];
        en[2] = D[6] * tau_nn[0] + D[7] * tau_nn[1] + D[8] * tau_nn[2];
        const double normS = std::sqrt(en[0] * en[0] + en[1] * en[1] + en[2] * en[2]);
        for (int k = 0; k < 3; ++k)
            if (en[k] > m->strain_cap) en[k] = en[k] * (m->strain_cap / normS);
        for (int k = 0; k < 3; ++k) S[k] = std::exp(en[k]);
        for (int r = 0; r < 3; ++r)
            for (int cc = 0; cc < 3; ++cc)
                F[r + 3 * cc] = S[0] * U[r] * V[cc] + S[1] * U[r + 3] * V[cc + 3] + S[2] * U[r + 6] * V[cc + 6];
    }
    // ExplicitTimeIntegrator.cu:286-369
    const double J = S[0] * S[1] * S[2];
    const double Jbar = std::pow(J, -kP23);
    double bb[3];
    for (int k = 0; k < 3; ++k) bb[k] = Jbar * S[k] * S[k];
    const double bbs = bb[0] + bb[1] + bb[2];
    const double lnJ = (J > 0.0) ? std::log(J) : 0.0;
    const double psi_vol = (kappa * 0.5) * (((J * J - 1.0) * 0.5) - lnJ);
    const double psi_dev = (mu * 0.5) * (bb[0] + bb[1] + bb[2] - 3.0);
    const double psi_pos = (J < 1.0) ? psi_dev : psi_dev + psi_vol;
    if (psi_pos > psi && psi_pos < m->psi_cap) psi = psi_pos;
    const double p = alpha / 2;
    double Gc;
    if (p < m->softening_onset)
        Gc = m->fracture_energy;
    else
        Gc = m->fracture_energy * (((1.0 - m->residual_fracture) * std::exp(m->softening_onset - p)) +
                                   m->residual_fracture);
    // theta is a float in the reference (`float theta = 0.0001f`, :334), so
    // (1 - theta) is a single-precision difference promoted to double.
    const double theta = (double)(float)m->theta;
    const double one_minus_theta = (double)(1.0f - (float)m->theta);
    const double L0 = m->length_scale;
    const double FP = 4 * L0 * one_minus_theta * psi * (1.0 / Gc) + 1.0;
    const double tvol = (kappa * 0.5) * (J * J - 1.0);
    const double third = (1.0 / 3.0) * bbs;
    double tdev[3];
    for (int k = 0; k < 3; ++k) tdev[k] = mu * (bb[k] - third);
    const double gn = c * c * one_minus_theta + theta;
    double Ph[3];
    for (int k = 0; k < 3; ++k) Ph[k] = (J < 1.0) ? gn * tdev[k] + tvol : gn * (tdev[k] + tvol);
    double P[9];
    for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc)
            P[r + 3 * cc] = Ph[0] * U[r] * V[cc] + Ph[1] * U[r + 3] * V[cc + 3] + Ph[2] * U[r + 6] * V[cc + 6];
    // contribution(r,c) = V0 * sum_k P(r,k) F(c,k)   (ExplicitTimeIntegrator.cu:362-369)
    for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc)
            o.contrib[r + 3 * cc] =
                (P[r] * F[cc] + P[r + 3] * F[cc + 3] + P[r + 6] * F[cc + 6]) * V0;
    // computePhase_field_vol on the projected F (ExplicitTimeIntegrator.cu:49-62)
    const double det = F[0] * F[4] * F[8] + F[3] * F[7] * F[2] + F[6] * F[1] * F[5] - F[2] * F[4] * F[6] -
                       F[1] * F[3] * F[8] - F[0] * F[5] * F[7];
    for (int i = 0; i < 9; ++i) o.F[i] = F[i];
    o.g = gn;
    o.alpha = alpha_out;
    o.psi = psi;
    o.FP = FP;
    o.vol = V0 * det;
}

// P = U diag(Ph) V^T and contribution(r,c) = V0 * sum_k P(r,k) F(c,k), as the
// reference's contribution kernels (ExplicitTimeIntegrator.cu:41-46, :440-445).
// U and V column-major.
static void elastic_contribution(const double* U, const double* V, const double* Ph, const double* F, double V0,
                                 double* contrib) {
    double P[9];
    for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc)
            P[r + 3 * cc] = Ph[0] * U[r] * V[cc] + Ph[1] * U[r + 3] * V[cc + 3] + Ph[2] * U[r + 6] * V[cc + 6];
    for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc)
            contrib[r + 3 * cc] = (P[r] * F[cc] + P[r + 3] * F[cc + 3] + P[r + 6] * F[cc + 6]) * V0;
}

static void svd_colmajor(const double* F, double* U, double* S, double* V) {
    M3 A, Um, Vm;
    for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc) A(r, cc) = F[r + 3 * cc];
    qr_svd(A, S, Um, Vm);
    for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc) {
            U[r + 3 * cc] = Um(r, cc);
            V[r + 3 * cc] = Vm(r, cc);
        }
}

static double det_colmajor(const double* F) {
    return F[0] * F[4] * F[8] + F[3] * F[7] * F[2] + F[6] * F[1] * F[5] - F[2] * F[4] * F[6] - F[1] * F[3] * F[8] -
           F[0] * F[5] * F[7];
}

// computeContributionFixedCorotated (ExplicitTimeIntegrator.cu:22-47): elastic,
// no fracture driving (FP = 1); F, alpha, psi and g unchanged.
void fixed_corotated(const MatConsts& mc, double V0, const double* F, double g, double alpha, double psi, VMOut& o) {
    double U[9], V[9], S[3];
    svd_colmajor(F, U, S, V);
    const double J = S[0] * S[1] * S[2];
    const double smu = 2.0 * mc.mu, slam = mc.lambda * (J - 1.0);
    const double Ph[3] = {smu * (S[0] - 1.0) + slam * (S[1] * S[2]), smu * (S[1] - 1.0) + slam * (S[0] * S[2]),
                          smu * (S[2] - 1.0) + slam * (S[0] * S[1])};
    elastic_contribution(U, V, Ph, F, V0, o.contrib);
    for (int i = 0; i < 9; ++i) o.F[i] = F[i];
    o.g = g;
    o.alpha = alpha;
    o.psi = psi;
    o.FP = 1.0;
    o.vol = V0 * det_colmajor(F);
}

// computeContributionNeoHookean (ExplicitTimeIntegrator.cu:372-446): elastic
// Neo-Hookean with the tension/compression split; psi+ history (cap 1e6),
// FP = 4 L0 (1 - 0.001f) psi / G_c + 1 with G_c = 3 and L0 = dx/2, and
// g = c^2 (1 - 1e-4f) + 1e-4f.  J^(-2/3) is the reference's single-precision
// power, taken here as the correctly rounded float value of the double power.
void neo_hookean_fracture(const MatConsts& mc, double V0, double dx, const double* F, double alpha, double c,
                          double psi, VMOut& o) {
    double U[9], V[9], S[3];
    svd_colmajor(F, U, S, V);
    const double mu = mc.mu, kappa = mc.kappa;
    const double J = S[0] * S[1] * S[2];
    const double Jbar = (double)(float)std::pow((double)(float)J, (double)(-2.0f / 3.0f));
    double bb[3];
    for (int k = 0; k < 3; ++k) bb[k] = Jbar * S[k] * S[k];
    const double bbs = bb[0] + bb[1] + bb[2];
    const double lnJ = std::log(J);
    const double psi_vol = kappa / 2.0 * ((J - 1.0) / 2.0 - lnJ);
    const double psi_dev = mu / 2.0 * (bb[0] + bb[1] + bb[2] - 3.0);
    const double psi_pos = (J < 1.0) ? psi_dev : psi_dev + psi_vol;
    if (psi_pos > psi && psi_pos < 1e6) psi = psi_pos;
    const double L0 = 0.5 * dx;
    const double FP = 4.0 * L0 * (double)(1.f - 0.001f) * psi * 1.0 / 3.0 + 1.0;
    const double tvol = kappa / 2.0 * (J * J - 1.0);
    const double third = (double)(1.f / 3.f) * bbs;
    const double gn = c * c * (double)(1.f - 0.0001f) + (double)0.0001f;
    double Ph[3];
    for (int k = 0; k < 3; ++k) {
        const double td = mu * (bb[k] - third);
        Ph[k] = (J < 1.0) ? gn * td + tvol : gn * (td + tvol);
    }
    elastic_contribution(U, V, Ph, F, V0, o.contrib);
    for (int i = 0; i < 9; ++i) o.F[i] = F[i];
    o.g = gn;
    o.alpha = alpha;
    o.psi = psi;
    o.FP = FP;
    o.vol = V0 * det_colmajor(F);
}

// The material's energy model (gmpm_material::energy_model).
void constitutive(const MatConsts& mc, double V0, double dx, const double* F, double g, double alpha, double c,
                  double psi, VMOut& o) {
    if (mc.m->energy_model == GMPM_ENERGY_FIXED_COROTATED)
        fixed_corotated(mc, V0, F, g, alpha, psi, o);
    else if (mc.m->energy_model == GMPM_ENERGY_NEO_HOOKEAN_FRACTURE)
        neo_hookean_fracture(mc, V0, dx, F, alpha, c, psi, o);
    else
        von_mises(mc, V0, F, g, alpha, c, psi, o);
}

// ---------------------------------------------------------------------------
// Quadratic B-spline weights (P2GKernal.cu:590-611, G2PKernal.cu:263-287).
// ---------------------------------------------------------------------------
struct Weights {
    double w[3][3], g[3][3];
};
void bspline(const double xp[3], double inv_dx, Weights& W) {
    for (int v = 0; v < 3; ++v) {
        double d0 = xp[v] * inv_dx;
        double z = 1.5 - d0;
        W.w[v][0] = 0.5 * z * z;
        W.g[v][0] = -z;
        d0 = d0 - 1;
        W.w[v][1] = 0.75 - d0 * d0;
        W.g[v][1] = -d0 * 2;
        z = 1.5 - (1 - d0);
        W.w[v][2] = 0.5 * z * z;
        W.g[v][2] = z;
    }
    for (int v = 0; v < 3; ++v)
        for (int q = 0; q < 3; ++q) W.g[v][q] *= inv_dx;
}

}  // namespace

// ---------------------------------------------------------------------------
// Scene
// ---------------------------------------------------------------------------

enum { CH_M = 0, CH_P0, CH_P1, CH_P2, CH_F0, CH_F1, CH_F2, CH_CW, CH_W, CH_VW, CH_VWFP, CH_KC, NCH };

struct orc_scene {
    gmpm_scene_desc desc;
    int64_t n = 0;
    double dx = 0, inv_dx = 0;
    MatConsts mc[GMPM_MAX_MATERIALS];
    // particle state in the current (sorted) order
    std::vector<double> x, v, F, B, c, alpha, psi, g, sigma, vol, FP, gradc, mass;
    std::vector<int32_t> id, mat;
    // binning
    std::vector<uint32_t> keys;
    std::vector<int32_t> perm;
    std::vector<uint32_t> block_keys, grid_keys;
    std::vector<int32_t> block_start, cell_start, adj;
    std::vector<int32_t> block_base;  // block coords (3 per block)
    std::vector<int32_t> grid_base;   // grid block coords (3 per grid block)
    // grid results of the last substep
    std::vector<double> tile;          // NB * 216 * NCH
    std::vector<double> gv, gdc, gcn;  // per grid node: v(3), dc, c_new
    double grid_mass = 0, grid_mom[3] = {0, 0, 0};
    double time = 0;
    int64_t substeps = 0;
    double dt_max = 0;  // the scene's dt (upper bound of the adaptive step)
    uint32_t flags = 0;
    // implicit phase field: per grid node rhs, Jacobi diagonal, c_grid, tag; iterations of the last solve
    std::vector<double> pcg_b, pcg_d, pcg_cg;
    std::vector<uint8_t> pcg_tag;
    int pcg_iterations = 0;
};

namespace {

template <typename T>
void permute(std::vector<T>& a, const std::vector<int32_t>& perm, int comps) {
    std::vector<T> t(a.size());
    const int64_t n = (int64_t)perm.size();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        for (int q = 0; q < comps; ++q) t[i * comps + q] = a[(int64_t)perm[i] * comps + q];
    a.swap(t);
}

// Key of a particle's stencil base node ⌊x/dx + 0.5⌋ - 1 (cal_cellId,
// Particle_kernal.cu:158-165), with the bounds check the reference lacks.
void base_node_of(double inv_dx, const int32_t* res, const double* xp, int b[3], uint32_t* flags) {
    for (int a = 0; a < 3; ++a) {
        int i = (int)(xp[a] * inv_dx + 0.5) - 1;
        const int hi = res[a] - 3;
        if (!(xp[a] * inv_dx + 0.5 >= 1.0) || i > hi) {
            *flags |= GMPM_FLAG_OUT_OF_DOMAIN;
            i = std::min(std::max(i, 0), hi);
        }
        b[a] = i;
    }
}

void base_node(const orc_scene& s, const double* xp, int b[3], uint32_t* flags) {
    base_node_of(s.inv_dx, s.desc.grid_res, xp, b, flags);
}

uint32_t rebin(orc_scene& s) {
    const int64_t n = s.n;
    uint32_t fl = 0;
    s.keys.assign(n, 0);
#pragma omp parallel for schedule(static) reduction(| : fl)
    for (int64_t p = 0; p < n; ++p) {
        int b[3];
        uint32_t f = 0;
        base_node(s, &s.x[3 * p], b, &f);
        fl |= f;
        const uint32_t cell = (uint32_t)(((b[0] & 3) << 4) | ((b[1] & 3) << 2) | (b[2] & 3));
        s.keys[p] = (page_key(b[0] >> 2, b[1] >> 2, b[2] >> 2) << 6) | cell;
    }
    // stable counting order by (key, previous slot) — the canonical order
    std::vector<int32_t> perm(n);
    for (int64_t i = 0; i < n; ++i) perm[i] = (int32_t)i;
    std::stable_sort(perm.begin(), perm.end(), [&](int32_t a, int32_t b) { return s.keys[a] < s.keys[b]; });
    s.perm = perm;
    permute(s.keys, perm, 1);
    permute(s.x, perm, 3);
    permute(s.v, perm, 3);
    permute(s.F, perm, 9);
    permute(s.B, perm, 9);
    permute(s.c, perm, 1);
    permute(s.alpha, perm, 1);
    permute(s.psi, perm, 1);
    permute(s.g, perm, 1);
    permute(s.sigma, perm, 9);
    permute(s.vol, perm, 1);
    permute(s.FP, perm, 1);
    permute(s.gradc, perm, 3);
    permute(s.mass, perm, 1);
    permute(s.id, perm, 1);
    permute(s.mat, perm, 1);
    // pages: segment heads of key >> 6 (markPageBoundary, Transformer_kernal.cu:38-47)
    s.block_keys.clear();
    s.block_start.clear();
    for (int64_t i = 0; i < n; ++i) {
        const uint32_t pk = s.keys[i] >> 6;
        if (i == 0 || pk != (s.keys[i - 1] >> 6)) {
            s.block_keys.push_back(pk);
            s.block_start.push_back((int32_t)i);
        }
    }
    s.block_start.push_back((int32_t)n);
    const int64_t nb = (int64_t)s.block_keys.size();
    s.cell_start.assign(nb * 64 + 1, 0);
    for (int64_t b = 0; b < nb; ++b) {
        int32_t cnt[64] = {0};
        for (int32_t i = s.block_start[b]; i < s.block_start[b + 1]; ++i) cnt[s.keys[i] & 63]++;
        int32_t run = s.block_start[b];
        for (int q = 0; q < 64; ++q) {
            s.cell_start[b * 64 + q] = run;
            run += cnt[q];
        }
    }
    s.cell_start[nb * 64] = (int32_t)n;
    s.block_base.resize(3 * nb);
    for (int64_t b = 0; b < nb; ++b)
        page_coords(s.block_keys[b], &s.block_base[3 * b], &s.block_base[3 * b + 1], &s.block_base[3 * b + 2]);
    // grid pages: active pages and their +x/+y/+z neighbours
    // (supplementAdjacentPages, Transformer_kernal.cu:70-96; offsets Transformer.cpp:27-34)
    std::vector<uint32_t> gk;
    gk.reserve(nb * 8);
    for (int64_t b = 0; b < nb; ++b)
        for (int d = 0; d < 8; ++d)
            gk.push_back(page_key(s.block_base[3 * b] + (d >> 2), s.block_base[3 * b + 1] + ((d >> 1) & 1),
                                  s.block_base[3 * b + 2] + (d & 1)));
    std::sort(gk.begin(), gk.end());
    gk.erase(std::unique(gk.begin(), gk.end()), gk.end());
    s.grid_keys = gk;
    const int64_t ng = (int64_t)gk.size();
    s.grid_base.resize(3 * ng);
    for (int64_t q = 0; q < ng; ++q)
        page_coords(gk[q], &s.grid_base[3 * q], &s.grid_base[3 * q + 1], &s.grid_base[3 * q + 2]);
    // establishPageTopology (Transformer_kernal.cu:98-114), slot 4i+2j+k
    s.adj.assign(nb * 8, -1);
    for (int64_t b = 0; b < nb; ++b)
        for (int d = 0; d < 8; ++d) {
            const uint32_t k = page_key(s.block_base[3 * b] + (d >> 2), s.block_base[3 * b + 1] + ((d >> 1) & 1),
                                        s.block_base[3 * b + 2] + (d & 1));
            s.adj[b * 8 + d] = (int32_t)(std::lower_bound(gk.begin(), gk.end(), k) - gk.begin());
        }
    s.flags |= fl;
    return fl;
}

int64_t find_block(const orc_scene& s, uint32_t key) {
    auto it = std::lower_bound(s.block_keys.begin(), s.block_keys.end(), key);
    if (it == s.block_keys.end() || *it != key) return -1;
    return it - s.block_keys.begin();
}

// P2G_APIC (P2GKernal.cu:512-702) plus the phase-field channels of
// volP2G_APIC / preConditionP2G_APIC / AxP2G_APIC (P2GKernal.cu:897-1326),
// accumulated per page tile then summed per grid page in fixed slot order.
void p2g(orc_scene& s) {
    const int64_t nb = (int64_t)s.block_keys.size();
    const double dx = s.dx, inv_dx = s.inv_dx;
    const double Dinv = 4.0 * inv_dx * inv_dx;  // D_inverse (Setting.h:17)
    s.tile.assign(nb * 216 * NCH, 0.0);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t b = 0; b < nb; ++b) {
        double* T = &s.tile[b * 216 * NCH];
        for (int32_t p = s.block_start[b]; p < s.block_start[b + 1]; ++p) {
            int base[3];
            uint32_t f = 0;
            base_node(s, &s.x[3 * p], base, &f);
            double xp[3];
            for (int a = 0; a < 3; ++a) xp[a] = s.x[3 * p + a] - base[a] * dx;
            Weights W;
            bspline(xp, inv_dx, W);
            const double* sig = &s.sigma[9 * p];
            double Bm[9];
            for (int q = 0; q < 9; ++q) Bm[q] = s.B[9 * p + q] * Dinv;
            const double* vel = &s.v[3 * p];
            const double mass = s.mass[p], C = s.c[p], V = s.vol[p], fp = s.FP[p];
            const gmpm_material* m = s.mc[s.mat[p]].m;
            const double L0 = m->length_scale;
            double q4[3];
            for (int a = 0; a < 3; ++a) q4[a] = 4.0 * L0 * L0 * V * s.gradc[3 * p + a];
            const int l0 = base[0] & 3, l1 = base[1] & 3, l2 = base[2] & 3;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) {
                        const double weight = W.w[0][i] * W.w[1][j] * W.w[2][k];
                        const double wg0 = W.g[0][i] * W.w[1][j] * W.w[2][k];
                        const double wg1 = W.w[0][i] * W.g[1][j] * W.w[2][k];
                        const double wg2 = W.w[0][i] * W.w[1][j] * W.g[2][k];
                        const double d0 = i * dx - xp[0], d1 = j * dx - xp[1], d2 = k * dx - xp[2];
                        double* t = &T[((l0 + i) * 36 + (l1 + j) * 6 + (l2 + k)) * NCH];
                        t[CH_M] += mass * weight;
                        t[CH_F0] += -(sig[0] * wg0 + sig[3] * wg1 + sig[6] * wg2);
                        t[CH_F1] += -(sig[1] * wg0 + sig[4] * wg1 + sig[7] * wg2);
                        t[CH_F2] += -(sig[2] * wg0 + sig[5] * wg1 + sig[8] * wg2);
                        t[CH_CW] += weight * C;
                        t[CH_W] += weight;
                        t[CH_P0] += (vel[0] + (Bm[0] * d0 + Bm[3] * d1 + Bm[6] * d2)) * (mass * weight);
                        t[CH_P1] += (vel[1] + (Bm[1] * d0 + Bm[4] * d1 + Bm[7] * d2)) * (mass * weight);
                        t[CH_P2] += (vel[2] + (Bm[2] * d0 + Bm[5] * d1 + Bm[8] * d2)) * (mass * weight);
                        t[CH_VW] += V * weight;
                        t[CH_VWFP] += V * weight * fp;
                        t[CH_KC] += wg0 * q4[0] + wg1 * q4[1] + wg2 * q4[2];
                    }
        }
    }
}

// ---------------------------------------------------------------------------
// Implicit phase field (ExplicitTimeIntegrator.cu:909-972)
// ---------------------------------------------------------------------------

// (K x)_i = sum_p grad w_ip . col_p with col_p = 4 L0^2 V_p sum_j grad w_jp x_j
// (AxG2P_APIC, G2PKernal.cu:1006-1123, and the stiffness term of AxP2G_APIC,
// P2GKernal.cu:1162-1326), summed per page tile in sorted particle order and
// per grid node over the 8 overlapping tiles in slot order.
void stiffness_apply(const orc_scene& s, const std::vector<double>& xv, std::vector<double>& out) {
    const int64_t nb = (int64_t)s.block_keys.size(), ng = (int64_t)s.grid_keys.size();
    const double dx = s.dx, inv_dx = s.inv_dx;
    std::vector<double> tile(nb * 216, 0.0);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t b = 0; b < nb; ++b) {
        double win[216];
        for (int a = 0; a < 6; ++a)
            for (int bb = 0; bb < 6; ++bb)
                for (int cc = 0; cc < 6; ++cc) {
                    const int d = ((a >> 2) << 2) | ((bb >> 2) << 1) | (cc >> 2);
                    const int32_t g = s.adj[b * 8 + d];
                    win[a * 36 + bb * 6 + cc] = g < 0 ? 0.0 : xv[(int64_t)g * 64 + (a & 3) * 16 + (bb & 3) * 4 + (cc & 3)];
                }
        double* T = &tile[b * 216];
        for (int32_t p = s.block_start[b]; p < s.block_start[b + 1]; ++p) {
            int base[3];
            uint32_t f = 0;
            base_node(s, &s.x[3 * p], base, &f);
            double xp[3];
            for (int a = 0; a < 3; ++a) xp[a] = s.x[3 * p + a] - base[a] * dx;
            Weights W;
            bspline(xp, inv_dx, W);
            const int l0 = base[0] & 3, l1 = base[1] & 3, l2 = base[2] & 3;
            double col[3] = {0, 0, 0};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) {
                        const double xn = win[(l0 + i) * 36 + (l1 + j) * 6 + (l2 + k)];
                        col[0] += W.g[0][i] * W.w[1][j] * W.w[2][k] * xn;
                        col[1] += W.w[0][i] * W.g[1][j] * W.w[2][k] * xn;
                        col[2] += W.w[0][i] * W.w[1][j] * W.g[2][k] * xn;
                    }
            const double L0 = s.mc[s.mat[p]].m->length_scale;
            const double para = s.vol[p] * 4.0 * L0 * L0;
            for (int a = 0; a < 3; ++a) col[a] *= para;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) {
                        const double hw = W.g[0][i] * W.w[1][j] * W.w[2][k] * col[0] +
                                          W.w[0][i] * W.g[1][j] * W.w[2][k] * col[1] +
                                          W.w[0][i] * W.w[1][j] * W.g[2][k] * col[2];
                        T[(l0 + i) * 36 + (l1 + j) * 6 + (l2 + k)] += hw;
                    }
        }
    }
    out.assign(ng * 64, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < ng; ++q) {
        const int gx = s.grid_base[3 * q], gy = s.grid_base[3 * q + 1], gz = s.grid_base[3 * q + 2];
        int64_t src[8];
        for (int d = 0; d < 8; ++d) {
            const int sx = gx - (d >> 2), sy = gy - ((d >> 1) & 1), sz = gz - (d & 1);
            src[d] = (sx < 0 || sy < 0 || sz < 0) ? -1 : find_block(s, page_key(sx, sy, sz));
        }
        for (int node = 0; node < 64; ++node) {
            const int ci = node >> 4, cj = (node >> 2) & 3, ck = node & 3;
            double v = 0.0;
            for (int d = 0; d < 8; ++d) {
                if (src[d] < 0) continue;
                const int a = 4 * (d >> 2) + ci, b = 4 * ((d >> 1) & 1) + cj, c = 4 * (d & 1) + ck;
                if (a >= 6 || b >= 6 || c >= 6) continue;
                v += tile[src[d] * 216 + a * 36 + b * 6 + c];
            }
            out[q * 64 + node] = v;
        }
    }
}

// Dot product over the node vectors (myDotSum + mysumFm,
// ExplicitTimeIntegrator.cu:573-610, 727-743): partial sums over consecutive
// runs of 128 entries, combined by a sum, or by a maximum when the reference's
// quirk is selected.
double pcg_dot(const std::vector<double>& a, const std::vector<double>& b, bool max_combine) {
    const int64_t n = (int64_t)a.size();
    double total = 0.0, best = 0.0;
    bool first = true;
    for (int64_t k = 0; k < n; k += 128) {
        double part = 0.0;
        for (int64_t i = k; i < std::min(n, k + 128); ++i) part += a[i] * b[i];
        total += part;
        if (first || part > best) best = part;
        first = false;
    }
    return max_combine ? best : total;
}

// max |r| (getNormSquare_b: max of squares, then sqrt; :711-725)
double pcg_norm(const std::vector<double>& r) {
    double m = 0.0;
    for (double v : r) m = std::max(m, v * v);
    return std::sqrt(m);
}

// The reference's Jacobi-preconditioned CG (ExplicitTimeIntegrator.cu:909-972)
// for (D + M K) x = b on the tagged nodes, x0 = 0; then dc = x - c_grid
// (update_grid_phase, :632-642).
void pcg_phase_field(orc_scene& s) {
    const int64_t N = (int64_t)s.pcg_b.size();
    const double Mob = s.desc.materials[0].mobility;
    const bool qmax = s.desc.pcg_max_combine != 0;
    const int max_it = s.desc.pcg_max_iterations;
    const double tol = s.desc.pcg_tolerance;
    std::vector<double> x(N, 0.0), r(N, 0.0), mr(N, 0.0), sd(N, 0.0), q(N, 0.0), kx;
    for (int64_t i = 0; i < N; ++i)
        if (s.pcg_tag[i]) r[i] = s.pcg_b[i];
    auto precondition = [&]() {  // precondition_subd (:677-700)
        for (int64_t i = 0; i < N; ++i)
            if (s.pcg_tag[i] && std::fabs(s.pcg_d[i]) >= 1e-30) mr[i] = r[i] / s.pcg_d[i];
    };
    precondition();
    sd = mr;
    double rho_old = pcg_dot(r, mr, qmax);
    int it = 0;
    for (; it < max_it; ++it) {
        stiffness_apply(s, sd, kx);
        for (int64_t i = 0; i < N; ++i) q[i] = s.pcg_tag[i] ? s.pcg_d[i] * sd[i] + Mob * kx[i] : 0.0;
        const double sq = pcg_dot(sd, q, qmax);
        const double alpha = rho_old / sq;
        for (int64_t i = 0; i < N; ++i)
            if (s.pcg_tag[i]) {
                x[i] += sd[i] * alpha;
                r[i] = r[i] - q[i] * alpha;
            }
        if (pcg_norm(r) < tol) {
            ++it;
            break;
        }
        precondition();
        const double rho = pcg_dot(r, mr, qmax);
        if (rho_old == 0.0) {
            std::fill(x.begin(), x.end(), 1e20);
            ++it;
            break;
        }
        const double rate = rho / rho_old;
        rho_old = rho;
        for (int64_t i = 0; i < N; ++i)
            if (s.pcg_tag[i]) sd[i] = sd[i] * rate + mr[i];
    }
    s.pcg_iterations = it;
    for (int64_t i = 0; i < N; ++i)
        if (s.pcg_tag[i]) {
            s.gdc[i] = x[i] - s.pcg_cg[i];
            s.gcn[i] = x[i];
        }
}

// Grid stage for one node: undateGrid_kernal (TimeIntegrator.cu:63-111), the
// explicit phase-field update, velocity conditions (PullGrid_kernal,
// TimeIntegrator.cu:169-261, generalised) and the sticky walls of
// collideWithGround (TimeIntegrator.cu:117-165).
// Node velocity of undateGrid_kernal (TimeIntegrator.cu:63-111): v = p/m, then
// gravity (the reference's hard-coded -10 dt on y; a parameter here), then the
// force term f dt/m where it is finite.
void node_velocity(const gmpm_scene_desc& d, double mass, const double* p, const double* f, double vel[3]) {
    const double dt = d.dt;
    const double im = 1.0 / mass;
    for (int a = 0; a < 3; ++a) vel[a] = p[a] * im;
    for (int a = 0; a < 3; ++a) vel[a] += d.gravity[a] * dt;
    const double dtm = dt * im;
    for (int a = 0; a < 3; ++a) {
        const double test = f[a] * dtm;
        if (std::isfinite(test)) vel[a] += test;
    }
}

// Velocity conditions at grid node idx, in the reference's order: slabs (the
// configs' end pulls), moving spheres (PullGrid_kernal, TimeIntegrator.cu:
// 169-214, later spheres winning), then the sticky walls within wall_layers
// nodes of each face, x low/high, y, z, each zeroing all three components
// (collideWithGround, :117-165).
void velocity_conditions(const gmpm_scene_desc& d, double t_now, const int idx[3], double vel[3]) {
    const double pos[3] = {idx[0] * d.dx, idx[1] * d.dx, idx[2] * d.dx};
    for (int sb = 0; sb < d.n_slab_bcs; ++sb) {
        const gmpm_slab_bc& sl = d.slabs[sb];
        if (pos[sl.axis] >= sl.lo && pos[sl.axis] <= sl.hi)
            for (int a = 0; a < 3; ++a) vel[a] = sl.velocity[a];
    }
    for (int sp = 0; sp < d.n_sphere_bcs; ++sp) {
        const gmpm_sphere_bc& b = d.spheres[sp];
        double d2 = 0;
        for (int a = 0; a < 3; ++a) {
            const double dd = pos[a] - (b.center[a] + b.velocity[a] * t_now);
            d2 += dd * dd;
        }
        if (d2 < b.radius * b.radius)
            for (int a = 0; a < 3; ++a) vel[a] = b.velocity[a];
    }
    if (d.wall_bc) {
        const int L = d.wall_layers;
        for (int a = 0; a < 3; ++a) {
            const int N = d.grid_res[a];
            if (idx[a] <= L && vel[a] < 0.0) vel[0] = vel[1] = vel[2] = 0.0;
            if (idx[a] > N - L && vel[a] > 0.0) vel[0] = vel[1] = vel[2] = 0.0;
        }
    }
}

void grid_update(orc_scene& s) {
    const int64_t ng = (int64_t)s.grid_keys.size();
    s.gv.assign(ng * 64 * 3, 0.0);
    s.gdc.assign(ng * 64, 0.0);
    s.gcn.assign(ng * 64, 0.0);
    const double dt = s.desc.dt, t_now = s.time;
    const double Mob = s.desc.materials[0].mobility;
    const bool pf = s.desc.phase_field == GMPM_PHASE_FIELD_EXPLICIT;
    const bool pcg = s.desc.phase_field == GMPM_PHASE_FIELD_IMPLICIT;
    if (pcg) {
        s.pcg_b.assign(ng * 64, 0.0);
        s.pcg_d.assign(ng * 64, 0.0);
        s.pcg_cg.assign(ng * 64, 0.0);
        s.pcg_tag.assign(ng * 64, 0);
    }
    double gm = 0, gp0 = 0, gp1 = 0, gp2 = 0;
#pragma omp parallel for schedule(static) reduction(+ : gm, gp0, gp1, gp2)
    for (int64_t q = 0; q < ng; ++q) {
        const int gx = s.grid_base[3 * q], gy = s.grid_base[3 * q + 1], gz = s.grid_base[3 * q + 2];
        int64_t src[8];
        for (int d = 0; d < 8; ++d) {
            const int sx = gx - (d >> 2), sy = gy - ((d >> 1) & 1), sz = gz - (d & 1);
            src[d] = (sx < 0 || sy < 0 || sz < 0) ? -1 : find_block(s, page_key(sx, sy, sz));
        }
        for (int node = 0; node < 64; ++node) {
            const int ci = node >> 4, cj = (node >> 2) & 3, ck = node & 3;
            double ch[NCH];
            for (int cc = 0; cc < NCH; ++cc) ch[cc] = 0.0;
            for (int d = 0; d < 8; ++d) {
                if (src[d] < 0) continue;
                const int a = 4 * (d >> 2) + ci, b = 4 * ((d >> 1) & 1) + cj, c = 4 * (d & 1) + ck;
                if (a >= 6 || b >= 6 || c >= 6) continue;
                const double* t = &s.tile[(src[d] * 216 + a * 36 + b * 6 + c) * NCH];
                for (int cc = 0; cc < NCH; ++cc) ch[cc] += t[cc];
            }
            const int64_t gi = q * 64 + node;
            const double mass = ch[CH_M];
            if (!(mass > 0.0)) continue;  // untouched node (reference: tag <= 1e-6)
            gm += mass;
            gp0 += ch[CH_P0] + dt * ch[CH_F0];
            gp1 += ch[CH_P1] + dt * ch[CH_F1];
            gp2 += ch[CH_P2] + dt * ch[CH_F2];
            const double cgrid = ch[CH_CW] / ch[CH_W];
            double vel[3];
            node_velocity(s.desc, mass, &ch[CH_P0], &ch[CH_F0], vel);
            // explicit phase field (see file header)
            double cnew = cgrid;
            if (pf) {
                const double diag = ch[CH_VW] / dt + Mob * ch[CH_VWFP];
                const double rhs = ch[CH_VW] * (cgrid / dt + Mob) - Mob * ch[CH_KC];
                if (diag != 0.0) cnew = rhs / diag;
            }
            if (pcg) {
                // rhs sum_p V w (c_grid/dt + M) (volP2G_APIC, P2GKernal.cu:897-1030) and Jacobi
                // diagonal sum_p V w (FP M + 1/dt) (preConditionP2G_APIC, :1032-1157)
                s.pcg_b[gi] = ch[CH_VW] * (cgrid / dt + Mob);
                s.pcg_d[gi] = Mob * ch[CH_VWFP] + ch[CH_VW] / dt;
                s.pcg_cg[gi] = cgrid;
                s.pcg_tag[gi] = 1;
            }
            const int node_idx[3] = {4 * gx + ci, 4 * gy + cj, 4 * gz + ck};
            velocity_conditions(s.desc, t_now, node_idx, vel);
            for (int a = 0; a < 3; ++a) s.gv[gi * 3 + a] = vel[a];
            s.gdc[gi] = cnew - cgrid;
            s.gcn[gi] = cnew;
        }
    }
    s.grid_mass = gm;
    s.grid_mom[0] = gp0;
    s.grid_mom[1] = gp1;
    s.grid_mom[2] = gp2;
    if (pcg) pcg_phase_field(s);
}

void stress_one(orc_scene& s, int64_t p) {
    const MatConsts& mc = s.mc[s.mat[p]];
    VMOut o;
    constitutive(mc, s.desc.particle_volume, s.desc.dx, &s.F[9 * p], s.g[p], s.alpha[p], s.c[p], s.psi[p], o);
    for (int q = 0; q < 9; ++q) {
        s.F[9 * p + q] = o.F[q];
        s.sigma[9 * p + q] = o.contrib[q];
    }
    s.g[p] = o.g;
    s.alpha[p] = o.alpha;
    s.psi[p] = o.psi;
    s.FP[p] = o.FP;
    s.vol[p] = o.vol;
}

// G2P_APIC (G2PKernal.cu:204-441) plus grad c for the next phase-field flux,
// followed by the constitutive update of the next substep.
uint32_t g2p(orc_scene& s) {
    const int64_t nb = (int64_t)s.block_keys.size();
    const double dx = s.dx, inv_dx = s.inv_dx, dt = s.desc.dt;
    uint32_t fl = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(| : fl)
    for (int64_t b = 0; b < nb; ++b) {
        for (int32_t p = s.block_start[b]; p < s.block_start[b + 1]; ++p) {
            int base[3];
            uint32_t f = 0;
            base_node(s, &s.x[3 * p], base, &f);
            double xp[3];
            for (int a = 0; a < 3; ++a) xp[a] = s.x[3 * p + a] - base[a] * dx;
            Weights W;
            bspline(xp, inv_dx, W);
            const int l0 = base[0] & 3, l1 = base[1] & 3, l2 = base[2] & 3;
            double vp[3] = {0, 0, 0}, dcp = 0, gv[9] = {0}, Bn[9] = {0}, gc[3] = {0, 0, 0};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) {
                        const int a = l0 + i, bb = l1 + j, c = l2 + k;
                        const int d = ((a >> 2) << 2) | ((bb >> 2) << 1) | (c >> 2);
                        const int64_t gi = (int64_t)s.adj[b * 8 + d] * 64 + (a & 3) * 16 + (bb & 3) * 4 + (c & 3);
                        const double* nv = &s.gv[gi * 3];
                        const double w = W.w[0][i] * W.w[1][j] * W.w[2][k];
                        const double wg[3] = {W.g[0][i] * W.w[1][j] * W.w[2][k], W.w[0][i] * W.g[1][j] * W.w[2][k],
                                              W.w[0][i] * W.w[1][j] * W.g[2][k]};
                        const double dd[3] = {i * dx - xp[0], j * dx - xp[1], k * dx - xp[2]};
                        for (int r = 0; r < 3; ++r) vp[r] += w * nv[r];
                        dcp += w * s.gdc[gi];
                        for (int cc = 0; cc < 3; ++cc)
                            for (int r = 0; r < 3; ++r) {
                                gv[r + 3 * cc] += nv[r] * wg[cc];
                                Bn[r + 3 * cc] += w * nv[r] * dd[cc];
                            }
                        for (int cc = 0; cc < 3; ++cc) gc[cc] += wg[cc] * s.gcn[gi];
                    }
            for (int r = 0; r < 3; ++r) s.v[3 * p + r] = vp[r];
            const double pc = s.c[p];
            const double nc = pc + dcp;
            s.c[p] = std::max(std::min(pc, nc), 0.0);
            for (int r = 0; r < 3; ++r) s.x[3 * p + r] += vp[r] * dt;
            double A[9];
            for (int q = 0; q < 9; ++q) A[q] = gv[q] * dt;
            A[0] += 1.0;
            A[4] += 1.0;
            A[8] += 1.0;
            double Fo[9];
            const double* Fi = &s.F[9 * p];
            for (int r = 0; r < 3; ++r)
                for (int cc = 0; cc < 3; ++cc)
                    Fo[r + 3 * cc] = A[r] * Fi[3 * cc] + A[r + 3] * Fi[3 * cc + 1] + A[r + 6] * Fi[3 * cc + 2];
            for (int q = 0; q < 9; ++q) {
                s.F[9 * p + q] = Fo[q];
                s.B[9 * p + q] = Bn[q];
            }
            for (int a = 0; a < 3; ++a) s.gradc[3 * p + a] = gc[a];
            stress_one(s, p);
            for (int q = 0; q < 9; ++q)
                if (!std::isfinite(s.F[9 * p + q])) fl |= GMPM_FLAG_NONFINITE;
            for (int a = 0; a < 3; ++a)
                if (!std::isfinite(s.x[3 * p + a])) fl |= GMPM_FLAG_NONFINITE;
        }
    }
    s.flags |= fl;
    return fl;
}

int g_threads = 0;

}  // namespace

extern "C" {

void orc_masks(uint64_t out[3]) { spgrid_masks(out); }
uint64_t orc_bit_spread(uint64_t mask, int64_t data) { return bit_spread(mask, (uint64_t)data); }
uint64_t orc_linear_offset(int i, int j, int k) { return linear_offset(i, j, k); }
uint64_t orc_packed_add(uint64_t a, uint64_t b) { return packed_add(masks().m, a, b); }
int64_t orc_bit_pack(uint64_t mask, uint64_t data) { return bit_pack(mask, data); }

void orc_svd3(const double* F, double* U, double* S, double* V) {
    M3 A, Um, Vm;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) A(r, c) = F[3 * r + c];
    qr_svd(A, S, Um, Vm);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            U[3 * r + c] = Um(r, c);
            V[3 * r + c] = Vm(r, c);
        }
}

void orc_lame(double E, double nu, double* lambda, double* mu, double* kappa) { lame(E, nu, lambda, mu, kappa); }

void orc_von_mises(const gmpm_material* mat, double V0, const double* io, double* out) {
    MatConsts mc;
    mc.init(mat);
    VMOut o;
    von_mises(mc, V0, io, io[9], io[10], io[11], io[12], o);
    for (int q = 0; q < 9; ++q) out[q] = o.F[q];
    out[9] = o.g;
    out[10] = o.alpha;
    out[11] = o.psi;
    out[12] = o.FP;
    for (int q = 0; q < 9; ++q) out[13 + q] = o.contrib[q];
    out[22] = o.vol;
}

void orc_constitutive(const gmpm_material* mat, double V0, double dx, const double* io, double* out) {
    MatConsts mc;
    mc.init(mat);
    VMOut o;
    constitutive(mc, V0, dx, io, io[9], io[10], io[11], io[12], o);
    for (int q = 0; q < 9; ++q) out[q] = o.F[q];
    out[9] = o.g;
    out[10] = o.alpha;
    out[11] = o.psi;
    out[12] = o.FP;
    for (int q = 0; q < 9; ++q) out[13 + q] = o.contrib[q];
    out[22] = o.vol;
}

int orc_base_node(double inv_dx, const int32_t res[3], const double x[3], int32_t out[3]) {
    uint32_t flags = 0;
    int b[3];
    base_node_of(inv_dx, res, x, b, &flags);
    for (int a = 0; a < 3; ++a) out[a] = b[a];
    return (int)flags;
}

void orc_grid_node(const gmpm_scene_desc* desc, double t, const int32_t node[3], const double ch[9], double out[4]) {
    double vel[3];
    node_velocity(*desc, ch[0], &ch[1], &ch[4], vel);
    const int idx[3] = {node[0], node[1], node[2]};
    velocity_conditions(*desc, t, idx, vel);
    for (int a = 0; a < 3; ++a) out[a] = vel[a];
    out[3] = ch[7] / ch[8];
}

void orc_set_threads(int n) {
    g_threads = n;
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#endif
}
int orc_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

orc_scene* orc_scene_create(const gmpm_scene_desc* desc, int64_t n, const double* pos, const double* vel,
                            const double* mass, const int32_t* mat_ids) {
    if (!desc || n <= 0 || !pos || !mass) return nullptr;
    orc_scene* s = new orc_scene();
    s->desc = *desc;
    s->dt_max = desc->dt;
    s->n = n;
    s->dx = desc->dx;
    s->inv_dx = 1.0 / desc->dx;
    for (int m = 0; m < desc->n_materials && m < GMPM_MAX_MATERIALS; ++m) s->mc[m].init(&s->desc.materials[m]);
    s->x.assign(pos, pos + 3 * n);
    s->v.assign(3 * n, 0.0);
    if (vel) s->v.assign(vel, vel + 3 * n);
    s->F.assign(9 * n, 0.0);
    s->B.assign(9 * n, 0.0);
    for (int64_t p = 0; p < n; ++p) s->F[9 * p] = s->F[9 * p + 4] = s->F[9 * p + 8] = 1.0;
    s->c.assign(n, 1.0);      // initArray(d_phase_C, 1) (Particle_kernal.cu:452)
    s->alpha.assign(n, 0.0);  // (:454)
    s->psi.assign(n, 0.0);    // (:451)
    s->g.assign(n, 1.0);      // (:453)
    s->sigma.assign(9 * n, 0.0);
    s->vol.assign(n, 0.0);
    s->FP.assign(n, 1.0);
    s->gradc.assign(3 * n, 0.0);
    s->mass.assign(mass, mass + n);
    s->id.resize(n);
    s->mat.assign(n, 0);
    for (int64_t p = 0; p < n; ++p) {
        s->id[p] = (int32_t)p;
        if (mat_ids) s->mat[p] = mat_ids[p];
    }
    // initial constitutive evaluation (the reference's first applyVonMises)
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) stress_one(*s, p);
    rebin(*s);
    return s;
}

void orc_scene_destroy(orc_scene* s) { delete s; }

uint32_t orc_rebin(orc_scene* s) { return rebin(*s); }

// CFL step of MPMSimulator::computeDt (Simulator.cpp:200-225): the maximum
// particle speed (calVelSqur + mymaxF, Particle_kernal.cu:421-440) bounds dt
// by dx * 0.3f / v_max, with the scene's dt as the upper bound.
static double cfl_dt(const orc_scene& s) {
    double v2max = 0.0;
    for (int64_t p = 0; p < s.n; ++p) {
        const double* v = &s.v[3 * p];
        v2max = std::max(v2max, v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
    const double vmax = std::sqrt(v2max);
    const double cfl = s.desc.cfl_number > 0 ? s.desc.cfl_number : (double)0.3f;
    double dt = s.dt_max;
    if (vmax > 0 && (s.dx * cfl) / vmax < s.dt_max) dt = (s.dx * cfl) / vmax;
    return dt;
}

uint32_t orc_substep(orc_scene* s, int n) {
    uint32_t fl = 0;
    for (int it = 0; it < n; ++it) {
        if (s->desc.adaptive_dt) s->desc.dt = cfl_dt(*s);
        fl |= rebin(*s);
        p2g(*s);
        grid_update(*s);
        fl |= g2p(*s);
        s->time += s->desc.dt;
        s->substeps += 1;
    }
    return fl;
}

int64_t orc_num_particles(const orc_scene* s) { return s->n; }
int64_t orc_num_blocks(const orc_scene* s) { return (int64_t)s->block_keys.size(); }
int64_t orc_num_grid_blocks(const orc_scene* s) { return (int64_t)s->grid_keys.size(); }

void orc_get_field(const orc_scene* s, int field, double* out) {
    const int64_t n = s->n;
    auto copy = [&](const std::vector<double>& a) { std::memcpy(out, a.data(), a.size() * sizeof(double)); };
    switch (field) {
        case GMPM_FIELD_POSITION: copy(s->x); break;
        case GMPM_FIELD_VELOCITY: copy(s->v); break;
        case GMPM_FIELD_F: copy(s->F); break;
        case GMPM_FIELD_B: copy(s->B); break;
        case GMPM_FIELD_DAMAGE: copy(s->c); break;
        case GMPM_FIELD_ALPHA: copy(s->alpha); break;
        case GMPM_FIELD_PSI_MAX: copy(s->psi); break;
        case GMPM_FIELD_STRESS:
            for (int64_t p = 0; p < n; ++p) {
                const double* q = &s->sigma[9 * p];
                out[6 * p + 0] = q[0];
                out[6 * p + 1] = q[4];
                out[6 * p + 2] = q[8];
                out[6 * p + 3] = 0.5 * (q[3] + q[1]);
                out[6 * p + 4] = 0.5 * (q[6] + q[2]);
                out[6 * p + 5] = 0.5 * (q[7] + q[5]);
            }
            break;
        case GMPM_FIELD_VOLUME: copy(s->vol); break;
        case GMPM_FIELD_FP: copy(s->FP); break;
        case GMPM_FIELD_PF_FLUX:
            for (int64_t p = 0; p < n; ++p) {
                const double L0 = s->desc.materials[s->mat[p]].length_scale;
                for (int a = 0; a < 3; ++a) out[3 * p + a] = 4.0 * L0 * L0 * s->vol[p] * s->gradc[3 * p + a];
            }
            break;
        case GMPM_FIELD_MASS: copy(s->mass); break;
        case GMPM_FIELD_ID:
            for (int64_t p = 0; p < n; ++p) out[p] = (double)s->id[p];
            break;
        default: break;
    }
}

void orc_get_binning(const orc_scene* s, int array, void* out) {
    switch (array) {
        case GMPM_BIN_COUNTS: {
            int64_t* o = (int64_t*)out;
            o[0] = s->n;
            o[1] = (int64_t)s->block_keys.size();
            o[2] = (int64_t)s->grid_keys.size();
            o[3] = 0;
            break;
        }
        case GMPM_BIN_PERM: std::memcpy(out, s->perm.data(), s->perm.size() * 4); break;
        case GMPM_BIN_KEYS: std::memcpy(out, s->keys.data(), s->keys.size() * 4); break;
        case GMPM_BIN_BLOCK_KEYS: std::memcpy(out, s->block_keys.data(), s->block_keys.size() * 4); break;
        case GMPM_BIN_BLOCK_START: std::memcpy(out, s->block_start.data(), s->block_start.size() * 4); break;
        case GMPM_BIN_CELL_START: std::memcpy(out, s->cell_start.data(), s->cell_start.size() * 4); break;
        case GMPM_BIN_GRID_KEYS: std::memcpy(out, s->grid_keys.data(), s->grid_keys.size() * 4); break;
        case GMPM_BIN_ADJ: std::memcpy(out, s->adj.data(), s->adj.size() * 4); break;
        default: break;
    }
}

void orc_diagnostics(const orc_scene* s, gmpm_diag* d) {
    std::memset(d, 0, sizeof(*d));
    double m = 0, p0 = 0, p1 = 0, p2 = 0, ke = 0, vmax = 0, cmin = 1e300;
    for (int64_t p = 0; p < s->n; ++p) {
        const double mm = s->mass[p];
        const double* v = &s->v[3 * p];
        m += mm;
        p0 += mm * v[0];
        p1 += mm * v[1];
        p2 += mm * v[2];
        const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        ke += 0.5 * mm * v2;
        vmax = std::max(vmax, std::sqrt(v2));
        cmin = std::min(cmin, s->c[p]);
    }
    d->particle_mass = m;
    d->particle_momentum[0] = p0;
    d->particle_momentum[1] = p1;
    d->particle_momentum[2] = p2;
    d->grid_mass = s->grid_mass;
    for (int a = 0; a < 3; ++a) d->grid_momentum[a] = s->grid_mom[a];
    d->kinetic_energy = ke;
    d->max_speed = vmax;
    d->min_damage = cmin;
    d->time = s->time;
    d->substeps = s->substeps;
    d->dt = s->desc.adaptive_dt ? cfl_dt(*s) : s->desc.dt;
    d->pcg_iterations = s->pcg_iterations;
    d->n_particles = s->n;
    d->n_blocks = (int32_t)s->block_keys.size();
    d->n_grid_blocks = (int32_t)s->grid_keys.size();
    d->flags = s->flags;
}

// ---- scene set-up for the CPU legs that must not load the product library ----

// The reference's compile-time configuration as a scene description: the
// constants of Setting.h, Simulator.cpp and applyVonMises with a caller-chosen
// grid (the same values the library's gmpm_scene_desc_reference_defaults sets).
int orc_scene_desc_reference_defaults(gmpm_scene_desc* d, double dx, int rx, int ry, int rz) {
    if (!d || !(dx > 0)) return GMPM_INVALID_ARG;
    std::memset(d, 0, sizeof(*d));
    d->dx = dx;
    d->grid_res[0] = rx;
    d->grid_res[1] = ry;
    d->grid_res[2] = rz;
    d->dt = 1e-4;                      // Simulator.cpp:172
    d->gravity[1] = -10.0;             // TimeIntegrator.cu:100
    d->particle_volume = dx * dx * dx / 8.0;
    d->n_materials = 1;
    gmpm_material& m = d->materials[0];
    m.youngs_modulus = 2e2;            // Simulator.cpp:114-116
    m.poisson_ratio = 0.4;
    m.density = 3.0;
    m.yield_stress = 800.0;            // ExplicitTimeIntegrator.cu:188
    m.hardening_law = GMPM_HARDENING_EXPONENTIAL;
    m.hardening = 3.0;                 // :189
    m.alpha_cap = 1.0;                 // :194
    m.dlambda_cap = 100.0;             // :217-220
    m.strain_cap = 3.0;                // :267-271
    m.psi_cap = 1e6;                   // :313
    m.fracture_energy = 3.0;           // :317
    m.softening_onset = 0.01;          // :320
    m.residual_fracture = 0.1;         // :327
    m.theta = (double)0.0001f;         // :334
    m.length_scale = 0.5 * dx;         // :335
    m.mobility = 50.0;                 // Materials.cpp:13
    d->wall_bc = 1;
    d->wall_layers = 4;                // TimeIntegrator.cu:134-164
    d->precision = GMPM_PRECISION_FP32;
    d->phase_field = GMPM_PHASE_FIELD_EXPLICIT;
    d->deterministic = 1;
    d->svd_fallback_ratio = 1e-3;
    d->cfl_number = (double)0.3f;      // Simulator.cpp:211
    d->pcg_max_iterations = 100;       // ExplicitTimeIntegrator.cu:925
    d->pcg_tolerance = (double)1e-6f;  // :926
    return GMPM_OK;
}

// Seeded particles of the synthetic scenes: every cell of the body gets ppc
// positions drawn uniformly in the cell from one splitmix64 stream (each
// draw's top 53 bits over 2^53), rounded to float, in the order plate, x
// cell, y cell, z cell, particle, axis; the notch (kind 0) drops the cells of
// notch_width z-indices centred at mid-length with y-index below notch_depth.
int orc_generate_particles(const gmpm_scene_geometry* g, int64_t* count, double* positions, int32_t* material_ids,
                           int64_t capacity) {
    if (!g || !count || g->kind < 0 || g->kind > 2 || g->ppc <= 0 || !(g->dx > 0)) return GMPM_INVALID_ARG;
    const int plates = g->kind == 1 ? g->n_plates : 1;
    if (plates <= 0 || g->cells[0] <= 0 || g->cells[1] <= 0 || g->cells[2] <= 0) return GMPM_INVALID_ARG;
    auto notch = [&](int iy, int iz) {
        if (g->kind != 0 || g->notch_width <= 0 || g->notch_depth <= 0) return false;
        const int z0 = g->cells[2] / 2 - g->notch_width / 2;
        return iz >= z0 && iz < z0 + g->notch_width && iy < g->notch_depth;
    };
    int64_t per_plate = 0;
    for (int iy = 0; iy < g->cells[1]; ++iy)
        for (int iz = 0; iz < g->cells[2]; ++iz)
            if (!notch(iy, iz)) per_plate += (int64_t)g->cells[0] * g->ppc;
    *count = per_plate * plates;
    if (!positions) return GMPM_OK;
    if (capacity < *count) return GMPM_INVALID_ARG;
    uint64_t state = g->seed;
    auto draw = [&state]() {
        state += 0x9e3779b97f4a7c15ull;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        z ^= z >> 31;
        return (double)(z >> 11) / 9007199254740992.0;
    };
    int64_t p = 0;
    for (int k = 0; k < plates; ++k)
        for (int ix = 0; ix < g->cells[0]; ++ix)
            for (int iy = 0; iy < g->cells[1]; ++iy)
                for (int iz = 0; iz < g->cells[2]; ++iz) {
                    if (notch(iy, iz)) continue;
                    const int cell[3] = {ix, iy + k * (g->cells[1] + g->gap_cells), iz};
                    for (int q = 0; q < g->ppc; ++q, ++p) {
                        for (int a = 0; a < 3; ++a)
                            positions[3 * p + a] = (double)(float)(g->origin[a] + (cell[a] + draw()) * g->dx);
                        if (material_ids) material_ids[p] = k;
                    }
                }
    return GMPM_OK;
}

}  // extern "C"
