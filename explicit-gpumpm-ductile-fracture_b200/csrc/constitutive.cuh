// Hencky-strain von Mises return mapping with hardening, tensile-energy
// history and the phase-field driving coefficient: the per-particle
// arithmetic of the reference's applyVonMises
// (ExplicitTimeIntegrator.cu:132-370, R() :64-68, computePhase_field_vol :49-62),
// and the reference's two other energy models (fixed-corotated and
// Neo-Hookean with fracture, :22-47 and :372-446).
#pragma once
#include "common.cuh"
#include "svd3.cuh"

namespace gmpm {

// The reference's FP64 build rounds these two constants through float:
// parameter1 = 2.f/3.f (ExplicitTimeIntegrator.cu:190) and sqrt(2.f/3.f) in R()
// (:67).  The same values are used here in both precisions.
template <typename R> __device__ __forceinline__ R c_p23() { return R(2.0f / 3.0f); }
template <typename R> __device__ __forceinline__ R c_sqrt_p23() { return sqrt(R(2.0f / 3.0f)); }
template <typename R> __device__ __forceinline__ R c_sqrt_p23_f() { return R(sqrtf(2.0f / 3.0f)); }

// FP32 exponentials and powers on the special-function unit (__expf, __powf:
// a few ulp for the small arguments here, the exponentials of strains and of
// softening terms and J^(-2/3) with J near 1); FP64 and the FP32 logarithms
// (Hencky strains and ln J near 1, where only a relative-accurate log keeps
// the small strains) use the accurate library functions.
__device__ __forceinline__ float exp_r(float x) { return __expf(x); }
__device__ __forceinline__ double exp_r(double x) { return exp(x); }
__device__ __forceinline__ float log_r(float x) { return logf(x); }
__device__ __forceinline__ double log_r(double x) { return log(x); }
__device__ __forceinline__ float pow_r(float x, float y) { return __powf(x, y); }
__device__ __forceinline__ double pow_r(double x, double y) { return pow(x, y); }

template <typename R, typename MR>
__device__ __forceinline__ R hardening_R(const MaterialDev<MR>& m, R alpha) {
    const R y = R(m.yield_stress);
    if (m.hardening_law == GMPM_HARDENING_LINEAR) return y + R(m.hardening) * alpha;
    const R sq = c_sqrt_p23_f<R>();
    return sq * y - div_r(sq * y - y, exp_r(R(m.hardening) * alpha));
}

template <typename R>
struct StressOut {
    R F[9];       // projected F, column-major
    R sigma[6];   // V0 * P F^T: xx yy zz xy xz yz
    R alpha, psi, FP, vol;
    R smin_over_smax;
    bool svd_ok;
};

// F column-major (r + 3c).  g_old: degradation used by the trial state (the
// reference's p_g from the previous update), c: current damage.
// SVD of F (column-major) into U, S, V (row-major), with its success and
// conditioning recorded in o.
template <typename R>
__device__ __forceinline__ void svd_of(const R* Fin, R* U, R* S, R* V, StressOut<R>& o) {
    R A[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) A[3 * r + q] = Fin[r + 3 * q];
    o.svd_ok = svd3(A, U, S, V);
    const R smax = fmax(fabs(S[0]), fmax(fabs(S[1]), fabs(S[2])));
    const R smin = fmin(fabs(S[0]), fmin(fabs(S[1]), fabs(S[2])));
    o.smin_over_smax = (smax > R(0)) ? div_r(smin, smax) : R(0);
}

template <typename R, typename MR>
__device__ __forceinline__ void von_mises_from_svd(const MaterialDev<MR>& m, R V0, const R* Fin, const R* U, R* S,
                                                   const R* V, R g, R alpha, R c, R psi, StressOut<R>& o) {
    const R lambda = R(m.lambda), mu = R(m.mu), kappa = R(m.kappa);
    const R C0 = R(2) * mu + lambda, C1 = lambda;
    R eps[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) eps[k] = (S[k] > R(0)) ? log_r(S[k]) : R(0);
    R tt[3];
    tt[0] = C0 * eps[0] + C1 * eps[1] + C1 * eps[2];
    tt[1] = C1 * eps[0] + C0 * eps[1] + C1 * eps[2];
    tt[2] = C1 * eps[0] + C1 * eps[1] + C0 * eps[2];
    const R ttF = sqrt(tt[0] * tt[0] + tt[1] * tt[1] + tt[2] * tt[2]);
    const R tsum = tt[0] + tt[1] + tt[2];
    const R divider = div_r(tsum, R(3));
    R tdev[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) tdev[k] = g * (tt[k] - divider);
    const R p23 = c_p23<R>();
    const R sp23 = c_sqrt_p23<R>();
    const R y = ttF - g * hardening_R<R>(m, alpha) * sp23;
    R alpha_out = alpha;
    R F[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) F[q] = Fin[q];
    if (y >= R(1e-12)) {
        R dl = R(0);
        const R bss = p23 * g * tsum;
        if (bss > R(0)) dl = div_r(y, bss);
        if (dl > R(m.dlambda_cap)) dl = R(m.dlambda_cap);
        if (alpha < R(m.alpha_cap)) {
            alpha += sp23 * dl;
            alpha_out = alpha;
        }
        if (alpha > R(m.alpha_cap)) alpha_out = R(m.alpha_cap);
        const R tn = sqrt(tdev[0] * tdev[0] + tdev[1] * tdev[1] + tdev[2] * tdev[2]);
        // The reference divides by |tau_dev| (ExplicitTimeIntegrator.cu:242); its
        // yield test uses the full trial stress, so a hydrostatic trial state
        // (equal singular values, exact in FP32) can yield with tau_dev = 0.
        // There is no deviator to scale then: the factor is 0 instead of NaN.
        const R taudiv = tn > R(0) ? div_r(R(1), tn) * p23 * g * tsum * dl : R(0);
        const R p2 = (R(1) / R(3)) * tsum;
        R tnn[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) tnn[k] = (tdev[k] - tdev[k] * taudiv) + p2;
        R en[3];
        en[0] = R(m.D[0]) * tnn[0] + R(m.D[1]) * tnn[1] + R(m.D[2]) * tnn[2];
        en[1] = R(m.D[3]) * tnn[0] + R(m.D[4]) * tnn[1] + R(m.D[5]) * tnn[2];
        en[2] = R(m.D[6]) * tnn[0] + R(m.D[7]) * tnn[1] + R(m.D[8]) * tnn[2];
        const R nS = sqrt(en[0] * en[0] + en[1] * en[1] + en[2] * en[2]);
        const R cap = R(m.strain_cap);
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (en[k] > cap) en[k] = en[k] * div_r(cap, nS);
#pragma unroll
        for (int k = 0; k < 3; ++k) S[k] = exp_r(en[k]);
        // F = U diag(S) V^T (column-major output)
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int q = 0; q < 3; ++q)
                F[r + 3 * q] = S[0] * U[3 * r] * V[3 * q] + S[1] * U[3 * r + 1] * V[3 * q + 1] +
                               S[2] * U[3 * r + 2] * V[3 * q + 2];
    }
    const R J = S[0] * S[1] * S[2];
    const R Jbar = pow_r(J, -p23);
    R bb[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) bb[k] = Jbar * S[k] * S[k];
    const R bbs = bb[0] + bb[1] + bb[2];
    const R lnJ = (J > R(0)) ? log_r(J) : R(0);
    const R psi_vol = (kappa * R(0.5)) * (((J * J - R(1)) * R(0.5)) - lnJ);
    const R psi_dev = (mu * R(0.5)) * (bbs - R(3));
    const R psi_pos = (J < R(1)) ? psi_dev : psi_dev + psi_vol;
    if (psi_pos > psi && psi_pos < R(m.psi_cap)) psi = psi_pos;
    const R p = alpha / R(2);
    R Gc;
    if (p < R(m.softening_onset))
        Gc = R(m.fracture_energy);
    else
        Gc = R(m.fracture_energy) *
             (((R(1) - R(m.residual_fracture)) * exp_r(R(m.softening_onset) - p)) + R(m.residual_fracture));
    const R theta = R(m.theta), one_minus_theta = R(m.one_minus_theta);
    o.FP = R(4) * R(m.length_scale) * one_minus_theta * psi * div_r(R(1), Gc) + R(1);
    const R tvol = (kappa * R(0.5)) * (J * J - R(1));
    const R third = (R(1) / R(3)) * bbs;
    const R gn = c * c * one_minus_theta + theta;
    R Ph[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const R td = mu * (bb[k] - third);
        Ph[k] = (J < R(1)) ? gn * td + tvol : gn * (td + tvol);
    }
    // sigma = V0 P F^T with P = U diag(Ph) V^T and F = U diag(S) V^T, i.e.
    // V0 U diag(Ph*S) U^T; evaluated as the reference does (P then P F^T) so
    // that F from the unprojected branch enters exactly.
    R P[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q)
            P[r + 3 * q] =
                Ph[0] * U[3 * r] * V[3 * q] + Ph[1] * U[3 * r + 1] * V[3 * q + 1] + Ph[2] * U[3 * r + 2] * V[3 * q + 2];
    R sig[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q)
            sig[r + 3 * q] = (P[r] * F[q] + P[r + 3] * F[q + 3] + P[r + 6] * F[q + 6]) * V0;
    o.sigma[0] = sig[0];
    o.sigma[1] = sig[4];
    o.sigma[2] = sig[8];
    o.sigma[3] = R(0.5) * (sig[3] + sig[1]);
    o.sigma[4] = R(0.5) * (sig[6] + sig[2]);
    o.sigma[5] = R(0.5) * (sig[7] + sig[5]);
    const R det = F[0] * F[4] * F[8] + F[3] * F[7] * F[2] + F[6] * F[1] * F[5] - F[2] * F[4] * F[6] -
                  F[1] * F[3] * F[8] - F[0] * F[5] * F[7];
#pragma unroll
    for (int q = 0; q < 9; ++q) o.F[q] = F[q];
    o.alpha = alpha_out;
    o.psi = psi;
    o.vol = V0 * det;
}

// Isotropic elastic stress from singular values: P = U diag(Ph) V^T, then
// sigma = V0 P F^T (symmetric part, xx yy zz xy xz yz), evaluated as the
// reference's contribution kernels do (P, then P F^T).  F column-major.
template <typename R>
__device__ __forceinline__ void elastic_sigma(const R* U, const R* V, const R* Ph, const R* F, R V0, R* sigma6) {
    R P[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q)
            P[r + 3 * q] =
                Ph[0] * U[3 * r] * V[3 * q] + Ph[1] * U[3 * r + 1] * V[3 * q + 1] + Ph[2] * U[3 * r + 2] * V[3 * q + 2];
    R sig[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q)
            sig[r + 3 * q] = (P[r] * F[q] + P[r + 3] * F[q + 3] + P[r + 6] * F[q + 6]) * V0;
    sigma6[0] = sig[0];
    sigma6[1] = sig[4];
    sigma6[2] = sig[8];
    sigma6[3] = R(0.5) * (sig[3] + sig[1]);
    sigma6[4] = R(0.5) * (sig[6] + sig[2]);
    sigma6[5] = R(0.5) * (sig[7] + sig[5]);
}

template <typename R>
__device__ __forceinline__ R det3(const R* F) {
    return F[0] * F[4] * F[8] + F[3] * F[7] * F[2] + F[6] * F[1] * F[5] - F[2] * F[4] * F[6] - F[1] * F[3] * F[8] -
           F[0] * F[5] * F[7];
}

// J^(-2/3) in single precision: the reference evaluates it with the float
// power intrinsic.  In FP64 it is taken in double and rounded to float, the
// correctly rounded single-precision value (reproducible on the host too).
__device__ __forceinline__ float jbar_r(float J) { return powf(J, -2.0f / 3.0f); }
__device__ __forceinline__ double jbar_r(double J) { return (double)(float)pow((double)(float)J, (double)(-2.0f / 3.0f)); }

// Elastic fixed-corotated energy (computeContributionFixedCorotated,
// ExplicitTimeIntegrator.cu:22-47): Ph_k = 2 mu (S_k - 1) + lambda (J - 1)
// prod_{l != k} S_l.  No plasticity and no fracture driving (FP = 1).
template <typename R, typename MR>
__device__ __forceinline__ void fixed_corotated_from_svd(const MaterialDev<MR>& m, R V0, const R* Fin, const R* U,
                                                         const R* S, const R* V, R alpha, R psi, StressOut<R>& o) {
    const R lambda = R(m.lambda), mu = R(m.mu);
    const R J = S[0] * S[1] * S[2];
    const R smu = R(2) * mu, slam = lambda * (J - R(1));
    const R Ph[3] = {smu * (S[0] - R(1)) + slam * (S[1] * S[2]), smu * (S[1] - R(1)) + slam * (S[0] * S[2]),
                     smu * (S[2] - R(1)) + slam * (S[0] * S[1])};
    elastic_sigma(U, V, Ph, Fin, V0, o.sigma);
#pragma unroll
    for (int q = 0; q < 9; ++q) o.F[q] = Fin[q];
    o.alpha = alpha;
    o.psi = psi;
    o.FP = R(1);
    o.vol = V0 * det3(Fin);
}

// Elastic Neo-Hookean energy with the tension/compression split and the
// phase-field driving (computeContributionNeoHookean,
// ExplicitTimeIntegrator.cu:372-446): psi+ history, FP = 4 L0 (1 - 0.001)
// psi+ / G_c + 1 with G_c = 3 and L0 = dx/2, degradation
// g = c^2 (1 - 1e-4) + 1e-4 on the deviatoric (compression) or whole
// (tension) Kirchhoff stress.  The reference's psi_vol uses (J - 1)/2.
template <typename R, typename MR>
__device__ __forceinline__ void neo_hookean_fracture_from_svd(const MaterialDev<MR>& m, R V0, R dx, const R* Fin,
                                                              const R* U, const R* S, const R* V, R alpha, R c,
                                                              R psi, StressOut<R>& o) {
    const R mu = R(m.mu), kappa = R(m.kappa);
    const R J = S[0] * S[1] * S[2];
    const R Jbar = jbar_r(J);
    R bb[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) bb[k] = Jbar * S[k] * S[k];
    const R bbs = bb[0] + bb[1] + bb[2];
    const R lnJ = log_r(J);
    const R psi_vol = kappa / R(2) * ((J - R(1)) / R(2) - lnJ);
    const R psi_dev = mu / R(2) * (bb[0] + bb[1] + bb[2] - R(3));
    const R psi_pos = (J < R(1)) ? psi_dev : psi_dev + psi_vol;
    if (psi_pos > psi && psi_pos < R(1e6)) psi = psi_pos;
    const R L0 = R(0.5) * dx;
    o.FP = R(4) * L0 * R(1.f - 0.001f) * psi * R(1) / R(3) + R(1);
    const R tvol = kappa / R(2) * (J * J - R(1));
    const R third = R(1.f / 3.f) * bbs;
    const R g = c * c * R(1.f - 0.0001f) + R(0.0001f);
    R Ph[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const R td = mu * (bb[k] - third);
        Ph[k] = (J < R(1)) ? g * td + tvol : g * (td + tvol);
    }
    elastic_sigma(U, V, Ph, Fin, V0, o.sigma);
#pragma unroll
    for (int q = 0; q < 9; ++q) o.F[q] = Fin[q];
    o.alpha = alpha;
    o.psi = psi;
    o.vol = V0 * det3(Fin);
}

// The material's energy model, after one SVD of F.  kAnyModel = false
// compiles the von Mises model alone (scenes whose materials all use it).
template <typename R, typename MR, bool kAnyModel = true>
__device__ __forceinline__ void constitutive_update(const MaterialDev<MR>& m, R V0, R dx, const R* Fin, R g_old,
                                                    R alpha, R c, R psi, StressOut<R>& o) {
    R U[9], V[9], S[3];
    svd_of(Fin, U, S, V, o);
    if (!kAnyModel)
        von_mises_from_svd<R, MR>(m, V0, Fin, U, S, V, g_old, alpha, c, psi, o);
    else if (m.energy_model == GMPM_ENERGY_FIXED_COROTATED)
        fixed_corotated_from_svd<R, MR>(m, V0, Fin, U, S, V, alpha, psi, o);
    else if (m.energy_model == GMPM_ENERGY_NEO_HOOKEAN_FRACTURE)
        neo_hookean_fracture_from_svd<R, MR>(m, V0, dx, Fin, U, S, V, alpha, c, psi, o);
    else
        von_mises_from_svd<R, MR>(m, V0, Fin, U, S, V, g_old, alpha, c, psi, o);
}

}  // namespace gmpm
