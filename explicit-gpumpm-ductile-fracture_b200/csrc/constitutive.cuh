// Hencky-strain von Mises return mapping with hardening, tensile-energy
// history and the phase-field driving coefficient: the per-particle
// arithmetic of the reference's applyVonMises
// (ExplicitTimeIntegrator.cu:132-370, R() :64-68, computePhase_field_vol :49-62).
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

__device__ __forceinline__ float exp_r(float x) { return expf(x); }
__device__ __forceinline__ double exp_r(double x) { return exp(x); }
__device__ __forceinline__ float log_r(float x) { return logf(x); }
__device__ __forceinline__ double log_r(double x) { return log(x); }
__device__ __forceinline__ float pow_r(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double pow_r(double x, double y) { return pow(x, y); }

template <typename R, typename MR>
__device__ __forceinline__ R hardening_R(const MaterialDev<MR>& m, R alpha) {
    const R y = R(m.yield_stress);
    if (m.hardening_law == GMPM_HARDENING_LINEAR) return y + R(m.hardening) * alpha;
    const R sq = c_sqrt_p23_f<R>();
    return sq * y - (sq * y - y) / exp_r(R(m.hardening) * alpha);
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
template <typename R, typename MR>
__device__ __forceinline__ void von_mises_update(const MaterialDev<MR>& m, R V0, const R* Fin, R g, R alpha,
                                                 R c, R psi, StressOut<R>& o) {
    R A[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) A[3 * r + q] = Fin[r + 3 * q];
    R U[9], V[9], S[3];
    o.svd_ok = svd3(A, U, S, V);
    {
        const R smax = fmax(fabs(S[0]), fmax(fabs(S[1]), fabs(S[2])));
        const R smin = fmin(fabs(S[0]), fmin(fabs(S[1]), fabs(S[2])));
        o.smin_over_smax = (smax > R(0)) ? smin / smax : R(0);
    }
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
    const R divider = tsum / R(3);
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
        if (bss > R(0)) dl = y / bss;
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
        const R taudiv = tn > R(0) ? (R(1) / tn) * p23 * g * tsum * dl : R(0);
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
            if (en[k] > cap) en[k] = en[k] * (cap / nS);
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
    const R theta = R(m.theta);
    o.FP = R(4) * R(m.length_scale) * (R(1) - theta) * psi * (R(1) / Gc) + R(1);
    const R tvol = (kappa * R(0.5)) * (J * J - R(1));
    const R third = (R(1) / R(3)) * bbs;
    const R gn = c * c * (R(1) - theta) + theta;
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

}  // namespace gmpm
