// kinetics.cuh -- the compiled rate laws, shared by the fused transport step (ade.cu) and the
// dissolution passes (geometry_update.cu).
#pragma once

#include "sparse.cuh"

namespace clb {

// Rate laws (clb_law), over the species in internal order (mobile first). C and B are the
// floored concentrations / biomasses; loops are unrolled to the species bucket NB so every array
// stays in registers.
template <int NB>
__device__ __forceinline__ void eval_rates(const AdeParams& P, const double (&C)[NB], const double* B, double (&R)[NB],
                                           double* RB) {
#pragma unroll
    for (int s = 0; s < NB; ++s) R[s] = 0.0;
    switch (P.law) {
        case CLB_LAW_DECAY:
#pragma unroll
            for (int s = 0; s < NB; ++s)
                if (s < P.S) R[s] = -P.prm[s] * C[s];
            break;
        case CLB_LAW_MONOD:
#pragma unroll
            for (int s = 0; s < NB; ++s)
                if (s < P.S) R[s] = -P.prm[s] * C[s] / (P.prm[CLB_MAX_SPECIES + s] + C[s]);
            break;
        case CLB_LAW_DUAL_MONOD: {
            const double mu = P.prm[0], ks = P.prm[1], Y = P.prm[2], kd = P.prm[3];
            const int don = P.donor;
            double Cd = 0.0;
#pragma unroll
            for (int s = 0; s < NB; ++s)
                if (s == don) Cd = C[s];
            double Rd = 0.0;
            for (int m = 0; m < P.M; ++m) {
                const int a = P.acceptor[m];
                RB[m] = 0.0;
                if (a < 0) continue;
                double Ca = 0.0;
#pragma unroll
                for (int s = 0; s < NB; ++s)
                    if (s == a) Ca = C[s];
                const double Bm = B[m];
                if (Bm <= 0.0) continue;
                const double growth = mu * (Cd / (ks + Cd)) * (Ca / (ks + Ca)) * Bm;
                RB[m] += growth - kd * Bm;
                Rd -= growth / Y;
#pragma unroll
                for (int s = 0; s < NB; ++s)
                    if (s == a) R[s] -= growth / Y;
            }
#pragma unroll
            for (int s = 0; s < NB; ++s)
                if (s == don) R[s] += Rd;
            break;
        }
        default:
            break;
    }
}

// Abiotic laws (clb_law CLB_LAW_PRECIP / CLB_LAW_MINERAL) over internal species indices, evaluated
// on the concentrations the biotic law left (run_abiotic_kinetics, complab3d_processors_part1.hh:
// 199-297, with the rate law of the reference's defineAbioticRxnKinetics).
template <int NB>
__device__ __forceinline__ void eval_rates2(const AdeParams& P, const double (&C)[NB], double (&R)[NB]) {
#pragma unroll
    for (int s = 0; s < NB; ++s) R[s] = 0.0;
    if (P.law2 == CLB_LAW_PRECIP) {
        const int a = (int)P.prm2[1], b = (int)P.prm2[2], q = (int)P.prm2[3];
        double Ca = 0.0, Cb = 0.0;
#pragma unroll
        for (int s = 0; s < NB; ++s) {
            if (s == a) Ca = C[s];
            if (s == b) Cb = C[s];
        }
        const double r = P.prm2[0] * fmax(Ca, 0.0) * fmax(Cb, 0.0);
#pragma unroll
        for (int s = 0; s < NB; ++s) {
            if (s == a) R[s] -= r;
            if (s == b) R[s] -= r;
            if (s == q) R[s] += r;
        }
    } else if (P.law2 == CLB_LAW_MINERAL) {
        const int q = (int)P.prm2[2];
        double la = 0.0;
#pragma unroll
        for (int s = 0; s < NB; ++s)
            if (s < P.S && s != q && P.prm2[3 + s] != 0.0) la += P.prm2[3 + s] * log10(fmax(C[s], 1e-30));
        const double rm = P.prm2[0] * (pow(10.0, la - P.prm2[1]) - 1.0);
#pragma unroll
        for (int s = 0; s < NB; ++s) {
            if (s == q) R[s] += rm;
            else if (s < P.S) R[s] -= P.prm2[3 + s] * rm;
        }
    }
}

// Dissolution law of a sealed mineral voxel (clb_dissolution_law; the reference's
// defineDissolutionRate hook, dissolutionVOP.hh:300-320), given the water averaged over the
// voxel's open faces. subsR over internal species; mR <= 0 is the mineral's rate.
__device__ __forceinline__ void dissol_rate(const AdeParams& P, const double* water, double mineral, double* subsR,
                                            double& mR) {
    for (int s = 0; s < CLB_MAX_SPECIES; ++s) subsR[s] = 0.0;
    mR = 0.0;
    if (P.dis_law == CLB_DISSOL_FIRST_ORDER) {
        const int hs = (int)P.dprm[1];
        const double rate = P.dprm[0] * (hs >= 0 ? fmax(water[hs], 0.0) : 1.0) * fmax(mineral, 0.0);
        mR = -rate;
        for (int s = 0; s < P.S; ++s) subsR[s] = P.dprm[2 + s] * rate;
    } else if (P.dis_law == CLB_DISSOL_MINERAL) {
        double la = 0.0;
        for (int s = 0; s < P.S; ++s)
            if (s != P.sM && P.dprm[2 + s] != 0.0) la += P.dprm[2 + s] * log10(fmax(water[s], 1e-30));
        const double om = pow(10.0, la - P.dprm[1]);
        if (om < 1.0) {
            mR = P.dprm[0] * (om - 1.0);
            for (int s = 0; s < P.S; ++s)
                if (s != P.sM) subsR[s] = -P.dprm[2 + s] * mR;
        }
    }
}

// The concentrations of every species at dense voxel n (stored on the species lattices, x in
// 1..nx-2) as the abiotic processors see them: the node's density at the start of the step
// (summed in the arithmetic type in the order the fused step sums it) plus the biotic increment
// the fused step will apply there.
template <typename TS, typename TC>
__device__ void post_biotic(const AdeParams& P, const SparseView& S, const TS* g, const TS* glink,
                            const double* imm, const double* bio, int n_mobile, int64_t n, int odd,
                            double* Craw) {
    const Geom G = P.g;
    TC init[7] = {};
    for (int s = 0; s < P.S; ++s) {
        if (s < n_mobile) {
            TC pop[7];
            natural<TS, TC, 7>(S, G, g + (int64_t)s * S.SS, glink + (int64_t)s * S.SS, n, odd, init, pop);
            TC r = 0;
            for (int i = 0; i < 7; ++i) r += pop[i];
            Craw[s] = (double)r + 1.0;
        } else {
            Craw[s] = imm[(int64_t)s * G.N + n];
        }
    }
    if (P.law == CLB_LAW_NONE) return;
    double C[CLB_MAX_SPECIES], R[CLB_MAX_SPECIES], B[CLB_MAX_MICROBES], RB[CLB_MAX_MICROBES];
    for (int s = 0; s < CLB_MAX_SPECIES; ++s) C[s] = s < P.S ? (Craw[s] < THRD ? 0.0 : Craw[s]) : 0.0;
    for (int mb = 0; mb < P.M; ++mb) {
        const double b = bio[(int64_t)mb * G.N + n];
        B[mb] = b < THRD ? 0.0 : b;
    }
    eval_rates<CLB_MAX_SPECIES>(P, C, B, R, RB);
    for (int s = 0; s < P.S; ++s) {
        double d = R[s] * P.dt;
        if (!(d > THRD || d < -THRD)) continue;
        if (d + C[s] < 0.0) d = -C[s];
        if (!(d > THRD || d < -THRD)) continue;
        Craw[s] += d;
    }
}

}  // namespace clb
