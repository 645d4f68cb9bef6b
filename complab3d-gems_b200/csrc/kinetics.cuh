// kinetics.cuh -- the compiled rate laws, shared by the fused transport step (ade.cu) and the
// dissolution passes (geometry_update.cu).
#pragma once

#include "sparse.cuh"

namespace clb {

// Biotic rate laws (clb_law) over the species in internal order (mobile first), in the kinetics
// type KT (the lattice's arithmetic type: FP64 for FP64 lattices, FP32 otherwise). C holds the
// floored concentrations; R receives the species rates. The biomass of microbe m (dense FP64 field
// bio[m][N] at voxel nd; the first bn microbes from the staged copy bc, stride bstride) is read and
// floored and, with APPLY_BIO, advanced in place with its
// clamped increment (dB = max(R_B dt, -B), applied when |dB| > THRD), microbe by microbe, so no
// per-microbe array is kept. Loops over species are unrolled to the bucket NB so every array stays
// in registers.
// ft: the thermodynamic factor of the voxel (thermo_gate); below 1 it scales every substrate and
// biomass rate before the increments are formed, as run_kinetics scales them.
template <typename KT, int NB, bool APPLY_BIO>
__device__ __forceinline__ void biotic_rates(const AdeParams& P, const KT (&C)[NB], KT (&R)[NB],
                                             const double* __restrict__ bio, int64_t nd, int64_t N,
                                             const double* bc = nullptr, int bstride = 0, int bn = 0,
                                             KT ft = (KT)1) {
    const KT thr = (KT)THRD;
#pragma unroll
    for (int s = 0; s < NB; ++s) R[s] = 0;
    switch (P.law) {
        case CLB_LAW_DECAY:
#pragma unroll
            for (int s = 0; s < NB; ++s)
                if (s < P.S) R[s] = -(KT)P.prm[s] * C[s];
            break;
        case CLB_LAW_MONOD:
#pragma unroll
            for (int s = 0; s < NB; ++s)
                if (s < P.S) R[s] = -(KT)P.prm[s] * C[s] / ((KT)P.prm[CLB_MAX_SPECIES + s] + C[s]);
            break;
        case CLB_LAW_DUAL_MONOD: {
            const KT mu = (KT)P.prm[0], ks = (KT)P.prm[1], invY = (KT)(1.0 / P.prm[2]), kd = (KT)P.prm[3];
            const int don = P.donor;
            KT Cd = 0;
#pragma unroll
            for (int s = 0; s < NB; ++s)
                if (s == don) Cd = C[s];
            KT Rd = 0;
            for (int m = 0; m < P.M; ++m) {
                const int a = P.acceptor[m];
                if (a < 0) continue;
                const double* bp = bio + (int64_t)m * N + nd;
                const double braw = m < bn ? bc[m * bstride] : *bp;  // staged copy, else memory
                const KT Bm = braw < THRD ? (KT)0 : (KT)braw;
                if (Bm <= (KT)0) continue;
                KT Ca = 0;
#pragma unroll
                for (int s = 0; s < NB; ++s)
                    if (s == a) Ca = C[s];
                // mu Cd/(ks + Cd) Ca/(ks + Ca) B with one division, and 1/Y formed once: the same
                // rate to the last bits or two
                const KT growth = mu * Cd * Ca * Bm / ((ks + Cd) * (ks + Ca));
                KT rbm = growth - kd * Bm;
                if (ft < (KT)1) rbm *= ft;
                const KT gy = growth * invY;
                Rd -= gy;
#pragma unroll
                for (int s = 0; s < NB; ++s)
                    if (s == a) R[s] -= gy;
                if (APPLY_BIO) {
                    KT d = rbm * (KT)P.dt;
                    if (d > thr || d < -thr) {
                        if (d + Bm < (KT)0) d = -Bm;
                        // braw is the value in memory (staged or read above; only this thread writes
                        // this voxel's biomass in a step): the same sum as `*bp += d`, without
                        // reading the field again inside the kinetics
                        *const_cast<double*>(bp) = braw + (double)d;
                    }
                }
            }
#pragma unroll
            for (int s = 0; s < NB; ++s)
                if (s == don) R[s] += Rd;
            break;
        }
        default:
            break;
    }
    if (ft < (KT)1) {
#pragma unroll
        for (int s = 0; s < NB; ++s) R[s] *= ft;
    }
}

// The thermodynamic factor of Jin & Bethke (2003, 2005) on the floored concentrations C of the
// rate law, used as activities: a_i = max(C_i conc_scale, cmin), ln Q = sum nu_i ln a_i,
// dG = dG0 + RT ln Q + dGloss, x = (dG + m dG_ATP) / (chi RT), F_T = 0 for x >= 0, 1 for
// x < -700, else 1 - exp(x) (complab3d_thermo.hh:215-258). In the lattice's arithmetic type KT:
// FP64 for FP64 lattices, FP32 (logf, expf) otherwise.
template <typename KT, int NB>
__device__ __forceinline__ KT thermo_gate(const AdeParams& P, const KT (&C)[NB]) {
    const KT cmin = (KT)P.gate_cmin, scale = (KT)P.gate_cscale;
    KT lq = 0;
    for (int i = 0; i < P.gate_n; ++i) {
        const int sp = P.gate_sp[i];
        KT c = 0;
#pragma unroll
        for (int s = 0; s < NB; ++s)
            if (s == sp) c = C[s];
        KT a = c * scale;
        if (!(a > cmin)) a = cmin;
        lq += (KT)P.gate_nu[i] * log(a);
    }
    // x = (dG0 + RT lnQ + dGloss + atp dGatp) / (chi RT) = x0 + lnQ / chi, with the constant x0
    // formed on the host in FP64 so that FP32 lattices do not lose x to the cancellation of dG0
    // against atp dGatp near the threshold; F = -expm1(x) keeps full relative precision there
    // (1 - exp(x) would cancel as x -> 0-)
    const KT x = (KT)P.gate_x0 + lq * (KT)P.gate_inv_chi;
    if (x >= (KT)0) return (KT)0;
    if (x < (KT)-700) return (KT)1;
    const KT F = -expm1(x);
    return F < (KT)0 ? (KT)0 : (F > (KT)1 ? (KT)1 : F);
}

// Abiotic laws (clb_law CLB_LAW_PRECIP / CLB_LAW_MINERAL) over internal species indices, evaluated
// on the concentrations the biotic law left (run_abiotic_kinetics, complab3d_processors_part1.hh:
// 199-297, with the rate law of the reference's defineAbioticRxnKinetics).
// SYM: also the abiotic rate-law file (CLB_LAW_SYMBOLIC); the instantiations without it keep their
// registers.
template <int NB, bool SYM = true>
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
    } else if (SYM && P.law2 == CLB_LAW_SYMBOLIC && P.gnn_abiotic) {
        // an abiotic graph network (run_graphnet_abiotic3D, complab3d_processors_abiotic_learned.hh:
        // 200-235): a rate per species it was trained on, no growth
        const GnnNet& G = P.gnn[CLB_MAX_MICROBES];
        double x[GNN_MAX_S], y[GNN_MAX_S + 1];
        for (int i = 0; i < G.nS; ++i) {
            double xv = 0.0;
#pragma unroll
            for (int s = 0; s < NB; ++s)
                if (s == G.sp[i]) xv = C[s];
            x[i] = xv;
        }
        gnn_eval(G, x, y);
        for (int i = 0; i < G.nS; ++i) {
#pragma unroll
            for (int s = 0; s < NB; ++s)
                if (s == G.sp[i]) R[s] += y[i];
        }
    } else if (SYM && P.law2 == CLB_LAW_SYMBOLIC) {
        // an abiotic rate-law file: the extent and the species rates it derives, on the floored
        // concentrations (complab3d_processors_abiotic_learned.hh reads the same values)
        const SymProg& S = P.sym[CLB_MAX_MICROBES];
        double x[SYM_MAX_VARS], y[SYM_MAX_RATES];
        for (int v = 0; v < S.n_vars; ++v) {
            double xv = 0.0;
#pragma unroll
            for (int s = 0; s < NB; ++s)
                if (s == S.var_src[v]) xv = C[s];
            x[v] = xv;
        }
        sym_eval(S, x, y);
        for (int r = 0; r < S.n_rates; ++r) {
#pragma unroll
            for (int s = 0; s < NB; ++s)
                if (s == S.rate_dst[r]) R[s] += y[r];
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
    TC init[7];  // an untouched slot: the equilibrium at 1
    for (int i = 0; i < 7; ++i) init[i] = (TC)(q7w(i) * (1.0 - ade_sigma<TC>()));
    TC rsum[CLB_MAX_SPECIES] = {};
    for (int s = 0; s < P.S; ++s) {
        if (s < n_mobile) {
            TC pop[7];
            natural<TS, TC, 7>(S, G, g + (int64_t)s * S.SS, glink + (int64_t)s * S.SS, n, odd, init, pop);
            TC r = 0;
            for (int i = 0; i < 7; ++i) r += pop[i];
            rsum[s] = r;
            Craw[s] = (double)r + ade_sigma<TC>();
        } else {
            Craw[s] = imm[(int64_t)s * G.N + n];
        }
    }
    if (P.law == CLB_LAW_NONE) return;
    // the biotic increment exactly as the fused step computes it, in the arithmetic type
    const TC thr = (TC)THRD;
    TC C[CLB_MAX_SPECIES], R[CLB_MAX_SPECIES];
#pragma unroll
    for (int s = 0; s < CLB_MAX_SPECIES; ++s) {
        TC c = 0;
        if (s < n_mobile) c = rsum[s] + (TC)ade_sigma<TC>();
        else if (s < P.S) c = (TC)Craw[s];
        C[s] = c < thr ? (TC)0 : c;
    }
    const TC ft = (P.gate_on && P.M >= 1) ? thermo_gate<TC, CLB_MAX_SPECIES>(P, C) : (TC)1;
    biotic_rates<TC, CLB_MAX_SPECIES, false>(P, C, R, bio, n, G.N, nullptr, 0, 0, ft);
#pragma unroll
    for (int s = 0; s < CLB_MAX_SPECIES; ++s) {
        if (s >= P.S) continue;
        TC d = R[s] * (TC)P.dt;
        if (!(d > thr || d < -thr)) continue;
        if (d + C[s] < (TC)0) d = -C[s];
        if (!(d > thr || d < -thr)) continue;
        Craw[s] += (double)d;
    }
}

}  // namespace clb
