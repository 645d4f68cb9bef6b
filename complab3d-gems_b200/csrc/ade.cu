// ade.cu -- every species' D3Q7 advection-diffusion lattice, the kinetics and the deposit
// in one fused pass per transport step.
//
// Reference behaviour (complab.cpp:2307-2315 collide, :2340-2452 run_kinetics +
// update_rxnLattices, :3251-3259 stream; complab_functions.hh:347-442 soluteDomainSetup):
//   AdvectionDiffusionBGK: g_i <- (1-w) g_i + w t_i (rb + 4 c_i.(rho u)), t0 = 1/4, ti = 1/8,
//   w per voxel (pore or biofilm); walls and solids bounce back; x faces Dirichlet /
//   Neumann / closed; kinetics on x = 1..nx-2 where the mask is neither solid nor wall, from
//   the post-collision densities, dC = max(R dt, -C), deposited as t_i dC on the
//   post-collision populations.  BGK conserves a node's density, so the rate is evaluated
//   on the density the thread already holds: one read and one write per population.
//
// Layout: the compacted node layout of sparse.cuh over the nodes that are not bounce-back for
// the species lattices (pore and biofilm). Mobile species m (rank of the species among the mobile
// ones) occupies [m SS, (m + 1) SS) of one buffer of the storage type: its 7 population rows of
// stride KS, then its wall link slots (glink = g + 7 KS), so that every storage slot of a species
// is a 32-bit offset from the species base; AA in-place pattern as in flow.cu. Immobile species
// and biomass are dense FP64 per-voxel fields imm[s][N], bio[m][N] (they must outlive a voxel's
// change of class); the
// advection velocity u[3][K] is in the arithmetic type.
// Algorithmic bytes per node update: 2*7*sizeof(storage) per mobile species, plus the velocity
// (3*sizeof(arith)) and the material byte shared by all species.
#include "batch.cuh"
#include "flow_node.cuh"
#include "kinetics.cuh"
#include "tma.cuh"

#include <algorithm>
#include <cstring>
#include <mutex>

namespace clb {

constexpr int ADE_THREADS = 128;

// EXT: the abiotic law and the increments gathered from dissolving neighbours (AdeExtra) are
// applied after the biotic ones (complab.cpp:2460-2525).
// Kinetics of node k (dense index nd; x = 1..nx-2, mask neither solid nor wall): biotic rates with
// the clamp in the lattice's arithmetic type TC, then, with EXT, the abiotic block in FP64. Returns
// the increments of the mobile species in dC (internal species m = slot m); immobile species and
// biomass are updated in place. `bc` holds the biomass of the first `bn` microbes as staged with
// the node's gathers (stride ADE_THREADS).
// The organisms' rate laws read from .sym files (CLB_LAW_SYMBOLIC), as run_symbolic3D applies them
// (complab3d_processors_symbolic.hh:100-200), in FP64: concentrations at or below 1e-12 read as 0;
// every organism whose biomass exceeds 1e-12 evaluates its program on them (its own biomass as
// its variable), requests rate x F_T x dt of each substrate and grows by growth x F_T x biomass x
// dt (never below zero); the requests of all organisms then share each substrate's headroom: a draw
// larger than what the voxel holds takes what it holds. F_T is the gate of microbe 0's block.
template <typename TC, int NM>
__device__ __noinline__ void sym_biotic(const AdeParams& P, int n_mobile, const TC* rb, double* __restrict__ imm,
                                        double* __restrict__ bio, int64_t nd, TC* dC) {
    const int64_t N = P.g.N;
    double C[NM], req[NM];
#pragma unroll
    for (int s = 0; s < NM; ++s) {
        double c = 0.0;
        if (s < n_mobile) c = (double)rb[s] + ade_sigma<TC>();
        else if (s < P.S) c = imm[(int64_t)s * N + nd];
        C[s] = c > THRD ? c : 0.0;
        req[s] = 0.0;
    }
    for (int m = 0; m < P.M; ++m) {
        const bool net = (P.gnn_mask >> m) & 1u;
        const bool srg = (P.srg_mask >> m) & 1u;
        if (!net && !srg && !((P.sym_mask >> m) & 1u)) continue;
        const double b = bio[(int64_t)m * N + nd];
        const double bm = b > THRD ? b : 0.0;
        if (!(bm > THRD)) continue;
        if (srg) {
            // a surrogate organism (run_surrogate3D, complab3d_processors_surrogate.hh:155-250, with
            // the run-time network of surrogateModel.hh): Michaelis-Menten uptake estimates in, the
            // growth rate out; the estimates are what it draws
            const SrgNet& Q = P.srg[m];
            double fin[NM];
#pragma unroll
            for (int s = 0; s < NM; ++s) {
                fin[s] = 0.0;
                if (s >= P.S) continue;
                const double av = C[s];
                const double mm = (Q.kc[s] + av > 0.0) ? av / (Q.kc[s] + av) : 0.0;
                const double cap = -srg_exhaustion(av, bm, Q.mw, P.dt);  // >= 0
                double v = Q.vmax[s] > THRD ? Q.vmax[s] * mm : cap * mm;
                if (cap > 0.0 && v > cap) v = cap;
                fin[s] = v;
            }
            double x[SRG_MAX_IN], y[SRG_MAX_W];
            for (int i = 0; i < Q.nIn; ++i) {
                double xv = 0.0;
#pragma unroll
                for (int s = 0; s < NM; ++s)
                    if (s == Q.subs[i]) xv = fin[s];
                x[i] = xv;
            }
            srg_eval(Q, x, y);
            double mu = y[0];
            const double ft = (m == 0 && P.gate_on) ? thermo_gate<double, NM>(P, C) : 1.0;
            if (ft < 1.0) {
#pragma unroll
                for (int s = 0; s < NM; ++s) fin[s] *= ft;
                mu *= ft;
            }
            double dB = (fabs(mu) < THRD) ? -Q.kd * bm * P.dt : mu * bm * P.dt / 3600.0;
            if (dB + bm < 0.0) dB = -bm;
            if (dB > THRD || dB < -THRD) bio[(int64_t)m * N + nd] += dB;
#pragma unroll
            for (int s = 0; s < NM; ++s)
                if (s < P.S) req[s] += -(fin[s] * (bm * Q.mw) * P.dt / 3.6e6);
            continue;
        }
        if (net) {
            // a graph network (run_graphnet3D, complab3d_processors_graphnet.hh:120-170): the
            // concentrations of the species it was trained on in, a signed rate per species and
            // a growth rate out; the same budget as a rate-law file
            const GnnNet& G = P.gnn[m];
            double x[GNN_MAX_S], y[GNN_MAX_S + 1];
            for (int i = 0; i < G.nS; ++i) {
                double xv = 0.0;
#pragma unroll
                for (int s = 0; s < NM; ++s)
                    if (s == G.sp[i]) xv = C[s];
                x[i] = xv;
            }
            gnn_eval(G, x, y);
            const double ft = (m == 0 && P.gate_on) ? thermo_gate<double, NM>(P, C) : 1.0;
            for (int i = 0; i < G.nS; ++i) {
#pragma unroll
                for (int s = 0; s < NM; ++s)
                    if (s == G.sp[i]) req[s] += y[i] * ft * P.dt;
            }
            if (G.growth) {
                double dB = y[G.nS] * ft * bm * P.dt;
                if (dB > THRD || dB < -THRD) {
                    if (dB + bm < 0.0) dB = -bm;
                    bio[(int64_t)m * N + nd] += dB;
                }
            }
            continue;
        }
        const SymProg& S = P.sym[m];
        double x[SYM_MAX_VARS], y[SYM_MAX_RATES];
        for (int v = 0; v < S.n_vars; ++v) {
            const int src = S.var_src[v];
            double xv = bm;
            if (src >= 0) {
#pragma unroll
                for (int s = 0; s < NM; ++s)
                    if (s == src) xv = C[s];
            }
            x[v] = xv;
        }
        sym_eval(S, x, y);
        const double ft = (m == 0 && P.gate_on) ? thermo_gate<double, NM>(P, C) : 1.0;
        double dB = 0.0;
        for (int r = 0; r < S.n_rates; ++r) {
            const int dst = S.rate_dst[r];
            if (dst >= 0) {
#pragma unroll
                for (int s = 0; s < NM; ++s)
                    if (s == dst) req[s] += y[r] * ft * P.dt;
            } else {
                dB += y[r] * ft * bm * P.dt;
            }
        }
        if (dB > THRD || dB < -THRD) {
            if (dB + bm < 0.0) dB = -bm;
            bio[(int64_t)m * N + nd] += dB;
        }
    }
#pragma unroll
    for (int s = 0; s < NM; ++s) {
        if (s >= P.S) continue;
        double draw = req[s];
        if (!(draw > THRD || draw < -THRD)) continue;
        if (draw + C[s] < 0.0) draw = -C[s];
        if (s < n_mobile) dC[s] = (TC)draw;
        else imm[(int64_t)s * N + nd] += draw;
    }
}

template <typename TC, int NM, int EXT>
__device__ __forceinline__ void node_kinetics(const AdeParams& P, const AdeExtra& X, int64_t k, int64_t nd, int code,
                                              bool west, bool east, int n_mobile, const TC (&rb)[NM],
                                              double* __restrict__ imm, double* __restrict__ bio,
                                              const double* bc, int bn, bool hb, TC (&dC)[NM]) {
    const Geom G = P.g;
#pragma unroll
    for (int s = 0; s < NM; ++s) dC[s] = 0;
    bool sym_done = false;
    if constexpr (EXT == 2) {
        if (P.law == CLB_LAW_SYMBOLIC && !west && !east && P.react[code]) {
            // no organism acts where no biomass reaches 1e-12: every request would be zero
            if (hb) sym_biotic<TC, NM>(P, n_mobile, rb, imm, bio, nd, dC);
            sym_done = true;
        }
    }
    // dual Monod without biomass: every rate is zero, so the block is skipped (same increments)
    if (!sym_done && P.law != CLB_LAW_NONE && P.law != CLB_LAW_SYMBOLIC && (hb || P.law != CLB_LAW_DUAL_MONOD) &&
        !west && !east && P.react[code]) {
        // biotic block in the lattice's arithmetic type (FP64 lattices: FP64 throughout)
        const TC thr = (TC)THRD;
        TC C[NM], R[NM];
#pragma unroll
        for (int s = 0; s < NM; ++s) {
            TC c = 0;
            if (s < n_mobile) c = rb[s] + (TC)ade_sigma<TC>();
            else if (s < P.S) c = (TC)imm[(int64_t)s * G.N + nd];
            C[s] = c < thr ? (TC)0 : c;
        }
        // the thermodynamic gate is compiled only into the EXT instantiations
        const TC ft = (EXT && P.gate_on && P.M >= 1) ? thermo_gate<TC, NM>(P, C) : (TC)1;
        biotic_rates<TC, NM, true>(P, C, R, bio, nd, G.N, bc, ADE_THREADS, bn, ft);  // advances the biomass too
#pragma unroll
        for (int s = 0; s < NM; ++s) {
            if (s >= P.S) continue;
            TC d = R[s] * (TC)P.dt;
            if (!(d > thr || d < -thr)) continue;
            if (d + C[s] < (TC)0) d = -C[s];
            if (!(d > thr || d < -thr)) continue;
            if (s < n_mobile) dC[s] = d;
            else imm[(int64_t)s * G.N + nd] += (double)d;
        }
    }
    if (EXT && (P.law2 != CLB_LAW_NONE || P.dis_on) && !west && !east && P.react[code]) {
        // abiotic block: increments from the concentrations the biotic law left, applied once
        // (update_abiotic_rxnLattices); next to a dissolving voxel they were computed ahead of
        // the step together with the gathered products
        double T2[NM];
#pragma unroll
        for (int s = 0; s < NM; ++s) T2[s] = 0.0;
        const int xi = X.xidx[k];
        if (xi >= 0) {
#pragma unroll
            for (int s = 0; s < NM; ++s)
                if (s < P.S) T2[s] = X.xdc[(int64_t)s * X.ng + xi];
        } else if (P.law2 != CLB_LAW_NONE && (!P.surf || X.iface[k])) {
            double C[NM], R[NM];
#pragma unroll
            for (int s = 0; s < NM; ++s) {
                double c = 0.0;
                if (s < n_mobile) c = (double)rb[s] + ade_sigma<TC>() + (double)dC[s];
                else if (s < P.S) c = imm[(int64_t)s * G.N + nd];
                C[s] = c < THRD ? 0.0 : c;
            }
            eval_rates2<NM, EXT == 2>(P, C, R);
#pragma unroll
            for (int s = 0; s < NM; ++s) {
                if (s >= P.S) continue;
                double d = R[s] * P.dt;
                if (!(d > THRD || d < -THRD)) continue;
                if (d + C[s] < 0.0) d = -C[s];
                if (!(d > THRD || d < -THRD)) continue;
                T2[s] = d;
            }
        }
#pragma unroll
        for (int s = 0; s < NM; ++s) {
            if (s >= P.S) continue;
            const double d = T2[s];
            if (!(d > THRD || d < -THRD)) continue;
            if (s < n_mobile) dC[s] += (TC)d;
            else imm[(int64_t)s * G.N + nd] += d;
        }
    }
}

// The per-node metadata a transport step reads before its gathers: material code, wall / box-edge
// masks with the link base residual, and (odd steps) the neighbour-row residuals. Loaded one node
// ahead by the pipelined step.
struct AdeMeta {
    int code;
    uint32_t mt;
    int2 dv;
    int nd;  // dense index of the voxel (per-voxel fields, boundary planes)
    int hb;  // 1: biomass may act at the node (AdeParams::bflag)
};

template <bool ODD>
__device__ __forceinline__ AdeMeta ade_meta(const SparseView& S, int64_t k, const uint8_t* __restrict__ bflag) {
    AdeMeta M;
    M.code = S.code[k];
    M.mt = S.meta[k];
    M.dv = ODD ? *reinterpret_cast<const int2*>(S.dres + 4 * k) : make_int2(0, 0);
    M.nd = S.node[k];
    M.hb = bflag ? bflag[k] : 1;
    return M;
}

// compact index of the source node a - c_i of each population on an odd step (from the
// per-tile row bases and the node's residuals dv)
__device__ __forceinline__ void odd_sources(const SparseView& S, int64_t k, int2 dv, int (&nb)[7]) {
    const int t = (int)(k >> 8);
    const int* tb = S.tdb + 4 * t;
    nb[0] = (int)k;
    nb[1] = (int)k + tb[0] + (int16_t)(dv.x & 0xFFFF);           // -x population comes from x+1
    nb[4] = (int)k + tb[1] + (int16_t)((uint32_t)dv.x >> 16);    // +x from x-1
    nb[2] = (int)k + tb[2] + (int16_t)(dv.y & 0xFFFF);           // -y from y+1
    nb[5] = (int)k + tb[3] + (int16_t)((uint32_t)dv.y >> 16);    // +y from y-1
    nb[3] = (int)k + 1;
    nb[6] = (int)k - 1;
}

constexpr int ADE_RESIDENT = 4;       // resident blocks per SM the carveout is sized for (odd step)
constexpr int ADE_RESIDENT_EVEN = 5;  // the even step reads only its own slots: less L1, more blocks

// What travels with a node's gathers besides its populations: with 4-byte arithmetic the velocity
// and the biomass of up to two microbes; FP64 slots already fill the shared memory three blocks
// can have, so FP64 reads both from memory where it uses them.
template <typename TC>
constexpr int ade_bio_cache() { return sizeof(TC) == 4 ? 2 : 0; }
template <typename TC>
constexpr int ade_u_staged() { return sizeof(TC) == 4 ? 3 : 0; }

// Shared memory of a CTA of the transport step, per thread (stride ADE_THREADS): the staged
// biomass (FP64), NM x 7 population slots and the staged velocity (the arithmetic type), and the
// 7 population offsets. What a node needs from memory beyond its metadata is staged here by
// asynchronous copies issued together, so one wait covers them all.
template <typename TC, int NM>
constexpr int ade_slot_bytes() {
    return ade_bio_cache<TC>() * ADE_THREADS * (int)sizeof(double) +
           (NM * 7 + ade_u_staged<TC>()) * ADE_THREADS * (int)sizeof(TC) + 7 * ADE_THREADS * (int)sizeof(uint32_t);
}

template <typename TC>
struct AdeFrame {
    double* bio;    // [ade_bio_cache]
    TC* pop;        // [NM * 7]
    TC* u;          // [3]
    uint32_t* off;  // [7]
};

// the calling thread's slots in slot set `set` of the CTA's shared memory
template <typename TC, int NM>
__device__ __forceinline__ AdeFrame<TC> ade_frame(unsigned char* smem, int set) {
    unsigned char* b = smem + (size_t)set * ade_slot_bytes<TC, NM>();
    const int t = threadIdx.x;
    AdeFrame<TC> F;
    F.bio = reinterpret_cast<double*>(b) + t;
    b += ade_bio_cache<TC>() * ADE_THREADS * sizeof(double);
    F.pop = reinterpret_cast<TC*>(b) + t;
    b += NM * 7 * ADE_THREADS * sizeof(TC);
    F.u = reinterpret_cast<TC*>(b) + t;
    b += ade_u_staged<TC>() * ADE_THREADS * sizeof(TC);
    F.off = reinterpret_cast<uint32_t*>(b) + t;
    return F;
}

// resident blocks per SM the shared slots allow (about 200 KB of shared memory per SM), at most 8
template <typename TC, int NM>
constexpr int ade_minb() {
    constexpr int b = (200 * 1024) / ade_slot_bytes<TC, NM>();
    return b < 1 ? 1 : (b > 8 ? 8 : b);
}

// One thread per node. The populations of all species pass through the thread's own slots of
// shared memory (NM x 7 x ADE_THREADS values of the arithmetic type) between the gather and the
// collision, so registers hold only the per-species sums and increments and many warps stay
// resident to hide memory latency.
// One node of the transport step (all species of compact node k) in two halves: ade_gather
// (slot offsets, then every species' incoming populations, the node's velocity and biomass into
// the calling thread's shared-memory frame F, by asynchronous copies where the element is 4 or
// 8 bytes) and ade_finish (boundary completion, kinetics, collision, deposit, scatter). Shared by
// the single-domain, the pipelined and the batched steps.
//
// Both AA steps are in-place permutations of 7 storage slots per node that every species shares:
// incoming j is read from slot j and outgoing opp(j) is written back to slot j. Even step: slot j is
// the node's own row j, or, for a wall link (a, i) with j = opp(i), the link's even-step slot X.
// Odd step: slot j is row opp(j) of the source node a - c_j, or the node's own row j when that
// source is a wall or outside the box. The offsets (from the species base, link slots at 7 KS +
// link index) are computed once per node and serve the gathers and the scatters of every species.

// Returns the mask of the species gathered (those that collide and stream at this node); a
// bounce-back node (a voxel sealed by precipitation: the identity on AA slots) gathers nothing.
template <typename TS, typename TC, bool ODD, int NM, typename AP>
__device__ __forceinline__ uint32_t ade_gather(TS* __restrict__ g, const TC* __restrict__ u,
                                               const double* __restrict__ bio, const SparseView& S, const AP& P,
                                               int n_mobile, const int* __restrict__ mob_species,
                                               int64_t k_west_end, int64_t k_east_begin, const AdeFrame<TC>& F,
                                               int64_t k, const AdeMeta& M) {
    constexpr int T = ADE_THREADS;
    if (P.dyn[M.code] == ADE_BB) return 0u;
    const uint32_t K32 = (uint32_t)S.KS;  // row stride; SS < 2^31 is checked when the layout is built
    const bool west = k < k_west_end, east = k >= k_east_begin;
    const uint32_t wm = M.mt & 0x7Fu;
    const uint32_t blk = wm | ((M.mt >> 7) & 0x7Fu);  // wall or outside the box
    uint32_t off[7];
    if (!ODD) {
        const uint32_t lb = 7u * K32 + (uint32_t)(S.tlb[(int)(k >> 8)] + (int)(M.mt >> 14));
#pragma unroll
        for (int i = 0; i < 7; ++i) {
            const int oi = q7opp(i);
            off[i] = (i != 0 && ((wm >> oi) & 1u)) ? lb + (uint32_t)__popc(wm & ((1u << oi) - 1u))
                                                   : (uint32_t)(i * K32) + (uint32_t)k;
        }
    } else {
        int nb[7];  // compact index of the source node a - c_i
        odd_sources(S, k, M.dv, nb);
        off[0] = (uint32_t)k;
#pragma unroll
        for (int i = 1; i < 7; ++i) {
            const int oi = q7opp(i);
            off[i] = ((blk >> oi) & 1u) ? (uint32_t)(i * K32) + (uint32_t)k : (uint32_t)(oi * K32) + (uint32_t)nb[i];
        }
    }
#pragma unroll
    for (int i = 0; i < 7; ++i) F.off[i * T] = off[i];
    uint32_t actm = 0;
#pragma unroll
    for (int m = 0; m < NM; ++m) {
        if (m >= n_mobile) continue;
        const int s = m;  // internal order puts the mobile species first: mobile slot m is species m
        if ((west && P.ltype[s] == CLB_CLOSED) || (east && P.rtype[s] == CLB_CLOSED)) continue;  // bounce-back
        actm |= 1u << m;
        const TS* f = g + (int64_t)m * S.SS;
        TC* slot = F.pop + (m * 7) * T;
        if constexpr (sizeof(TS) >= 4) {
            // 4- and 8-byte populations go straight to the slots as asynchronous copies, so a
            // thread has all of its loads in flight at once without holding them in registers
#pragma unroll
            for (int i = 0; i < 7; ++i) cp_async<sizeof(TS)>(slot + i * T, f + off[i]);
        } else {
#pragma unroll
            for (int i = 0; i < 7; ++i) slot[i * T] = ld<TS, TC>(f + off[i]);
        }
    }
    // the velocity and the biomass the kinetics reads travel with the populations
    const int64_t K = S.K;
    if constexpr (ade_u_staged<TC>() == 3) {
        cp_async<sizeof(TC)>(F.u, u + k);
        cp_async<sizeof(TC)>(F.u + T, u + K + k);
        cp_async<sizeof(TC)>(F.u + 2 * T, u + 2 * K + k);
    }
    // biomass where it can act (bit 31 of the returned mask tells ade_finish)
    const bool hb = M.hb != 0;
    if (hb) actm |= 1u << 31;
    if (hb && P.law == CLB_LAW_DUAL_MONOD && !west && !east && P.react[M.code]) {
        const int bn = P.M < ade_bio_cache<TC>() ? P.M : ade_bio_cache<TC>();
        for (int mb = 0; mb < bn; ++mb) cp_async<8>(F.bio + mb * T, bio + (int64_t)mb * P.g.N + M.nd);
    }
    return actm;
}

// The second half, once the staged values are in the frame: boundary completion, sums, kinetics,
// collision with the deposit, scatter back to the node's slots.
template <typename TS, typename TC, bool ODD, int NM, int EXT, typename AP>
__device__ __forceinline__ void ade_finish(TS* __restrict__ g, double* __restrict__ imm, double* __restrict__ bio,
                                           const TC* __restrict__ u, const SparseView& S, const double* __restrict__ neu, const AP& P,
                                           int n_mobile, const int* __restrict__ mob_species, int64_t k_west_end,
                                           int64_t k_east_begin, const AdeExtra& X, const AdeFrame<TC>& F,
                                           int64_t k, const AdeMeta& M, uint32_t actm) {
    constexpr int T = ADE_THREADS;
    const int code = M.code;
    const int dyn = P.dyn[code];
    if (dyn == ADE_BB) return;
    const Geom G = P.g;
    const bool west = k < k_west_end, east = k >= k_east_begin;
    int p = 0;
    if (west || east) p = (int)(M.nd % G.plane);
    TC rb[NM];
#pragma unroll
    for (int m = 0; m < NM; ++m) {
        rb[m] = 0;
        if (!((actm >> m) & 1u)) continue;
        TC* slot = F.pop + (m * 7) * T;
        if ((west || east) && dyn != ADE_NONE) {
            // AdvectionDiffusionBoundaryDynamics: the one inward population makes the
            // node's density equal to the stored value
            const int s = m;  // internal order puts the mobile species first: mobile slot m is species m
            const int type = west ? P.ltype[s] : P.rtype[s];
            double rs;
            if (type == CLB_DIRICHLET) rs = west ? P.lbc[s] : P.rbc[s];
            else rs = neu[((int64_t)s * 2 + (west ? 0 : 1)) * G.plane + p];
            const int miss = west ? 4 : 1;
            TC sum = 0;
#pragma unroll
            for (int i = 0; i < 7; ++i)
                if (i != miss) sum += slot[i * T];
            slot[miss * T] = (TC)(rs - ade_sigma<TC>()) - sum;
        }
        TC r = 0;
#pragma unroll
        for (int i = 0; i < 7; ++i) r += slot[i * T];
        rb[m] = r;
    }
    {
        // a NaN or infinite density in any species makes the sum non-finite: flag it for the host
        TC chk = 0;
#pragma unroll
        for (int m = 0; m < NM; ++m) chk += rb[m];
        if (!isfinite(chk) && P.nonfinite) *(volatile int*)P.nonfinite = 1;
    }
    TC dC[NM];  // increments of the mobile species, in the arithmetic type of the deposit
    node_kinetics<TC, NM, EXT>(P, X, k, M.nd, code, west, east, n_mobile, rb, imm, bio, F.bio,
                               P.M < ade_bio_cache<TC>() ? P.M : ade_bio_cache<TC>(), (actm >> 31) & 1u, dC);
    // ---- phase 2: collide, deposit, stream, species by species from the shared slots
    uint32_t off2[7];  // read back rather than kept live through the kinetics
#pragma unroll
    for (int i = 0; i < 7; ++i) off2[i] = F.off[i * T];
    TC ux, uy, uz;
    if constexpr (ade_u_staged<TC>() == 3) {
        ux = F.u[0];
        uy = F.u[T];
        uz = F.u[2 * T];
    } else {
        ux = u[k];
        uy = u[S.K + k];
        uz = u[2 * S.K + k];
    }
#pragma unroll
    for (int m = 0; m < NM; ++m) {
        if (!((actm >> m) & 1u)) continue;
        const int s = m;  // internal order puts the mobile species first: mobile slot m is species m
        TC q[7], o[7];
#pragma unroll
        for (int i = 0; i < 7; ++i) q[i] = F.pop[(m * 7 + i) * T];
        if (dyn == ADE_NONE) {
#pragma unroll
            for (int i = 0; i < 7; ++i) o[i] = q[i];
        } else {
            const TC w = (TC)(dyn == ADE_BIO ? P.wbio[s] : P.wpore[s]);
            const TC omw = (TC)1 - w;
            const TC rho = rb[m] + (TC)ade_sigma<TC>();
            const TC jx = rho * ux, jy = rho * uy, jz = rho * uz;
            const TC d = dC[m];
            // feq_i = t_i (rb + 4 c_i . j), in opposite-pair form (no zero products)
            const TC r8 = (TC)0.125 * rb[m], d8 = (TC)0.125 * d;
            o[0] = q[0] * omw + w * ((TC)0.25 * rb[m]) + (TC)0.25 * d;
            o[1] = q[1] * omw + w * (r8 - (TC)0.5 * jx) + d8;
            o[4] = q[4] * omw + w * (r8 + (TC)0.5 * jx) + d8;
            o[2] = q[2] * omw + w * (r8 - (TC)0.5 * jy) + d8;
            o[5] = q[5] * omw + w * (r8 + (TC)0.5 * jy) + d8;
            o[3] = q[3] * omw + w * (r8 - (TC)0.5 * jz) + d8;
            o[6] = q[6] * omw + w * (r8 + (TC)0.5 * jz) + d8;
        }
        TS* f = g + (int64_t)m * S.SS;
#pragma unroll
        for (int j = 0; j < 7; ++j) st<TS, TC>(f + off2[j], o[q7opp(j)]);  // outgoing opp(j) back to slot j
    }
}

template <typename TS, typename TC, bool ODD, int NM, int EXT, typename AP>
__device__ __forceinline__ void ade_node(TS* __restrict__ g, double* __restrict__ imm, double* __restrict__ bio,
                                         const TC* __restrict__ u, const SparseView& S,
                                         const double* __restrict__ neu, const AP& P, int n_mobile,
                                         const int* __restrict__ mob_species, int64_t k_west_end,
                                         int64_t k_east_begin, const AdeExtra& X, const AdeFrame<TC>& F, int64_t k) {
    const AdeMeta M = ade_meta<ODD>(S, k, P.bflag);
    const uint32_t actm = ade_gather<TS, TC, ODD, NM>(g, u, bio, S, P, n_mobile, mob_species, k_west_end,
                                                      k_east_begin, F, k, M);
    cp_async_wait_all();  // each thread reads only its own slots
    ade_finish<TS, TC, ODD, NM, EXT>(g, imm, bio, u, S, neu, P, n_mobile, mob_species, k_west_end, k_east_begin, X,
                                     F, k, M, actm);
}

template <typename TS, typename TC, bool ODD, int NM, int EXT>
__global__ void __launch_bounds__(ADE_THREADS, (ade_minb<TC, NM>()))
    k_ade_aa(TS* __restrict__ g, double* __restrict__ imm, double* __restrict__ bio, const TC* __restrict__ u,
             const SparseView S, const double* __restrict__ neu, const AdeParams P, int n_mobile,
             const int* __restrict__ mob_species, int64_t k_west_end, int64_t k_east_begin, const AdeExtra X) {
    const int64_t K = S.K;
    extern __shared__ __align__(16) unsigned char ade_smem[];
    const AdeFrame<TC> F = ade_frame<TC, NM>(ade_smem, 0);
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x)
        ade_node<TS, TC, ODD, NM, EXT>(g, imm, bio, u, S, neu, P, n_mobile, mob_species, k_west_end, k_east_begin,
                                       X, F, k);
}

// resident blocks per SM of the pipelined step (two slot sets per thread); 0: does not fit twice
template <typename TC, int NM>
constexpr int ade_pipe_minb() {
    constexpr int b = (200 * 1024) / (2 * ade_slot_bytes<TC, NM>());
    return b > 4 ? 4 : b;
}

// The transport step with the gathers of the next node in flight while a node is finished: two
// slot sets per thread; node k + stride's values go to one by asynchronous copies while node k is
// finished from the other, and the metadata of the node after that is loading. Same arithmetic
// and memory traffic as k_ade_aa. For 4- and 8-byte storage where two slot sets leave at least
// two resident blocks per SM.
template <typename TS, typename TC, bool ODD, int NM, int EXT>
__global__ void __launch_bounds__(ADE_THREADS, (ade_pipe_minb<TC, NM>() < 1 ? 1 : ade_pipe_minb<TC, NM>()))
    k_ade_pipe(TS* __restrict__ g, double* __restrict__ imm, double* __restrict__ bio, const TC* __restrict__ u,
               const SparseView S, const double* __restrict__ neu, const AdeParams P, int n_mobile,
               const int* __restrict__ mob_species, int64_t k_west_end, int64_t k_east_begin, const AdeExtra X) {
    const int64_t K = S.K;
    extern __shared__ __align__(16) unsigned char ade_smem[];
    const AdeFrame<TC> F0 = ade_frame<TC, NM>(ade_smem, 0), F1 = ade_frame<TC, NM>(ade_smem, 1);
    const int64_t sk = (int64_t)gridDim.x * blockDim.x;
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    AdeMeta cur, nxt;
    uint32_t acur = 0, anxt = 0;
    if (k < K) {
        cur = ade_meta<ODD>(S, k, P.bflag);
        acur = ade_gather<TS, TC, ODD, NM>(g, u, bio, S, P, n_mobile, mob_species, k_west_end, k_east_begin, F0, k,
                                           cur);
    }
    cp_async_commit();
    int64_t kn = k + sk;
    if (kn < K) nxt = ade_meta<ODD>(S, kn, P.bflag);
    int q = 0;
    while (k < K) {
        if (kn < K)
            anxt = ade_gather<TS, TC, ODD, NM>(g, u, bio, S, P, n_mobile, mob_species, k_west_end, k_east_begin,
                                               q ? F0 : F1, kn, nxt);
        cp_async_commit();
        const int64_t knn = kn + sk;
        AdeMeta nn;
        if (knn < K) nn = ade_meta<ODD>(S, knn, P.bflag);
        cp_async_wait_group<1>();  // node k's values have landed
        ade_finish<TS, TC, ODD, NM, EXT>(g, imm, bio, u, S, neu, P, n_mobile, mob_species, k_west_end, k_east_begin, X,
                                         q ? F1 : F0, k, cur, acur);
        k = kn;
        kn = knn;
        cur = nxt;
        nxt = nn;
        acur = anxt;
        q ^= 1;
    }
    cp_async_wait_group<0>();
}

// The stored density of every Neumann plane node: the density of its inner neighbour as it
// stands before the step (FlatAdiabaticBoundaryFunctional3D after the previous stream). A node
// whose inner neighbour is not a fluid node keeps its previous value.
// The Neumann planes of one step, by side (0: x = 0, 1: x = nx - 1): species and mobile slot.
struct NeumannPlanes {
    int n[2];
    int s[2][CLB_MAX_SPECIES], m[2][CLB_MAX_SPECIES];
};

// One thread per plane pixel and side: the inner neighbour's 7 storage locations are found once
// (they are the same in every species' buffer, a species stride apart) and serve every species
// with a Neumann face on that side, whose loads are then all independent.
template <typename TS, typename TC>
__global__ void k_ade_neumann(const TS* __restrict__ g, const TS* __restrict__ glink, const SparseView S,
                              const int8_t* __restrict__ mat, double* __restrict__ neu, const AdeParams P,
                              const NeumannPlanes J, int odd) {
    const Geom G = P.g;
    const int side = blockIdx.y;
    const int ns = J.n[side];
    if (ns == 0) return;
    const int xb = side == 0 ? 0 : G.nx - 1, xi = side == 0 ? 1 : G.nx - 2;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < G.plane; p += gridDim.x * blockDim.x) {
        const int64_t nb = (int64_t)xb * G.plane + p, ni = (int64_t)xi * G.plane + p;
        const int db = P.dyn[mat[nb]], di = P.dyn[mat[ni]];
        if (!(db == ADE_PORE || db == ADE_BIO) || !(di == ADE_PORE || di == ADE_BIO)) continue;
        int x, y, z;
        decode(G, ni, x, y, z);
        const TS* loc[7];  // in species 0's buffer; nullptr: never written, the initial value
#pragma unroll
        for (int i = 0; i < 7; ++i) loc[i] = natural_slot<const TS, 7>(S, G, g, glink, ni, x, y, z, i, odd);
#pragma unroll 2
        for (int j = 0; j < ns; ++j) {
            const int s = J.s[side][j];
            const int64_t sh = (int64_t)J.m[side][j] * S.SS;
            const double c0 = P.c0[s];
            TC pop[7];
#pragma unroll
            for (int i = 0; i < 7; ++i)
                pop[i] = loc[i] ? ld<TS, TC>(loc[i] + sh) : (TC)(q7w(i) * (c0 - ade_sigma<TC>()));
            double r = ade_sigma<TC>();
#pragma unroll
            for (int i = 0; i < 7; ++i) r += (double)pop[i];
            neu[((int64_t)s * 2 + side) * G.plane + p] = r;
        }
    }
}

template <typename TS>
__global__ void k_ade_init(TS* __restrict__ g, TS* __restrict__ glink, int64_t K, int64_t L, int64_t SS,
                           int n_mobile, const double* __restrict__ c0m) {
    // K here is the padded row stride: the padding slots are initialised too
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K || k < L;
         k += (int64_t)gridDim.x * blockDim.x) {
        for (int m = 0; m < n_mobile; ++m) {
            double c = c0m[m];
            if (c < THRD && c > -THRD) c = 0.0;
            if (k < K)
                for (int i = 0; i < 7; ++i) {
                    double v = q7w(i) * (c - ade_sigma<TS>());
                    if constexpr (std::is_same<TS, __half>::value) g[(int64_t)m * SS + (int64_t)i * K + k] = to_half(v);
                    else g[(int64_t)m * SS + (int64_t)i * K + k] = (TS)v;
                }
            if (k < L) {
                // a wall slot holds population j of the wall node; every j != 0 has weight 1/8
                double v = 0.125 * (c - ade_sigma<TS>());
                if constexpr (std::is_same<TS, __half>::value) glink[(int64_t)m * SS + k] = to_half(v);
                else glink[(int64_t)m * SS + k] = (TS)v;
            }
        }
    }
}

// shifted != 0: the populations g_i - t_i go out; 0: the stored values g_i - sigma t_i as they are
template <typename TS>
__global__ void k_ade_get_pops(const TS* __restrict__ g, const TS* __restrict__ glink, const SparseView S,
                               const Geom G, int odd, double c0, int shifted, double* __restrict__ out) {
    constexpr double sig = ade_sigma<TS>();
    double init[7];
    for (int i = 0; i < 7; ++i) init[i] = q7w(i) * (c0 - sig);
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < G.N; n += (int64_t)gridDim.x * blockDim.x) {
        double v[7];
        natural<TS, double, 7>(S, G, g, glink, n, odd, init, v);
        for (int i = 0; i < 7; ++i) out[(int64_t)i * G.N + n] = (sig == 1.0 || !shifted) ? v[i] : v[i] - q7w(i) * (1.0 - sig);
    }
}

// computeDensity of species s (internal index) at every voxel: BGK nodes of a Dirichlet / Neumann
// plane report the stored value; every other voxel 1 + the sum of its incoming populations (a voxel
// that is not a node holds the initial equilibrium at c0).
template <typename TS>
__global__ void k_ade_density(const TS* __restrict__ g, const TS* __restrict__ glink, const SparseView S,
                              const int8_t* __restrict__ mat, const AdeParams P, int s, int odd,
                              const double* __restrict__ neu, double* __restrict__ out) {
    const Geom G = P.g;
    double init[7];
    for (int i = 0; i < 7; ++i) init[i] = q7w(i) * (P.c0[s] - ade_sigma<TS>());
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < G.N; n += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(n / G.plane);
        const int p = (int)(n - (int64_t)x * G.plane);
        const int dyn = P.dyn[(uint8_t)mat[n]];
        const bool bgk = dyn == ADE_PORE || dyn == ADE_BIO;
        if (bgk && x == 0 && P.ltype[s] != CLB_CLOSED) {
            out[n] = P.ltype[s] == CLB_DIRICHLET ? P.lbc[s] : neu[p];
            continue;
        }
        if (bgk && x == G.nx - 1 && P.rtype[s] != CLB_CLOSED) {
            out[n] = P.rtype[s] == CLB_DIRICHLET ? P.rbc[s] : neu[G.plane + p];
            continue;
        }
        double v[7];
        natural<TS, double, 7>(S, G, g, glink, n, odd, init, v);
        double r = ade_sigma<TS>();
        for (int i = 0; i < 7; ++i) r += v[i];
        out[n] = r;
    }
}

// shifted != 0: `in` holds g_i - t_i; 0: the stored values g_i - sigma t_i
template <typename TS>
__global__ void k_ade_set_pops(TS* __restrict__ g, TS* __restrict__ glink, const SparseView S, const Geom G, int odd,
                               int shifted, const double* __restrict__ in) {
    const double add = shifted ? 1.0 - ade_sigma<TS>() : 0.0;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < G.N; n += (int64_t)gridDim.x * blockDim.x) {
        double v[7];
        for (int i = 0; i < 7; ++i) v[i] = in[(int64_t)i * G.N + n] + q7w(i) * add;
        put_natural<TS, 7>(S, G, g, glink, n, odd, v);
    }
}

// Deterministic FP64 reductions of the live fields. Block (b, r) of a grid of RED_BLOCKS x (S + 1)
// covers the nodes k = b*256 + t + j*RED_BLOCKS*256 (thread t, j = 0, 1, ...) in that order; row
// r < S reduces species r, row S the biomass fields and the open-voxel count. Each thread
// accumulates in registers, a warp combines its lanes with a fixed shuffle tree, and warp 0 adds
// the warps' partials in warp order, so every partial -- and k_reduce_combine's sum of them in
// block order -- is the same number on every call: no atomics anywhere.
// Partial rows (each RED_BLOCKS wide): [S total][S content][S min][S max][S non-finite][M bio][open].
// total/min/max/non-finite over open voxels of x=1..nx-2 (stored nodes that react); content = sum
// over stored nodes of (sum of populations + 1) plus the wall link slots (the content held in walls
// that can move).
constexpr int RED_THREADS = 256;

__device__ __forceinline__ double warp_sum_fixed(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// fixed-order block combination; op 0 sum, 1 min, 2 max; result valid in thread 0
__device__ __forceinline__ double block_fixed(double v, int op, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_down_sync(0xffffffffu, v, o);
        v = op == 0 ? v + w : (op == 1 ? fmin(v, w) : fmax(v, w));
    }
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = sh[0];
    if (threadIdx.x == 0)
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k)
            r = op == 0 ? r + sh[k] : (op == 1 ? fmin(r, sh[k]) : fmax(r, sh[k]));
    return r;
}

template <typename TS>
__global__ void __launch_bounds__(RED_THREADS)
    k_ade_reduce(const TS* __restrict__ g, const TS* __restrict__ glink, const double* __restrict__ imm,
                 const double* __restrict__ bio, const SparseView S, const AdeParams P, double* __restrict__ part,
                 int64_t k_west_end, int64_t k_east_begin, int odd) {
    __shared__ double sh[RED_THREADS / 32];
    const int S_ = P.S, M = P.M, B = gridDim.x, row = blockIdx.y;
    const int64_t K = S.K;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t k0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row < S_) {
        const int s = row, m = P.slot[s];
        double tot = 0.0, cont = 0.0, mn = 1e300, mx = -1e300, nonf = 0.0;
        // content in the shifted convention whatever the storage: a link slot holds a population of
        // weight 1/8
        constexpr double sig = ade_sigma<TS>();
        if (m >= 0)
            for (int64_t k = k0; k < S.L; k += stride) cont += ldd(glink + (int64_t)m * S.SS + k) - 0.125 * (1.0 - sig);
        for (int64_t k = k0; k < K; k += stride) {
            const int code = S.code[k];
            const bool open = k >= k_west_end && k < k_east_begin && P.react[code];
            double c = 0.0;
            if (m >= 0) {
                // content: the node's own slots (every slot of the lattice counted once)
                double sum = sig;
#pragma unroll
                for (int i = 0; i < 7; ++i) sum += ldd(g + (int64_t)m * S.SS + (int64_t)i * S.KS + k);
                cont += sum;
                if (open) {
                    // concentration: the node's incoming populations wherever the step parity keeps
                    // them (computeDensity after the stream)
                    double zero[7];  // an untouched slot: the equilibrium at 1
                    for (int i = 0; i < 7; ++i) zero[i] = q7w(i) * (1.0 - sig);
                    double pop[7];
                    natural<TS, double, 7>(S, P.g, g + (int64_t)m * S.SS, glink + (int64_t)m * S.SS, S.node[k], odd,
                                           zero, pop);
                    c = sig;
#pragma unroll
                    for (int i = 0; i < 7; ++i) c += pop[i];
                }
            } else {
                c = imm[(int64_t)s * P.g.N + S.node[k]];
                cont += c;
            }
            if (open) {
                tot += c;
                if (!isfinite(c)) nonf += 1.0;
                mn = fmin(mn, c);
                mx = fmax(mx, c);
            }
        }
        const double v[5] = {tot, cont, mn, mx, nonf};
        const int op[5] = {0, 0, 1, 2, 0};
#pragma unroll
        for (int j = 0; j < 5; ++j) {
            const double r = block_fixed(v[j], op[j], sh);
            if (threadIdx.x == 0) part[(int64_t)(j * S_ + s) * B + blockIdx.x] = r;
        }
    } else {
        double open_n = 0.0;
        for (int64_t k = k0; k < K; k += stride) {
            const bool inner = k >= k_west_end && k < k_east_begin;
            if (inner && P.react[S.code[k]]) open_n += 1.0;
        }
        double r = block_fixed(open_n, 0, sh);
        if (threadIdx.x == 0) part[(int64_t)(5 * S_ + M) * B + blockIdx.x] = r;
        for (int mb = 0; mb < M; ++mb) {
            double b = 0.0;
            for (int64_t k = k0; k < K; k += stride)
                if (k >= k_west_end && k < k_east_begin) b += bio[(int64_t)mb * P.g.N + S.node[k]];
            r = block_fixed(b, 0, sh);
            if (threadIdx.x == 0) part[(int64_t)(5 * S_ + mb) * B + blockIdx.x] = r;
        }
    }
}

// Combines the partial rows in block order into the result layout
// [S total][S content][S min][S max][M bio][non-finite][open]: one thread per result, a fixed
// sequential order, so the result is bit-identical from call to call.
__global__ void k_reduce_combine(const double* __restrict__ part, int blocks, int S, int M, double* __restrict__ out) {
    const int nq = 4 * S + M + 2;
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        int row, op = 0, rows = 1;
        if (q < 4 * S) { row = q; op = (q >= 2 * S && q < 3 * S) ? 1 : (q >= 3 * S ? 2 : 0); }
        else if (q < 4 * S + M) row = 5 * S + (q - 4 * S);
        else if (q == 4 * S + M) { row = 4 * S; rows = S; }  // non-finite of every species
        else row = 5 * S + M;
        double acc = op == 1 ? 1e300 : (op == 2 ? -1e300 : 0.0);
        for (int r = 0; r < rows; ++r)
            for (int b = 0; b < blocks; ++b) {
                const double v = part[(int64_t)(row + r) * blocks + b];
                acc = op == 0 ? acc + v : (op == 1 ? fmin(acc, v) : fmax(acc, v));
            }
        out[q] = acc;
    }
}

// ------------------------------------------------------------------ host side

// Doubles of scratch a reduction needs (S species, M microbes): the partial rows, then the result.
static int64_t reduce_scratch_doubles(int S, int M, int blocks) {
    return (int64_t)(5 * S + M + 1) * blocks + (4 * S + M + 2);
}

static int reduce_blocks(const clb_handle* h) { return h->num_sms * 2; }

static size_t esize(int prec) { return prec == CLB_F64 ? 8 : (prec == CLB_F32 ? 4 : 2); }
static size_t usize(int prec) { return prec == CLB_F64 ? 8 : 4; }

void ade_free(clb_handle* h) {
    cudaFree(h->d_g); h->d_g = nullptr;
    h->d_glink = nullptr;  // inside d_g
    cudaFree(h->d_imm); h->d_imm = nullptr;
    cudaFree(h->d_bio); h->d_bio = nullptr;
    cudaFree(h->d_bflag); h->d_bflag = nullptr;
    cudaFree(h->d_u); h->d_u = nullptr;
    cudaFree(h->d_neu); h->d_neu = nullptr;
    cudaFree(h->d_red); h->d_red = nullptr;
    cudaFree(h->d_stage); h->d_stage = nullptr;
    precip_free(h);
    ca_free(h);
    sparse_free(h->ade_sp);
    h->ade_ready = false;
}

static int* mob_table(clb_handle* h) {
    // device copy of the mobile-species table lives after the boundary store
    return (int*)(h->d_neu + (size_t)h->S * 2 * h->g.plane);
}

clb_status ade_init(clb_handle* h, const clb_species_desc* sp, int S) {
    const clb_domain_desc& d = h->d;
    if (S < 1 || S > CLB_MAX_SPECIES) return fail(h, CLB_INVALID_ARG, "species count out of range");
    ade_free(h);
    AdeParams& P = h->ap;
    std::memset(&P, 0, sizeof(P));
    P.g = h->g;
    P.S = S;
    P.M = 0;
    P.law = CLB_LAW_NONE;
    P.dt = 1.0;
    // soluteDomainSetup + complab.cpp:1630: pore BGK(pore omega), biofilm BGK(biofilm omega),
    // wall bounce-back, solid bounce-back for mobile species; unknown codes default to pore.
    for (int c = 0; c < MAX_CODES; ++c) { P.dyn[c] = ADE_PORE; P.react[c] = 1; }
    for (int m = 0; m < d.n_microbes; ++m)
        if (d.bio_codes[m] >= 0 && d.bio_codes[m] < MAX_CODES) P.dyn[d.bio_codes[m]] = ADE_BIO;
    if (d.bounce_back_code >= 0 && d.bounce_back_code < MAX_CODES) {
        P.dyn[d.bounce_back_code] = ADE_BB;
        P.react[d.bounce_back_code] = 0;
    }
    if (d.solid_code >= 0 && d.solid_code < MAX_CODES) {
        P.dyn[d.solid_code] = ADE_BB;
        P.react[d.solid_code] = 0;
    }
    h->species.assign(sp, sp + S);
    // internal order: mobile species first (user order), then immobile ones
    std::vector<int> order;
    for (int s = 0; s < S; ++s) if (sp[s].mobile) order.push_back(s);
    for (int s = 0; s < S; ++s) if (!sp[s].mobile) order.push_back(s);
    std::vector<int> mob;
    std::vector<double> c0m;
    for (int i = 0; i < S; ++i) {
        const clb_species_desc& d_ = sp[order[i]];
        h->i2u[i] = order[i];
        h->u2i[order[i]] = i;
        P.mobile[i] = d_.mobile ? 1 : 0;
        P.slot[i] = -1;
        if (d_.mobile) { P.slot[i] = (int)mob.size(); mob.push_back(i); c0m.push_back(d_.c0); }
        P.ltype[i] = d_.left_type;
        P.rtype[i] = d_.right_type;
        P.lbc[i] = d_.left_bc;
        P.rbc[i] = d_.right_bc;
        P.wpore[i] = d_.omega_pore;
        P.wbio[i] = d_.omega_biofilm;
        P.c0[i] = d_.c0;
    }
    P.donor = 0;
    for (int m = 0; m < CLB_MAX_MICROBES; ++m) P.acceptor[m] = -1;
    h->S = S;
    h->n_mobile = (int)mob.size();
    if (h->n_mobile > 16) return fail(h, CLB_INVALID_ARG, "at most 16 mobile species");
    h->M = 0;
    h->ade_prec = d.ade_precision;

    int8_t cls[MAX_CODES];
    for (int c = 0; c < MAX_CODES; ++c) cls[c] = (P.dyn[c] != ADE_BB);
    clb_status st = sparse_build(h, cls, 7, h->ade_sp);
    if (st != CLB_OK) return st;
    const int64_t K = h->ade_sp.K, L = h->ade_sp.L;
    int64_t kw = 0, ke = 0;
    for (int64_t n = 0; n < h->g.plane; ++n) kw += cls[(uint8_t)h->h_mat[n] & 127] != 0;
    for (int64_t n = h->g.N - h->g.plane; n < h->g.N; ++n) ke += cls[(uint8_t)h->h_mat[n] & 127] != 0;
    h->ade_west_end = kw;
    h->ade_east_begin = K - ke;
    const size_t K1 = (size_t)std::max<int64_t>(1, K);
    const int nm1 = std::max(1, h->n_mobile);
    cudaError_t e;
    const size_t KS = (size_t)h->ade_sp.KS;
    // one buffer: species m's 7 population rows, then its link slots, at [m SS, (m + 1) SS)
    const size_t SSz = (size_t)h->ade_sp.SS;
    if ((e = cudaMalloc(&h->d_g, esize(h->ade_prec) * SSz * nm1)) != cudaSuccess)
        return cuda_check(h, e, "species populations");
    h->d_glink = (char*)h->d_g + esize(h->ade_prec) * 7 * KS;
    const size_t N1 = (size_t)h->g.N;
    if ((e = cudaMalloc(&h->d_imm, sizeof(double) * N1 * S)) != cudaSuccess) return cuda_check(h, e, "immobile fields");
    if ((e = cudaMalloc(&h->d_u, usize(h->ade_prec) * 3 * K1)) != cudaSuccess) return cuda_check(h, e, "velocity");
    if ((e = cudaMalloc(&h->d_neu, sizeof(double) * S * 2 * h->g.plane + sizeof(int) * 16)) != cudaSuccess)
        return cuda_check(h, e, "boundary store");
    if (!h->h_flags) {
        // host-mapped flags the transport step sets (read by the host without a copy)
        if ((e = cudaHostAlloc((void**)&h->h_flags, 16, cudaHostAllocMapped)) != cudaSuccess)
            return cuda_check(h, e, "status flags");
        std::memset(h->h_flags, 0, 16);
        if ((e = cudaHostGetDevicePointer((void**)&h->d_flags, h->h_flags, 0)) != cudaSuccess)
            return cuda_check(h, e, "status flags");
    }
    if ((e = cudaMalloc(&h->d_red, sizeof(double) * reduce_scratch_doubles(S, CLB_MAX_MICROBES, reduce_blocks(h)))) != cudaSuccess)
        return cuda_check(h, e, "reduction scratch");
    if ((e = cudaMalloc(&h->d_bflag, K1)) != cudaSuccess) return cuda_check(h, e, "biomass flags");
    cudaMemsetAsync(h->d_bflag, 1, K1, h->stream);  // until biomass is set, every node may hold some
    h->ap.bflag = h->d_bflag;
    cudaMemsetAsync(h->d_u, 0, usize(h->ade_prec) * 3 * K1, h->stream);
    // immobile species: uniform c0 (initial_concentration applies to the whole domain)
    std::vector<double> immh(N1);
    for (int i = 0; i < S; ++i) {
        if (P.mobile[i]) continue;
        std::fill(immh.begin(), immh.end(), P.c0[i]);
        cudaMemcpy(h->d_imm + (size_t)i * N1, immh.data(), sizeof(double) * N1, cudaMemcpyHostToDevice);
    }
    // stored boundary densities: Dirichlet value, else c0 (lattice.initialize() runs the
    // Neumann processor once on the equilibrium field)
    std::vector<double> neu((size_t)S * 2 * h->g.plane);
    for (int i = 0; i < S; ++i)
        for (int side = 0; side < 2; ++side) {
            int t = side == 0 ? P.ltype[i] : P.rtype[i];
            double v = t == CLB_DIRICHLET ? (side == 0 ? P.lbc[i] : P.rbc[i]) : P.c0[i];
            std::fill(neu.begin() + ((size_t)i * 2 + side) * h->g.plane,
                      neu.begin() + ((size_t)i * 2 + side + 1) * h->g.plane, v);
        }
    cudaMemcpy(h->d_neu, neu.data(), sizeof(double) * neu.size(), cudaMemcpyHostToDevice);
    int mt[16] = {0};
    for (size_t k = 0; k < mob.size(); ++k) mt[k] = mob[k];
    cudaMemcpy(mob_table(h), mt, sizeof(mt), cudaMemcpyHostToDevice);
    if (!c0m.empty()) {
        double* dc0 = nullptr;
        cudaMalloc(&dc0, sizeof(double) * c0m.size());
        cudaMemcpy(dc0, c0m.data(), sizeof(double) * c0m.size(), cudaMemcpyHostToDevice);
        const int grid = h->num_sms * 8;
        switch (h->ade_prec) {
            case CLB_F64: k_ade_init<double><<<grid, 256, 0, h->stream>>>((double*)h->d_g, (double*)h->d_glink, (int64_t)KS, L, (int64_t)SSz, h->n_mobile, dc0); break;
            case CLB_F32: k_ade_init<float><<<grid, 256, 0, h->stream>>>((float*)h->d_g, (float*)h->d_glink, (int64_t)KS, L, (int64_t)SSz, h->n_mobile, dc0); break;
            default: k_ade_init<__half><<<grid, 256, 0, h->stream>>>((__half*)h->d_g, (__half*)h->d_glink, (int64_t)KS, L, (int64_t)SSz, h->n_mobile, dc0); break;
        }
        cudaStreamSynchronize(h->stream);
        cudaFree(dc0);
    }
    h->ade_iters = 0;
    h->neu_iter = -1;
    h->ade_grid = h->num_sms * 4;
    P.nonfinite = h->d_flags;
    if (h->h_flags) h->h_flags[0] = 0;
    h->ade_ready = true;
    return cuda_check(h, cudaGetLastError(), "ade init");
}

clb_status ade_set_kinetics(clb_handle* h, int law, const double* prm, int nprm, double dt) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (nprm < 0 || nprm > 4 * CLB_MAX_SPECIES) return fail(h, CLB_INVALID_ARG, "too many kinetics parameters");
    if (law < 0 || law > CLB_LAW_DUAL_MONOD) return fail(h, CLB_INVALID_ARG, "unknown rate law");
    AdeParams& P = h->ap;
    const int S = h->S;
    P.law = law;
    P.sym_mask = 0;  // a compiled law replaces the organisms' rate-law files and networks
    P.gnn_mask = 0;
    P.srg_mask = 0;
    std::memset(P.prm, 0, sizeof(P.prm));
    switch (law) {
        case CLB_LAW_DECAY:
            if (nprm < S) return fail(h, CLB_INVALID_ARG, "decay needs one rate per species");
            for (int i = 0; i < S; ++i) P.prm[i] = prm[h->i2u[i]];
            break;
        case CLB_LAW_MONOD:
            if (nprm < 2 * S) return fail(h, CLB_INVALID_ARG, "Monod needs k[S] then Ks[S]");
            for (int i = 0; i < S; ++i) {
                P.prm[i] = prm[h->i2u[i]];
                P.prm[CLB_MAX_SPECIES + i] = prm[S + h->i2u[i]];
            }
            break;
        case CLB_LAW_DUAL_MONOD:
            if (nprm < 4) return fail(h, CLB_INVALID_ARG, "dual Monod needs mu_max, Ks, Y, kd");
            for (int k = 0; k < 4; ++k) P.prm[k] = prm[k];
            P.donor = h->u2i[0];
            for (int m = 0; m < CLB_MAX_MICROBES; ++m) P.acceptor[m] = (1 + m < S) ? h->u2i[1 + m] : -1;
            break;
        default:
            break;
    }
    P.dt = dt;
    return CLB_OK;
}

clb_status ade_set_abiotic(clb_handle* h, int law, const double* prm, int nprm, int surface_only) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    AdeParams& P = h->ap;
    const int S = h->S;
    auto species = [&](double v, int& out) {
        const int s = (int)v;
        if ((double)s != v || s < 0 || s >= S) return false;
        out = h->u2i[s];
        return true;
    };
    std::memset(P.prm2, 0, sizeof(P.prm2));
    switch (law) {
        case CLB_LAW_NONE:
            break;
        case CLB_LAW_PRECIP: {
            if (nprm < 4) return fail(h, CLB_INVALID_ARG, "precipitation law needs kp, a, b, p");
            int a, b, q;
            if (!species(prm[1], a) || !species(prm[2], b) || !species(prm[3], q))
                return fail(h, CLB_INVALID_ARG, "precipitation law: species index out of range");
            P.prm2[0] = prm[0];
            P.prm2[1] = a;
            P.prm2[2] = b;
            P.prm2[3] = q;
            break;
        }
        case CLB_LAW_MINERAL: {
            if (nprm < 3 + S) return fail(h, CLB_INVALID_ARG, "mineral law needs k, log10 Ksp, p, nu[S]");
            int q;
            if (!species(prm[2], q)) return fail(h, CLB_INVALID_ARG, "mineral law: species index out of range");
            P.prm2[0] = prm[0];
            P.prm2[1] = prm[1];
            P.prm2[2] = q;
            for (int i = 0; i < S; ++i) P.prm2[3 + i] = prm[3 + h->i2u[i]];
            break;
        }
        default:
            return fail(h, CLB_INVALID_ARG, "not an abiotic rate law");
    }
    P.law2 = law;
    P.gnn_abiotic = 0;
    P.surf = surface_only ? 1 : 0;
    return geometry_refresh(h);
}

// the concentration field of an immobile species (user index), FP64 [N]
clb_status ade_set_immobile(clb_handle* h, int s, const double* host) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (s < 0 || s >= h->S) return fail(h, CLB_INVALID_ARG, "species index out of range");
    const int si = h->u2i[s];
    if (h->ap.slot[si] >= 0) return fail(h, CLB_INVALID_ARG, "not an immobile species");
    return cuda_check(h, cudaMemcpy(h->d_imm + (size_t)si * h->g.N, host, sizeof(double) * (size_t)h->g.N,
                                    cudaMemcpyHostToDevice), "immobile concentration");
}

// A species' concentration field (user index s, FP64 [N]): an immobile species takes it as it is; a
// mobile species gets the populations of the equilibrium at rest with that density,
// f_i - t_i = t_i (C - 1) (initializeScalarLattice3D / the reference's initial concentration,
// complab3d_processors_part3.hh:215-258), at every node of its lattice.
clb_status ade_set_concentration(clb_handle* h, int s, const double* host) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (s < 0 || s >= h->S) return fail(h, CLB_INVALID_ARG, "species index out of range");
    if (h->ap.slot[h->u2i[s]] < 0) return ade_set_immobile(h, s, host);
    const size_t N = (size_t)h->g.N;
    // in the storage's own convention, so a small concentration is not rounded through C - 1
    const double sig = h->ade_prec == CLB_F64 ? 1.0 : 0.0;
    std::vector<double> pops(7 * N);
    for (int i = 0; i < 7; ++i) {
        const double w = q7w(i);
        for (size_t n = 0; n < N; ++n) pops[(size_t)i * N + n] = w * (host[n] - sig);
    }
    return ade_set_populations(h, s, pops.data(), 0);
}

clb_status ade_set_thermo(clb_handle* h, const clb_thermo_desc* d) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    AdeParams& P = h->ap;
    if (!d || d->n_terms == 0) {
        P.gate_on = 0;
        P.gate_n = 0;
        return CLB_OK;
    }
    if (d->n_terms < 0 || d->n_terms > CLB_MAX_SPECIES) return fail(h, CLB_INVALID_ARG, "thermo gate: term count out of range");
    if (!(d->cmin > 0.0)) return fail(h, CLB_INVALID_ARG, "thermo gate: cmin <= 0, so ln Q can be -inf");
    if (d->dGloss < 0.0) return fail(h, CLB_INVALID_ARG, "thermo gate: negative dGloss");
    if (!(d->temperature > 0.0) || !(d->gas_constant > 0.0) || !(d->conc_scale > 0.0))
        return fail(h, CLB_INVALID_ARG, "thermo gate: temperature, gas constant and concentration scale must be positive");
    for (int i = 0; i < d->n_terms; ++i) {
        if (d->species[i] < 0 || d->species[i] >= h->S) return fail(h, CLB_INVALID_ARG, "thermo gate: species index out of range");
        P.gate_sp[i] = h->u2i[d->species[i]];
        P.gate_nu[i] = d->nu[i];
    }
    P.gate_n = d->n_terms;
    P.gate_dG0 = d->dG0;
    P.gate_dGloss = d->dGloss;
    P.gate_atp = d->atp;
    P.gate_dGatp = d->dGatp;
    P.gate_chi = d->chi > 0.0 ? d->chi : 1.0;
    P.gate_cmin = d->cmin;
    P.gate_RT = d->gas_constant * d->temperature;
    P.gate_cscale = d->conc_scale;
    P.gate_x0 = (P.gate_dG0 + P.gate_dGloss + P.gate_atp * P.gate_dGatp) / (P.gate_chi * P.gate_RT);
    P.gate_inv_chi = 1.0 / P.gate_chi;
    P.gate_on = 1;
    return CLB_OK;
}

// the biomass flag of every species-lattice node: 1 where some microbe's biomass is not below 1e-12
// (NaN included, so a non-finite field still reaches the kinetics and is reported)
__global__ void k_bflag(uint8_t* __restrict__ flag, const int32_t* __restrict__ node, int64_t K,
                        const double* __restrict__ bio, int M, int64_t N) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t nd = node[k];
        uint8_t f = 0;
        for (int m = 0; m < M; ++m) f |= !(bio[(int64_t)m * N + nd] < THRD);
        flag[k] = f;
    }
}

static clb_status refresh_bflag(clb_handle* h) {
    if (!h->d_bflag || h->M < 1 || !h->d_bio) return CLB_OK;
    ++h->launches;
    k_bflag<<<h->num_sms * 4, 256, 0, h->stream>>>(h->d_bflag, h->ade_sp.node, h->ade_sp.K, h->d_bio, h->M, h->g.N);
    return cuda_check(h, cudaGetLastError(), "biomass flags");
}

clb_status ade_set_biomass(clb_handle* h, int M, const double* b) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (M < 0 || M > CLB_MAX_MICROBES) return fail(h, CLB_INVALID_ARG, "microbe count out of range");
    cudaFree(h->d_bio);
    h->d_bio = nullptr;
    h->M = M;
    h->ap.M = M;
    h->ca_full = true;  // the automaton's next mask pass looks at every voxel's new biomass
    if (M == 0) return CLB_OK;
    cudaError_t e = cudaMalloc(&h->d_bio, sizeof(double) * M * (size_t)h->g.N);
    if (e != cudaSuccess) return cuda_check(h, e, "biomass");
    clb_status st = cuda_check(h, cudaMemcpy(h->d_bio, b, sizeof(double) * M * (size_t)h->g.N, cudaMemcpyHostToDevice),
                               "biomass copy");
    return st == CLB_OK ? refresh_bflag(h) : st;
}

// Resident blocks per SM of a transport-step instantiation with `smem` bytes of shared memory
// (set up once per instantiation), times the SM count: the persistent grid.
static int ade_grid_for(const void* kern, int smem, int num_sms, int threads, int resident = ADE_RESIDENT) {
    struct Known { const void* kern; int smem, threads, blocks; };
    static std::mutex mu;
    static std::vector<Known> known;
    std::lock_guard<std::mutex> lock(mu);
    int set_max = 0;  // the kernel's dynamic shared-memory limit so far (one attribute for every caller)
    for (auto& kv : known) {
        if (kv.kern == kern && kv.smem == smem && kv.threads == threads) return kv.blocks * num_sms;
        if (kv.kern == kern) set_max = std::max(set_max, kv.smem);
    }
    if (smem > 48 * 1024 && smem > set_max) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    // Shared memory for at most `resident` blocks per SM; the rest of the SM's 256 KB stays L1
    // cache, which the odd step's neighbour gathers reuse (five resident blocks with less L1 ran
    // the odd step slower on B200; the even step, which reads only its own slots, gained from five).
    {
        const int per_block = smem + 1024;  // the runtime reserves 1 KB per block
        const int fit = std::max(1, (228 * 1024) / per_block);
        const int res = std::min(resident, fit);
        const int pct = (int)((100LL * res * per_block + 228 * 1024 - 1) / (228 * 1024));
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct > 100 ? 100 : pct);
    }
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads, smem) != cudaSuccess || nb < 1) nb = 1;
    known.push_back({kern, smem, threads, nb});
    return nb * num_sms;
}

template <typename TS, typename TC, bool ODD>
static void launch_ade_t(clb_handle* h) {
    ++h->launches;  // one transport launch per call
    const int nm = h->n_mobile;
    const int nb = h->S;  // register bucket covers every species (mobile first, then immobile)
    TS* g = (TS*)h->d_g;
    const TC* u = (const TC*)h->d_u;
    int* mt = mob_table(h);
    const SparseView S = view_of(h->ade_sp);
    const bool ext = h->ap.law2 != CLB_LAW_NONE || h->ap.dis_on || h->ap.gate_on || h->ap.law == CLB_LAW_SYMBOLIC;
    const AdeExtra X = ade_extra(h);
#define CLB_ADE(NM, EXT)                                                                                          \
    do {                                                                                                          \
        if constexpr (sizeof(TS) >= 4 && ade_pipe_minb<TC, NM>() >= 2) {                                           \
            if (h->ade_pipe) {                                                                                    \
            auto kern = k_ade_pipe<TS, TC, ODD, NM, EXT>;                                                          \
            const int sm = 2 * ade_slot_bytes<TC, NM>();                                                           \
            const int gr = ade_grid_for((const void*)kern, sm, h->num_sms, ADE_THREADS);                           \
            kern<<<gr, ADE_THREADS, sm, h->stream>>>(g, h->d_imm, h->d_bio, u, S, h->d_neu, h->ap, nm, mt,        \
                                                     h->ade_west_end, h->ade_east_begin, X);                      \
            break;                                                                                                \
            }                                                                                                     \
        }                                                                                                         \
        auto kern = k_ade_aa<TS, TC, ODD, NM, EXT>;                                                               \
        const int sm = ade_slot_bytes<TC, NM>();                                                                  \
        const int gr = ade_grid_for((const void*)kern, sm, h->num_sms, ADE_THREADS, ODD ? ADE_RESIDENT : ADE_RESIDENT_EVEN); \
        kern<<<gr, ADE_THREADS, sm, h->stream>>>(g, h->d_imm, h->d_bio, u, S, h->d_neu, h->ap, nm, mt,            \
                                                 h->ade_west_end, h->ade_east_begin, X);                          \
    } while (0)
    // EXT: 0 the compiled biotic laws alone; 1 with the abiotic block, dissolution and the
    // thermodynamic gate; 2 also the rate-law files (their interpreter's registers and stack stay
    // out of the other instantiations)
    const bool sym = h->ap.law == CLB_LAW_SYMBOLIC || h->ap.law2 == CLB_LAW_SYMBOLIC;
    if (sym) {
        if (nb <= 4) CLB_ADE(4, 2);
        else if (nb <= 8) CLB_ADE(8, 2);
        else CLB_ADE(16, 2);
    } else if (ext) {
        if (nb <= 4) CLB_ADE(4, 1);
        else if (nb <= 8) CLB_ADE(8, 1);
        else CLB_ADE(16, 1);
    } else if (nb <= 1) CLB_ADE(1, 0);
    else if (nb <= 2) CLB_ADE(2, 0);
    else if (nb <= 4) CLB_ADE(4, 0);
    else if (nb <= 8) CLB_ADE(8, 0);
    else CLB_ADE(16, 0);
#undef CLB_ADE
}

template <typename TS, typename TC>
static void launch_neumann(clb_handle* h, int odd) {
    const SparseView S = view_of(h->ade_sp);
    NeumannPlanes J;
    J.n[0] = J.n[1] = 0;
    for (int s = 0; s < h->S; ++s) {
        const int m = h->ap.slot[s];
        if (m < 0) continue;
        for (int side = 0; side < 2; ++side) {
            const int t = side == 0 ? h->ap.ltype[s] : h->ap.rtype[s];
            if (t != CLB_NEUMANN) continue;
            J.s[side][J.n[side]] = s;
            J.m[side][J.n[side]] = m;
            ++J.n[side];
        }
    }
    if (J.n[0] + J.n[1] == 0) return;
    const dim3 grid(std::max(1, std::min(h->num_sms * 4, (h->g.plane + 127) / 128)), 2);
    ++h->launches;
    k_ade_neumann<TS, TC><<<grid, 128, 0, h->stream>>>((const TS*)h->d_g, (const TS*)h->d_glink, S, h->d_mat,
                                                       h->d_neu, h->ap, J, odd);
}

// The stored densities are those after the latest stream; they are recomputed lazily, once per
// transport iteration, so that a readback or a change of the material map between two steps
// (clb_geometry_update refreshes them before it converts voxels) does not alter them.
static void refresh_neumann(clb_handle* h) {
    if (h->neu_iter == h->ade_iters) return;
    h->neu_iter = h->ade_iters;
    const int odd = (int)(h->ade_iters & 1);
    switch (h->ade_prec) {
        case CLB_F64: launch_neumann<double, double>(h, odd); break;
        case CLB_F32: launch_neumann<float, float>(h, odd); break;
        default: launch_neumann<__half, float>(h, odd); break;
    }
}

// ------------------------------------------------------------------ batched step of many domains

__device__ __forceinline__ int batch_find(const int64_t* off, int n, int64_t t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// One transport step of every domain (no abiotic law, no dissolution). Each CTA takes a
// contiguous run of the tile table (tiles are in domain order) and copies a tile's domain
// description into shared memory when it differs from the previous tile's; the per-node code is
// the single-domain step's, its parameters read from that copy.
template <typename TS, typename TC, bool ODD, int NM>
__global__ void __launch_bounds__(ADE_THREADS, (ade_minb<TC, NM>() > 6 ? 6 : ade_minb<TC, NM>()))
    k_ade_batch(const BatchView B) {
    extern __shared__ __align__(16) unsigned char ade_smem[];
    __shared__ __align__(16) BatchDomain sd;
    const AdeFrame<TC> F = ade_frame<TC, NM>(ade_smem, 0);
    const int tid = threadIdx.x;
    AdeExtra X;
    X.iface = nullptr;
    X.xidx = nullptr;
    X.xdc = nullptr;
    X.ng = 0;
    const int per = (B.nat + gridDim.x - 1) / gridDim.x;
    const int t0 = blockIdx.x * per, t1 = min(B.nat, t0 + per);
    int cur = -1;
    for (int t = t0; t < t1; ++t) {
        const BatchTile T = B.atiles[t];
        if (T.d != cur) {
            __syncthreads();  // every thread is done with the previous domain
            const uint64_t* src = reinterpret_cast<const uint64_t*>(B.dom + T.d);
            uint64_t* dst = reinterpret_cast<uint64_t*>(&sd);
            for (int q = tid; q < (int)(sizeof(BatchDomain) / 8); q += ADE_THREADS) dst[q] = src[q];
            __syncthreads();
            cur = T.d;
        }
        for (int64_t k = T.first + tid; k < T.first + T.count; k += ADE_THREADS)
            ade_node<TS, TC, ODD, NM, 0>((TS*)sd.g, sd.imm, sd.bio, (const TC*)sd.u, sd.as, sd.neu, sd.ap, sd.n_mobile,
                                         sd.mob, sd.akw, sd.ake, X, F, k);
    }
}

// the Neumann planes of every domain (as k_ade_neumann): one thread per pixel of a face that some
// species treats as Neumann; the inner neighbour's storage locations serve all those species
template <typename TS, typename TC>
__global__ void k_neumann_batch(const BatchView B, int odd) {
    const int64_t total = B.foff_faces[B.nfaces];
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int j = batch_find(B.foff_faces, B.nfaces, t);
        const NeumannFace J = B.faces[j];
        const BatchDomain& d = B.dom[J.d];
        const Geom G = d.ap.g;
        const int p = (int)(t - B.foff_faces[j]);
        const int xb = J.side == 0 ? 0 : G.nx - 1, xi = J.side == 0 ? 1 : G.nx - 2;
        const int64_t nb = (int64_t)xb * G.plane + p, ni = (int64_t)xi * G.plane + p;
        const int db = d.ap.dyn[d.mat[nb]], di = d.ap.dyn[d.mat[ni]];
        if (!(db == ADE_PORE || db == ADE_BIO) || !(di == ADE_PORE || di == ADE_BIO)) continue;
        int x, y, z;
        decode(G, ni, x, y, z);
        const TS* g0 = (const TS*)d.g;
        const TS* loc[7];
#pragma unroll
        for (int i = 0; i < 7; ++i) loc[i] = natural_slot<const TS, 7>(d.as, G, g0, (const TS*)d.glink, ni, x, y, z, i, odd);
        const int S = d.ap.S;
        for (int s = 0; s < S; ++s) {
            const int m = d.ap.slot[s];
            if (m < 0 || (J.side == 0 ? d.ap.ltype[s] : d.ap.rtype[s]) != CLB_NEUMANN) continue;
            const int64_t sh = (int64_t)m * d.as.SS;
            const double c0 = d.ap.c0[s];
            TC pop[7];
#pragma unroll
            for (int i = 0; i < 7; ++i)
                pop[i] = loc[i] ? ld<TS, TC>(loc[i] + sh) : (TC)(q7w(i) * (c0 - ade_sigma<TC>()));
            double r = ade_sigma<TC>();
#pragma unroll
            for (int i = 0; i < 7; ++i) r += (double)pop[i];
            d.neu[((int64_t)s * 2 + J.side) * G.plane + p] = r;
        }
    }
}

void launch_neumann_batch(const BatchView& B, int prec, bool odd, int grid, cudaStream_t st) {
    if (B.nfaces == 0) return;
    switch (prec) {
        case CLB_F64: k_neumann_batch<double, double><<<grid, 256, 0, st>>>(B, odd ? 1 : 0); break;
        case CLB_F32: k_neumann_batch<float, float><<<grid, 256, 0, st>>>(B, odd ? 1 : 0); break;
        default: k_neumann_batch<__half, float><<<grid, 256, 0, st>>>(B, odd ? 1 : 0); break;
    }
}

// `resident` blocks per SM the shared-memory carveout is sized for (the rest of the SM stays L1,
// which the odd step's neighbour gathers reuse); set on every launch, since the batch's autotuner
// tries several
template <typename TS, typename TC, bool ODD, int NM>
static void launch_ade_batch_t(const BatchView& B, int grid_mult, int resident, int num_sms, cudaStream_t st) {
    auto kern = k_ade_batch<TS, TC, ODD, NM>;
    const int sm = ade_slot_bytes<TC, NM>();
    const int per_block = sm + (int)sizeof(BatchDomain) + 1024;  // the runtime reserves 1 KB per block
    const int fit = std::max(1, std::min(resident, (228 * 1024) / per_block));
    const int pct = std::min(100, (int)((100LL * fit * per_block + 228 * 1024 - 1) / (228 * 1024)));
    if (sm > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, ADE_THREADS, sm) != cudaSuccess || nb < 1) nb = 1;
    nb = std::min(nb, fit);
    const int grid = std::max(1, std::min(nb * num_sms * grid_mult, B.nat));
    kern<<<grid, ADE_THREADS, sm, st>>>(B);
}

template <typename TS, typename TC, bool ODD>
static void launch_ade_batch_p(const BatchView& B, int nm, int grid_mult, int resident, int num_sms, cudaStream_t st) {
    if (nm <= 1) launch_ade_batch_t<TS, TC, ODD, 1>(B, grid_mult, resident, num_sms, st);
    else if (nm <= 2) launch_ade_batch_t<TS, TC, ODD, 2>(B, grid_mult, resident, num_sms, st);
    else if (nm <= 4) launch_ade_batch_t<TS, TC, ODD, 4>(B, grid_mult, resident, num_sms, st);
    else if (nm <= 8) launch_ade_batch_t<TS, TC, ODD, 8>(B, grid_mult, resident, num_sms, st);
    else launch_ade_batch_t<TS, TC, ODD, 16>(B, grid_mult, resident, num_sms, st);
}

void launch_ade_batch(const BatchView& B, int prec, bool odd, int nm, int grid_mult, int resident, int num_sms,
                      cudaStream_t st) {
    switch (prec) {
        case CLB_F64:
            if (odd) launch_ade_batch_p<double, double, true>(B, nm, grid_mult, resident, num_sms, st);
            else launch_ade_batch_p<double, double, false>(B, nm, grid_mult, resident, num_sms, st);
            break;
        case CLB_F32:
            if (odd) launch_ade_batch_p<float, float, true>(B, nm, grid_mult, resident, num_sms, st);
            else launch_ade_batch_p<float, float, false>(B, nm, grid_mult, resident, num_sms, st);
            break;
        default:
            if (odd) launch_ade_batch_p<__half, float, true>(B, nm, grid_mult, resident, num_sms, st);
            else launch_ade_batch_p<__half, float, false>(B, nm, grid_mult, resident, num_sms, st);
            break;
    }
}

// ------------------------------------------------------------------ persistent batched steps
// One launch advances every domain of a batch by several steps. The work is a table of items,
// each a tile of one lattice of one domain at one step of the launch (flow nodes, the Neumann
// planes of the domain's species, transport nodes). CTAs take items in table order from one
// ticket counter; an item starts once the items it depends on are done: the same lattice of the
// same domain at the previous step (an AA step reads what the neighbours wrote), and, for the
// transport tiles, the Neumann planes of their own step. Finished items are counted per (step,
// lattice, domain). The table orders step s of domain d by d + W s (W, the lag, a schedule
// parameter), so step s + 1 of a domain follows step s of it while its populations are still in
// L2, and every item depends only on items earlier in the table. Tickets are taken in order, so
// an awaited item is held by a CTA that is running: the schedule cannot deadlock. Each wait is
// still bounded (wait_ns) and gives up with a status rather than spin for ever.
//
// Visibility across CTAs: the finishing CTA's threads store, meet at a barrier, and one thread
// fences and increments the counter; the waiting CTA's thread reads the counter, fences, and
// meets its threads at a barrier before any of them reads -- the pattern of a grid-wide barrier.
// No pointer of the launch is a read-only kernel argument, so no load goes through the
// non-coherent read-only path.

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// waits until *c >= target; false when the wait gave up (limit reached or another wait gave up)
__device__ __forceinline__ bool persist_wait(const int* c, int target, const int* status, int64_t limit_ns) {
    const uint64_t t0 = global_ns();
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        if (*(const volatile int*)c >= target) {
            __threadfence();
            return true;
        }
        if (*(const volatile int*)status) return false;
        if ((it & 31u) == 31u && (int64_t)(global_ns() - t0) > limit_ns) return false;
        __nanosleep(64);
    }
    return false;
}

// coherent (L2) read of one stored population
template <typename TS, typename TC>
__device__ __forceinline__ TC ld_cg(const TS* p) {
    if constexpr (std::is_same<TS, __half>::value) return (TC)(__half2float(__ldcg(p)) * HALF_INV);
    else return (TC)__ldcg(p);
}

// k_neumann_batch's value for plane pixel p of job J, with coherent reads
template <typename TS, typename TC>
__device__ __forceinline__ void persist_neumann_pixel(const BatchDomain& d, const NeumannJob& J, int p, int odd) {
    const Geom G = d.ap.g;
    const int xb = J.side == 0 ? 0 : G.nx - 1, xi = J.side == 0 ? 1 : G.nx - 2;
    const int64_t nb = (int64_t)xb * G.plane + p, ni = (int64_t)xi * G.plane + p;
    const int db = d.ap.dyn[d.mat[nb]], di = d.ap.dyn[d.mat[ni]];
    if (!(db == ADE_PORE || db == ADE_BIO) || !(di == ADE_PORE || di == ADE_BIO)) return;
    const double c0 = d.ap.c0[J.s];
    const TS* f = (const TS*)d.g + (int64_t)J.m * d.as.SS;
    const TS* link = (const TS*)d.glink + (int64_t)J.m * d.as.SS;
    int x, y, z;
    decode(G, ni, x, y, z);
    double r = ade_sigma<TC>();
    for (int i = 0; i < 7; ++i) {
        const TS* q = natural_slot<const TS, 7>(d.as, G, f, link, ni, x, y, z, i, odd);
        const TC v = q ? ld_cg<TS, TC>(q) : (TC)(q7w(i) * (c0 - ade_sigma<TC>()));
        r += (double)v;
    }
    d.neu[((int64_t)J.s * 2 + J.side) * G.plane + p] = r;
}

// MINB: resident CTAs per SM the registers are budgeted for (4: no spills; 6 and 8 trade some
// spilled registers for more warps to hide memory latency)
template <typename TS, typename TC, int NM, int MINB>
__global__ void __launch_bounds__(ADE_THREADS, MINB) k_batch_persistent(const PersistView V) {
    extern __shared__ __align__(16) unsigned char ade_smem[];
    const AdeFrame<TC> F = ade_frame<TC, NM>(ade_smem, 0);
    __shared__ __align__(16) BatchDomain sd;
    __shared__ int s_next, s_abort;
    const int tid = threadIdx.x;
    const int ndom = V.B.ndom;
    AdeExtra X;
    X.iface = nullptr;
    X.xidx = nullptr;
    X.xdc = nullptr;
    X.ng = 0;
    if (tid == 0) s_next = atomicAdd(V.ticket, 1);
    __syncthreads();
    int t = s_next;
    while (t < V.n_items) {
        const BatchItem it = V.items[t];
        if (tid == 0) {
            const int s = it.step, d = it.d;
            const int* w = nullptr;
            int target = 0;
            if (it.kind == BI_FLOW) {
                if (s > 0) { w = V.done + ((s - 1) * 3 + BI_FLOW) * ndom + d; target = V.need[BI_FLOW * ndom + d]; }
            } else if (it.kind == BI_NEUMANN) {
                if (s > 0) { w = V.done + ((s - 1) * 3 + BI_TRANSPORT) * ndom + d; target = V.need[BI_TRANSPORT * ndom + d]; }
            } else if (V.need[BI_NEUMANN * ndom + d] > 0) {
                w = V.done + (s * 3 + BI_NEUMANN) * ndom + d;
                target = V.need[BI_NEUMANN * ndom + d];
            } else if (s > 0) {
                w = V.done + ((s - 1) * 3 + BI_TRANSPORT) * ndom + d;
                target = V.need[BI_TRANSPORT * ndom + d];
            }
            bool ok = w ? persist_wait(w, target, V.status, V.wait_ns) : (*(const volatile int*)V.status == 0);
            if (!ok) atomicExch(V.status, 1);
            s_abort = ok ? 0 : 1;
            s_next = atomicAdd(V.ticket, 1);
        }
        // the item's domain into shared memory
        {
            const uint64_t* src = reinterpret_cast<const uint64_t*>(V.B.dom + it.d);
            uint64_t* dst = reinterpret_cast<uint64_t*>(&sd);
            for (int q = tid; q < (int)(sizeof(BatchDomain) / 8); q += ADE_THREADS) dst[q] = src[q];
        }
        __syncthreads();
        const int tn = s_next;
        if (s_abort) break;
        const int64_t k0 = it.first, k1 = it.first + it.count;
        if (it.kind == BI_FLOW) {
            TS* f = (TS*)sd.f;
            TS* fl = (TS*)sd.flink;
            if ((V.fodd ^ it.step) & 1) {
                for (int64_t k = k0 + tid; k < k1; k += ADE_THREADS)
                    flow_node<TS, TC, true>(f, fl, sd.fs, sd.fp, k, sd.fkw, sd.fke);
            } else {
                for (int64_t k = k0 + tid; k < k1; k += ADE_THREADS)
                    flow_node<TS, TC, false>(f, fl, sd.fs, sd.fp, k, sd.fkw, sd.fke);
            }
        } else if (it.kind == BI_NEUMANN) {
            const int odd = (V.aodd ^ it.step) & 1;
            for (int j = V.jbeg[it.d]; j < V.jbeg[it.d + 1]; ++j) {
                const NeumannJob J = V.B.jobs[j];
                for (int p = tid; p < sd.ap.g.plane; p += ADE_THREADS) persist_neumann_pixel<TS, TC>(sd, J, p, odd);
            }
        } else {
            TS* g = (TS*)sd.g;
            if ((V.aodd ^ it.step) & 1) {
                for (int64_t k = k0 + tid; k < k1; k += ADE_THREADS)
                    ade_node<TS, TC, true, NM, 0>(g, sd.imm, sd.bio, (const TC*)sd.u, sd.as, sd.neu, sd.ap, sd.n_mobile,
                                                  sd.mob, sd.akw, sd.ake, X, F, k);
            } else {
                for (int64_t k = k0 + tid; k < k1; k += ADE_THREADS)
                    ade_node<TS, TC, false, NM, 0>(g, sd.imm, sd.bio, (const TC*)sd.u, sd.as, sd.neu, sd.ap, sd.n_mobile,
                                                   sd.mob, sd.akw, sd.ake, X, F, k);
            }
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicAdd(V.done + (it.step * 3 + it.kind) * ndom + it.d, 1);
        }
        t = tn;
    }
}

template <typename TS, typename TC, int NM, int MINB>
static void persist_launch_t(const PersistView& V, int blocks_per_sm, int num_sms, cudaStream_t st) {
    // the shared-memory attribute was set on this device by batch_persistent_resident (batch set-up)
    k_batch_persistent<TS, TC, NM, MINB><<<blocks_per_sm * num_sms, ADE_THREADS, ade_slot_bytes<TC, NM>(), st>>>(V);
}

template <typename TS, typename TC, int NM, int MINB>
static int persist_resident_t() {
    auto kern = k_batch_persistent<TS, TC, NM, MINB>;
    const int sm = ade_slot_bytes<TC, NM>();
    cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (const void*)kern, ADE_THREADS, sm) != cudaSuccess) b = 1;
    return std::max(1, b);
}

// register budgets built: 4 for every lattice; 6 and 8 also for FP32 arithmetic with up to 4
// mobile species (the ensemble sweeps)
int persist_minb(int prec, int nm, int minb) {
    if (prec != CLB_F64 && nm <= 4 && (minb == 6 || minb == 8)) return minb;
    return 4;
}

#define CLB_PERSIST_M(F, TS, TC, NMV, ...)                                                                     \
    (mb == 8 ? F<TS, TC, NMV, 8>(__VA_ARGS__) : mb == 6 ? F<TS, TC, NMV, 6>(__VA_ARGS__) : F<TS, TC, NMV, 4>(__VA_ARGS__))
#define CLB_PERSIST_NM(F, TS, TC, ...)                                                                         \
    (nm <= 1 ? CLB_PERSIST_M(F, TS, TC, 1, __VA_ARGS__)                                                       \
     : nm <= 2 ? CLB_PERSIST_M(F, TS, TC, 2, __VA_ARGS__)                                                     \
     : nm <= 4 ? CLB_PERSIST_M(F, TS, TC, 4, __VA_ARGS__)                                                     \
     : nm <= 8 ? F<TS, TC, 8, 4>(__VA_ARGS__) : F<TS, TC, 16, 4>(__VA_ARGS__))

void launch_batch_persistent(const PersistView& V, int prec, int nm, int minb, int blocks_per_sm, int num_sms,
                             cudaStream_t st) {
    const int mb = persist_minb(prec, nm, minb);
    switch (prec) {
        case CLB_F64: nm <= 1 ? persist_launch_t<double, double, 1, 4>(V, blocks_per_sm, num_sms, st)
                      : nm <= 2 ? persist_launch_t<double, double, 2, 4>(V, blocks_per_sm, num_sms, st)
                      : nm <= 4 ? persist_launch_t<double, double, 4, 4>(V, blocks_per_sm, num_sms, st)
                      : nm <= 8 ? persist_launch_t<double, double, 8, 4>(V, blocks_per_sm, num_sms, st)
                                : persist_launch_t<double, double, 16, 4>(V, blocks_per_sm, num_sms, st);
                      break;
        case CLB_F32: CLB_PERSIST_NM(persist_launch_t, float, float, V, blocks_per_sm, num_sms, st); break;
        default: CLB_PERSIST_NM(persist_launch_t, __half, float, V, blocks_per_sm, num_sms, st); break;
    }
}

int batch_persistent_resident(int prec, int nm, int minb) {
    const int mb = persist_minb(prec, nm, minb);
    switch (prec) {
        case CLB_F64: return nm <= 1 ? persist_resident_t<double, double, 1, 4>()
                           : nm <= 2 ? persist_resident_t<double, double, 2, 4>()
                           : nm <= 4 ? persist_resident_t<double, double, 4, 4>()
                           : nm <= 8 ? persist_resident_t<double, double, 8, 4>()
                                     : persist_resident_t<double, double, 16, 4>();
        case CLB_F32: return CLB_PERSIST_NM(persist_resident_t, float, float);
        default: return CLB_PERSIST_NM(persist_resident_t, __half, float);
    }
}
#undef CLB_PERSIST_NM
#undef CLB_PERSIST_M

void ade_refresh_neumann(clb_handle* h) { refresh_neumann(h); }

// A transport step that meets a NaN or infinite density sets a host-mapped flag; the run then
// stops cleanly, as the reference stops on non-finite biomass or flow energy
// (complab.cpp:2796, 3116-3117): the next clb_ade_step, and clb_synchronize once that step has
// completed, return CLB_NONFINITE. Setting a species' populations clears the flag.
clb_status ade_nonfinite_check(clb_handle* h) {
    if (h->h_flags && ((volatile int*)h->h_flags)[0])
        return fail(h, CLB_NONFINITE, "a transport step met a non-finite (NaN or Inf) concentration");
    return CLB_OK;
}

clb_status ade_step(clb_handle* h, int n) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (h->M > 0 && h->d_bio == nullptr) return fail(h, CLB_INVALID_ARG, "biomass missing");
    if (ade_nonfinite_check(h) != CLB_OK) return CLB_NONFINITE;
    for (int k = 0; k < n; ++k) {
        const bool odd = (h->ade_iters & 1) != 0;
        if (h->ap.dis_on) {
            clb_status st = dissolution_pre_step(h);
            if (st != CLB_OK) return st;
        }
        refresh_neumann(h);
        switch (h->ade_prec) {
            case CLB_F64: if (odd) launch_ade_t<double, double, true>(h); else launch_ade_t<double, double, false>(h); break;
            case CLB_F32: if (odd) launch_ade_t<float, float, true>(h); else launch_ade_t<float, float, false>(h); break;
            default: if (odd) launch_ade_t<__half, float, true>(h); else launch_ade_t<__half, float, false>(h); break;
        }
        h->ade_iters += 1;
        if (h->spec_mode != CLB_SPEC_OFF) {
            clb_status st = speciation_step(h);
            if (st != CLB_OK) return st;
        }
    }
    return cuda_check(h, cudaGetLastError(), "ade step");
}

clb_status ade_couple(clb_handle* h) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (!h->flow_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_flow_init first");
    return flow_velocity_at(h, h->ade_sp.node, h->ade_sp.K, h->d_u, h->ade_sp.K, h->ade_prec == CLB_F64 ? 0 : 1);
}

static clb_status ade_populations_i(clb_handle* h, int s, double* host, int shifted = 1) {
    if (h->ap.slot[s] < 0) return fail(h, CLB_INVALID_ARG, "not a mobile species");
    const int m = h->ap.slot[s];
    double* buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, sizeof(double) * 7 * (size_t)h->g.N);
    if (e != cudaSuccess) return cuda_check(h, e, "population buffer");
    const int odd = (int)(h->ade_iters & 1);
    const int grid = h->num_sms * 8;
    const size_t off = (size_t)m * h->ade_sp.SS, loff = off;
    const SparseView S = view_of(h->ade_sp);
    const double c0 = h->ap.c0[s];
    switch (h->ade_prec) {
        case CLB_F64: k_ade_get_pops<double><<<grid, 256, 0, h->stream>>>((const double*)h->d_g + off, (const double*)h->d_glink + loff, S, h->g, odd, c0, shifted, buf); break;
        case CLB_F32: k_ade_get_pops<float><<<grid, 256, 0, h->stream>>>((const float*)h->d_g + off, (const float*)h->d_glink + loff, S, h->g, odd, c0, shifted, buf); break;
        default: k_ade_get_pops<__half><<<grid, 256, 0, h->stream>>>((const __half*)h->d_g + off, (const __half*)h->d_glink + loff, S, h->g, odd, c0, shifted, buf); break;
    }
    e = cudaMemcpyAsync(host, buf, sizeof(double) * 7 * (size_t)h->g.N, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(buf);
    return cuda_check(h, e, "population copy");
}

clb_status ade_populations(clb_handle* h, int s, double* host, int shifted) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (s < 0 || s >= h->S) return fail(h, CLB_INVALID_ARG, "species index out of range");
    return ade_populations_i(h, h->u2i[s], host, shifted);
}

clb_status ade_set_populations(clb_handle* h, int s, const double* host, int shifted) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (s < 0 || s >= h->S) return fail(h, CLB_INVALID_ARG, "species index out of range");
    if (h->h_flags) {
        cudaStreamSynchronize(h->stream);  // no step in flight may set the flag after the clear
        h->h_flags[0] = 0;
    }
    s = h->u2i[s];
    if (h->ap.slot[s] < 0) return fail(h, CLB_INVALID_ARG, "not a mobile species");
    const int m = h->ap.slot[s];
    double* buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, sizeof(double) * 7 * (size_t)h->g.N);
    if (e != cudaSuccess) return cuda_check(h, e, "population buffer");
    cudaMemcpy(buf, host, sizeof(double) * 7 * (size_t)h->g.N, cudaMemcpyHostToDevice);
    const int odd = (int)(h->ade_iters & 1);
    const int grid = h->num_sms * 8;
    const size_t off = (size_t)m * h->ade_sp.SS, loff = off;
    const SparseView S = view_of(h->ade_sp);
    switch (h->ade_prec) {
        case CLB_F64: k_ade_set_pops<double><<<grid, 256, 0, h->stream>>>((double*)h->d_g + off, (double*)h->d_glink + loff, S, h->g, odd, shifted, buf); break;
        case CLB_F32: k_ade_set_pops<float><<<grid, 256, 0, h->stream>>>((float*)h->d_g + off, (float*)h->d_glink + loff, S, h->g, odd, shifted, buf); break;
        default: k_ade_set_pops<__half><<<grid, 256, 0, h->stream>>>((__half*)h->d_g + off, (__half*)h->d_glink + loff, S, h->g, odd, shifted, buf); break;
    }
    e = cudaStreamSynchronize(h->stream);
    cudaFree(buf);
    h->neu_iter = -1;
    return cuda_check(h, e, "set populations");
}

// computeDensity: BGK nodes of a Dirichlet / Neumann plane report the stored value; every
// other node the sum of its populations + 1; immobile species their field (zero off the nodes).
clb_status ade_density(clb_handle* h, int s, double* host) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (s < 0 || s >= h->S) return fail(h, CLB_INVALID_ARG, "species index out of range");
    s = h->u2i[s];
    const size_t N = (size_t)h->g.N;
    if (h->ap.slot[s] < 0)
        return cuda_check(h, cudaMemcpy(host, h->d_imm + (size_t)s * N, sizeof(double) * N, cudaMemcpyDeviceToHost), "immobile copy");
    // the Neumann planes' stored values as the reference holds them after the last stream
    refresh_neumann(h);
    if (!h->d_stage) {
        cudaError_t e = cudaMalloc(&h->d_stage, sizeof(double) * N);
        if (e != cudaSuccess) return cuda_check(h, e, "field staging buffer");
    }
    const int m = h->ap.slot[s];
    const int odd = (int)(h->ade_iters & 1);
    const size_t off = (size_t)m * h->ade_sp.SS;
    const SparseView Sv = view_of(h->ade_sp);
    const double* neu = h->d_neu + (size_t)s * 2 * h->g.plane;
    const int grid = h->num_sms * 8;
#define CLB_DENS(TS)                                                                                              \
    k_ade_density<TS><<<grid, 256, 0, h->stream>>>((const TS*)h->d_g + off, (const TS*)h->d_glink + off, Sv, h->d_mat, \
                                                   h->ap, s, odd, neu, h->d_stage)
    switch (h->ade_prec) {
        case CLB_F64: CLB_DENS(double); break;
        case CLB_F32: CLB_DENS(float); break;
        default: CLB_DENS(__half); break;
    }
#undef CLB_DENS
    cudaError_t e = cudaMemcpyAsync(host, h->d_stage, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return cuda_check(h, e, "concentration copy");
}

clb_status ade_biomass(clb_handle* h, int m, double* host) {
    if (!h->ade_ready || m < 0 || m >= h->M) return fail(h, CLB_INVALID_ARG, "no such biomass field");
    h->ca_full = true;
    return cuda_check(h, cudaMemcpy(host, h->d_bio + (size_t)m * h->g.N, sizeof(double) * h->g.N, cudaMemcpyDeviceToHost), "biomass copy");
}

clb_status ade_set_biomass_field(clb_handle* h, int m, const double* host) {
    if (!h->ade_ready || m < 0 || m >= h->M) return fail(h, CLB_INVALID_ARG, "no such biomass field");
    h->ca_full = true;
    clb_status st = cuda_check(
        h, cudaMemcpy(h->d_bio + (size_t)m * h->g.N, host, sizeof(double) * h->g.N, cudaMemcpyHostToDevice), "biomass copy");
    return st == CLB_OK ? refresh_bflag(h) : st;
}

__global__ void k_u_to_dense(const void* __restrict__ u, int f64, const int32_t* __restrict__ node, int64_t K,
                             int64_t N, double* __restrict__ out) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x)
        for (int a = 0; a < 3; ++a)
            out[a * N + node[k]] = f64 ? ((const double*)u)[a * K + k] : (double)((const float*)u)[a * K + k];
}

__global__ void k_u_to_compact(const double* __restrict__ in, int f64, const int32_t* __restrict__ node, int64_t K,
                               int64_t N, void* __restrict__ u) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x)
        for (int a = 0; a < 3; ++a) {
            if (f64) ((double*)u)[a * K + k] = in[a * N + node[k]];
            else ((float*)u)[a * K + k] = (float)in[a * N + node[k]];
        }
}

clb_status ade_velocity(clb_handle* h, double* host) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    const size_t N = (size_t)h->g.N;
    double* tmp = nullptr;
    cudaError_t e = cudaMalloc(&tmp, sizeof(double) * 3 * N);
    if (e != cudaSuccess) return cuda_check(h, e, "velocity buffer");
    cudaMemsetAsync(tmp, 0, sizeof(double) * 3 * N, h->stream);
    k_u_to_dense<<<h->num_sms * 4, 256, 0, h->stream>>>(h->d_u, h->ade_prec == CLB_F64, h->ade_sp.node, h->ade_sp.K, N, tmp);
    e = cudaMemcpyAsync(host, tmp, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(tmp);
    return cuda_check(h, e, "velocity copy");
}

clb_status ade_set_velocity(clb_handle* h, const double* host) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    const size_t N = (size_t)h->g.N;
    double* tmp = nullptr;
    cudaError_t e = cudaMalloc(&tmp, sizeof(double) * 3 * N);
    if (e != cudaSuccess) return cuda_check(h, e, "velocity buffer");
    e = cudaMemcpyAsync(tmp, host, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, h->stream);
    k_u_to_compact<<<h->num_sms * 4, 256, 0, h->stream>>>(tmp, h->ade_prec == CLB_F64, h->ade_sp.node, h->ade_sp.K, N, h->d_u);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(tmp);
    return cuda_check(h, e, "velocity upload");
}

// Runs the reduction kernels on the handle's stream with scratch `buf` (reduce_scratch_doubles(S, M)
// doubles) and reads the result back.
static clb_status reduce_into(clb_handle* h, double* buf, clb_stats* out) {
    std::memset(out, 0, sizeof(*out));
    const int S = h->S, M = h->M;
    const int nq = 4 * S + M + 2;
    const int blocks = reduce_blocks(h);
    double* fin = buf + (size_t)(5 * S + M + 1) * blocks;
    const SparseView Sv = view_of(h->ade_sp);
    const dim3 grid(blocks, S + 1);
    const int odd = (int)(h->ade_iters & 1);
    switch (h->ade_prec) {
        case CLB_F64: k_ade_reduce<double><<<grid, RED_THREADS, 0, h->stream>>>((const double*)h->d_g, (const double*)h->d_glink, h->d_imm, h->d_bio, Sv, h->ap, buf, h->ade_west_end, h->ade_east_begin, odd); break;
        case CLB_F32: k_ade_reduce<float><<<grid, RED_THREADS, 0, h->stream>>>((const float*)h->d_g, (const float*)h->d_glink, h->d_imm, h->d_bio, Sv, h->ap, buf, h->ade_west_end, h->ade_east_begin, odd); break;
        default: k_ade_reduce<__half><<<grid, RED_THREADS, 0, h->stream>>>((const __half*)h->d_g, (const __half*)h->d_glink, h->d_imm, h->d_bio, Sv, h->ap, buf, h->ade_west_end, h->ade_east_begin, odd); break;
    }
    k_reduce_combine<<<1, 128, 0, h->stream>>>(buf, blocks, S, M, fin);
    double q[4 * CLB_MAX_SPECIES + CLB_MAX_MICROBES + 2];
    cudaError_t e = cudaMemcpyAsync(q, fin, sizeof(double) * nq, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_check(h, e, "reduce");
    for (int i = 0; i < S; ++i) {
        const int s = h->i2u[i];
        out->total[s] = q[i];
        out->content[s] = q[S + i];
        out->min_c[s] = q[2 * S + i];
        out->max_c[s] = q[3 * S + i];
    }
    for (int mb = 0; mb < M; ++mb) out->biomass[mb] = q[4 * S + mb];
    out->nonfinite = (int64_t)q[4 * S + M];
    out->open_voxels = (int64_t)q[4 * S + M + 1];
    out->ade_iterations = h->ade_iters;
    return CLB_OK;
}

// clb_reduce: the scratch is the handle's own buffer, allocated by ade_init.
clb_status ade_reduce(clb_handle* h, clb_stats* out) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    return reduce_into(h, h->d_red, out);
}

// ------------------------------------------------------------------ reduction without allocation
//
// clb_reduce_noalloc computes what clb_reduce computes, but takes its per-block partial sums from
// a fixed buffer compiled into the library instead of a cudaMalloc'd one, and combines them on
// the device, so the call neither allocates nor frees memory, on the device or on the host. It
// is meant for callers that must not allocate while they monitor a run: an application whose
// device memory is all handed to its own pool (where a cudaMalloc fails), or a loop that cannot
// afford the device-wide synchronisation a cudaFree implies.
//
// Limit: the buffer holds REDUCE_SCRATCH_DOUBLES doubles; a call needs blocks x (5 S + M + 1) +
// (4 S + M + 2) of them (blocks = 2 x the SM count, S species, M microbes: 26,418 on a 148-SM B200
// at the largest S = 16, M = 8) and is refused with CLB_INVALID_ARG when that does not fit. Every word of the buffer a call reads was written
// earlier in the same call, so nothing has to start at zero. The buffer is one per device and
// shared by all handles on it: two calls that overlap in time on one device (different host
// threads, or different streams without ordering between them) race on it and return wrong
// sums. The first call on each device looks up the buffer's device address (set-up); make that
// first call before any stream capture begins.
constexpr int REDUCE_SCRATCH_DOUBLES = 65536;  // 512 KiB
static __device__ __align__(256) double g_reduce_scratch[REDUCE_SCRATCH_DOUBLES];

static std::mutex g_scratch_mutex;
constexpr int MAX_DEVICES = 64;
static double* g_scratch_addr[MAX_DEVICES] = {};

// Device address of g_reduce_scratch on the current device (looked up once per device).
static clb_status reduce_scratch(clb_handle* h, double** ptr) {
    if (h->device < 0 || h->device >= MAX_DEVICES) return fail(h, CLB_INVALID_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[h->device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_reduce_scratch);
        if (e != cudaSuccess) return cuda_check(h, e, "scratch buffer address");
        g_scratch_addr[h->device] = (double*)p;
    }
    *ptr = g_scratch_addr[h->device];
    return CLB_OK;
}

clb_status ade_reduce_noalloc(clb_handle* h, clb_stats* out) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    std::memset(out, 0, sizeof(*out));
    if (reduce_scratch_doubles(h->S, h->M, reduce_blocks(h)) > REDUCE_SCRATCH_DOUBLES)
        return fail(h, CLB_INVALID_ARG, "reduction needs more scratch than the fixed 65536-double buffer holds");
    double* part = nullptr;
    clb_status st = reduce_scratch(h, &part);
    if (st != CLB_OK) return st;
    return reduce_into(h, part, out);
}

}  // namespace clb
