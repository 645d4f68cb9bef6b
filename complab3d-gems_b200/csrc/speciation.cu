// speciation.cu -- per-voxel equilibrium speciation in FP64 on the GPU.
//
// Reference behaviour: the species model and totals of EquilibriumChemistry
// (complab3d_processors_part4_eqsolver.hh: calc_species :450-505, log10 c clamped to [-30, 1],
// c to [1e-30, 10]; calc_component_totals :520-535; a species takes part when its tableau row
// has an entry above 1e-10, :386-395) solved by the reference's Newton-Raphson formulation
// (complab3d_processors_part4_eqsolver_NR_reserve.hh:309-640): residual F = S^T c - T,
// Jacobian J_jk = ln10 sum_i S_ij S_ik c_i, partial-pivot elimination (singular below 1e-30),
// Armijo backtracking (at most 40 halvings, sufficient decrease 1e-4 alpha), converged when
// |F| < tol or when the step is below tol/1000 with |F| < 100 tol; inside the loop the species
// are unclamped and a step moves no log10 concentration by more than 2 (see eq_species_free).
// The speciation step
// (run_equilibrium_biotic, :1393-1545) caps each change at max(1e-9, 0.1 |C|), floors the new
// concentration at 1e-20 and deposits t_i dC when |dC| > 1e-12.
//
// One thread solves one voxel; the tableau sits in the kernel parameter space (constant bank).
#include "sparse.cuh"
#include "speciation.cuh"

#include <algorithm>
#include <cstring>

namespace clb {

// The solver is built for tableau shapes fixed at compile time (NC components, NS species; the
// loops unroll and the per-voxel arrays live in registers) and for any shape (NC = NS = 0: sizes
// from the parameters, arrays of the largest size in local memory). The arithmetic and its order
// are the same in every build.
#define EQ_NC(NC) ((NC) > 0 ? (NC) : CLB_MAX_COMPONENTS)
#define EQ_NS(NS) ((NS) > 0 ? (NS) : CLB_MAX_EQ_SPECIES)

template <int NC, int NS>
__device__ __forceinline__ void eq_species(const SpecParams& P, const double* x, const double* init, double* c) {
    const int nc = NC > 0 ? NC : P.nc, ns = NS > 0 ? NS : P.ns;
#pragma unroll (NS > 0 ? NS : 1)
    for (int i = 0; i < ns; ++i) {
        if (!P.eq[i]) {
            c[i] = init[i] > EQ_MIN_C ? fmin(init[i], EQ_MAX_C) : EQ_MIN_C;
            continue;
        }
        double lc = P.logK[i];
#pragma unroll (NC > 0 ? NC : 1)
        for (int j = 0; j < nc; ++j) lc = fma(P.S[i * CLB_MAX_COMPONENTS + j], x[j], lc);
        lc = fmax(fmin(lc, EQ_MAX_LOG), EQ_MIN_LOG);
        double v = exp10(lc);
        if (isnan(v) || isinf(v)) v = init[i] > EQ_MIN_C ? init[i] : EQ_MIN_C;
        c[i] = fmax(fmin(v, EQ_MAX_C), EQ_MIN_C);
    }
}

// Inside the Newton loop the species follow mass action without the [1e-30, 10] clamps (a
// species saturated at a clamp has a zero derivative the Jacobian does not see, and the iteration
// stalls from a far initial guess); the clamps apply to the answer only.
template <int NC, int NS>
__device__ __forceinline__ void eq_species_free(const SpecParams& P, const double* x, const double* init, double* c) {
    const int nc = NC > 0 ? NC : P.nc, ns = NS > 0 ? NS : P.ns;
#pragma unroll (NS > 0 ? NS : 1)
    for (int i = 0; i < ns; ++i) {
        if (!P.eq[i]) {
            c[i] = init[i] > EQ_MIN_C ? fmin(init[i], EQ_MAX_C) : EQ_MIN_C;
            continue;
        }
        double lc = P.logK[i];
#pragma unroll (NC > 0 ? NC : 1)
        for (int j = 0; j < nc; ++j) lc = fma(P.S[i * CLB_MAX_COMPONENTS + j], x[j], lc);
        c[i] = exp10(fmax(fmin(lc, 300.0), -300.0));
    }
}

constexpr double EQ_MAX_STEP = 2.0;  // largest log10 change of a component in one Newton step

template <int NC, int NS>
__device__ __forceinline__ double eq_residual(const SpecParams& P, const double* x, const double* T,
                                              const double* init, double* c, double* F) {
    const int nc = NC > 0 ? NC : P.nc, ns = NS > 0 ? NS : P.ns;
    eq_species_free<NC, NS>(P, x, init, c);
    double s = 0;
#pragma unroll (NC > 0 ? NC : 1)
    for (int j = 0; j < nc; ++j) {
        double v = -T[j];
#pragma unroll (NS > 0 ? NS : 1)
        for (int i = 0; i < ns; ++i)
            if (P.eq[i]) v = fma(P.S[i * CLB_MAX_COMPONENTS + j], c[i], v);
        F[j] = v;
        s = fma(v, v, s);
    }
    return sqrt(s);
}

template <int NC, int NS>
__device__ __forceinline__ void eq_totals(const SpecParams& P, const double* cin, double* T) {
    const int nc = NC > 0 ? NC : P.nc, ns = NS > 0 ? NS : P.ns;
#pragma unroll (NC > 0 ? NC : 1)
    for (int j = 0; j < nc; ++j) {
        double v = 0;
#pragma unroll (NS > 0 ? NS : 1)
        for (int i = 0; i < ns; ++i)
            if (P.eq[i]) v = fma(P.S[i * CLB_MAX_COMPONENTS + j], fmax(fmin(cin[i], EQ_MAX_C), EQ_MIN_C), v);
        T[j] = fmax(v, EQ_MIN_C);
    }
}

// v[i] for a run-time i < n; in a fixed-shape build a select over every i, so v stays in registers
template <int NS>
__device__ __forceinline__ double eq_pick(const double* v, int i, int n) {
    if constexpr (NS > 0) {
        double r = 0.0;
#pragma unroll
        for (int q = 0; q < NS; ++q)
            if (q == i) r = v[q];
        return r;
    } else {
        return i < n ? v[i] : 0.0;
    }
}

// v[i] = x for a run-time i; in a fixed-shape build a predicated store to every slot
template <int NS>
__device__ __forceinline__ void eq_put(double* v, int i, double x) {
    if constexpr (NS > 0) {
#pragma unroll
        for (int q = 0; q < NS; ++q)
            if (q == i) v[q] = x;
    } else {
        v[i] = x;
    }
}

// x0: optional starting log10 component concentrations (else the reference's guess from the
// component species, 1e-7 for a component that is not a species); max_it < 0: the tableau's cap.
template <int NC, int NS>
__device__ __forceinline__ bool eq_solve_nr(const SpecParams& P, const double* cin, double* cout, int* iters,
                                            const double* x0, int max_it) {
    constexpr int MC = EQ_NC(NC), MS = EQ_NS(NS);
    const int nc = NC > 0 ? NC : P.nc, ns = NS > 0 ? NS : P.ns;
    double T[MC], x[MC], F[MC], xn[MC], d[MC];
    double A[MC][MC + 1];
    double c[MS];
    eq_totals<NC, NS>(P, cin, T);
#pragma unroll (NC > 0 ? NC : 1)
    for (int j = 0; j < nc; ++j) {
        if (x0) {
            x[j] = fmax(fmin(x0[j], EQ_MAX_LOG), EQ_MIN_LOG);
        } else {
            double cc = 1e-7;  // the component's species (selected, not indexed: see eq_pick)
            if (P.comp[j] >= 0) cc = eq_pick<NS>(cin, P.comp[j], ns);
            x[j] = log10(fmax(fmin(cc, EQ_MAX_C), EQ_MIN_C));
        }
    }
    bool conv = false;
    int it = 0;
    const double ln10 = 2.302585092994045684;
    const int cap = max_it < 0 ? P.max_it : max_it;
    for (; it < cap; ++it) {
        const double fn = eq_residual<NC, NS>(P, x, T, cin, c, F);
        if (fn < P.tol) { conv = true; ++it; break; }
#pragma unroll (NC > 0 ? NC : 1)
        for (int j = 0; j < nc; ++j) {
#pragma unroll (NC > 0 ? NC : 1)
            for (int k = 0; k < nc; ++k) {
                double v = 0;
#pragma unroll (NS > 0 ? NS : 1)
                for (int i = 0; i < ns; ++i)
                    if (P.eq[i]) v = fma(ln10 * P.S[i * CLB_MAX_COMPONENTS + j] * P.S[i * CLB_MAX_COMPONENTS + k], c[i], v);
                A[j][k] = v;
            }
            A[j][nc] = -F[j];
        }
        bool ok = true;
#pragma unroll (NC > 0 ? NC : 1)
        for (int p = 0; p < nc; ++p) {
            int r = p;
            double mv = fabs(A[p][p]);
#pragma unroll (NC > 0 ? NC : 1)
            for (int q = p + 1; q < nc; ++q)
                if (fabs(A[q][p]) > mv) { mv = fabs(A[q][p]); r = q; }
            if (mv < 1e-30) { ok = false; break; }
            if (r != p) {
                // row swap by predicated selects, so a fixed-shape build keeps A in registers
#pragma unroll (NC > 0 ? NC : 1)
                for (int q = p + 1; q < nc; ++q) {
                    if (q != r) continue;
#pragma unroll (NC > 0 ? NC + 1 : 1)
                    for (int m = 0; m <= nc; ++m) { const double t = A[p][m]; A[p][m] = A[q][m]; A[q][m] = t; }
                }
            }
#pragma unroll (NC > 0 ? NC : 1)
            for (int q = p + 1; q < nc; ++q) {
                const double fct = A[q][p] / A[p][p];
#pragma unroll (NC > 0 ? NC + 1 : 1)
                for (int m = p; m <= nc; ++m) A[q][m] -= fct * A[p][m];
            }
        }
        if (!ok) { ++it; break; }
#pragma unroll (NC > 0 ? NC : 1)
        for (int p = nc - 1; p >= 0; --p) {
            double v = A[p][nc];
#pragma unroll (NC > 0 ? NC : 1)
            for (int q = p + 1; q < nc; ++q) v -= A[p][q] * d[q];
            d[p] = v / A[p][p];
        }
        double dmax = 0;
#pragma unroll (NC > 0 ? NC : 1)
        for (int j = 0; j < nc; ++j) dmax = fmax(dmax, fabs(d[j]));
        if (dmax > EQ_MAX_STEP) {
#pragma unroll (NC > 0 ? NC : 1)
            for (int j = 0; j < nc; ++j) d[j] *= EQ_MAX_STEP / dmax;
        }
        double alpha = 1.0, fnew = 0;
        for (int ls = 0; ls < 40; ++ls) {
#pragma unroll (NC > 0 ? NC : 1)
            for (int j = 0; j < nc; ++j) xn[j] = fmax(fmin(x[j] + alpha * d[j], EQ_MAX_LOG), EQ_MIN_LOG);
            fnew = eq_residual<NC, NS>(P, xn, T, cin, c, F);
            if (fnew < fn * (1.0 - 0.0001 * alpha) || alpha < 1e-15) break;
            alpha *= 0.5;
        }
        double dn = 0;
#pragma unroll (NC > 0 ? NC : 1)
        for (int j = 0; j < nc; ++j) { x[j] = xn[j]; dn = fma(d[j], d[j], dn); }
        if (alpha * sqrt(dn) < P.tol * 1e-3 && fnew < P.tol * 100) { conv = true; ++it; break; }
    }
    eq_species<NC, NS>(P, x, cin, cout);
#pragma unroll (NS > 0 ? NS : 1)
    for (int i = 0; i < ns; ++i) {
        double v = cout[i];
        if (isnan(v) || isinf(v)) v = cin[i] > EQ_MIN_C ? fmin(cin[i], EQ_MAX_C) : EQ_MIN_C;
        cout[i] = fmax(fmin(v, EQ_MAX_C), EQ_MIN_C);
    }
    if (x0) {
#pragma unroll (NC > 0 ? NC : 1)
        for (int j = 0; j < nc; ++j) const_cast<double*>(x0)[j] = x[j];  // hand back where it stopped
    }
    *iters = it;
    return conv;
}

template <int NC, int NS>
__global__ void k_eq_batch(const SpecParams P, const double* __restrict__ cin, double* __restrict__ cout,
                           int* __restrict__ iters, int n) {
    const int ns = NS > 0 ? NS : P.ns;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        double ci[EQ_NS(NS)], co[EQ_NS(NS)];
#pragma unroll (NS > 0 ? NS : 1)
        for (int i = 0; i < ns; ++i) ci[i] = cin[(int64_t)t * ns + i];
        int it = 0;
        eq_solve_nr<NC, NS>(P, ci, co, &it, nullptr, -1);
#pragma unroll (NS > 0 ? NS : 1)
        for (int i = 0; i < ns; ++i) cout[(int64_t)t * ns + i] = co[i];
        if (iters) iters[t] = it;
    }
}

// the tableau shapes with a build of their own: the 5 x 12 tableau of the fracture configuration
// and the two-component carbonate system; any other shape runs the general build
#define CLB_EQ_SHAPES(P, X)                                      \
    do {                                                         \
        if ((P).nc == 5 && (P).ns == 12) X(5, 12);               \
        else if ((P).nc == 2 && (P).ns == 4) X(2, 4);            \
        else X(0, 0);                                            \
    } while (0)

template <int NC, int NS>
static void launch_eq_batch(const SpecParams& P, const double* cin, double* cout, int* iters, int n, int num_sms,
                            cudaStream_t st) {
    k_eq_batch<NC, NS><<<std::max(1, std::min(num_sms * 8, (n + 127) / 128)), 128, 0, st>>>(P, cin, cout, iters, n);
}

// Where outgoing population i of node k sits after a step of parity `odd` (AA pattern,
// sparse.cuh): even -> own opposite slot, or the even wall slot X; odd -> the destination's slot
// i, or the own opposite slot when the destination is a wall or outside the box.
template <typename TS>
__device__ __forceinline__ TS* out_slot7(const SparseView& S, TS* f, TS* link, int k, int i, int odd) {
    if (i == 0) return f + k;
    const uint32_t mt = S.meta[k];
    const uint32_t wm = mt & 0x7Fu, blk = wm | ((mt >> 7) & 0x7Fu);
    const int oi = q7opp(i);
    if (!odd) {
        if ((wm >> i) & 1u) return link + S.tlb[k >> 8] + (int)(mt >> 14) + __popc(wm & ((1u << i) - 1u));
        return f + (int64_t)oi * S.KS + k;
    }
    if ((blk >> i) & 1u) return f + (int64_t)oi * S.KS + k;
    // destination a + c_i is the source of direction opp(i)
    int dst;
    if (i == 3) dst = k - 1;
    else if (i == 6) dst = k + 1;
    else {
        const int s4 = (i == 1) ? 1 : (i == 4) ? 0 : (i == 2) ? 3 : 2;  // row of a + c_i
        dst = k + S.tdb[(k >> 8) * 4 + s4] + S.dres[(int64_t)k * 4 + s4];
    }
    return f + (int64_t)i * S.KS + dst;
}

// Surrogate evaluation for the warp (tensor-core tiles, all lanes together): each lane brings its
// voxel's species, the surrogate predicts the equilibrium, and `M.polish` FP64 Newton iterations
// start from the surrogate's component values. Accepted (true) when the input lies inside the
// trained range and, when `check`, the polished answer has converged; x0_out returns where the
// polish stopped so a fallback can continue from there.
template <int NC, int NS>
__device__ __forceinline__ bool mlp_warp_speciate(const MlpView& M, const SpecParams& P, bool active,
                                                  const double* c, double* e, bool check, float* ws,
                                                  double* x0_out, int* it_used) {
    const int lane = threadIdx.x & 31;
    double T[EQ_NC(NC)];
    bool in_range = active;
    float* row = ws + lane * 16;
    for (int q = 0; q < 16; ++q) row[q] = 0.f;
    const int nc = NC > 0 ? NC : P.nc, ns = NS > 0 ? NS : P.ns;
    if (active) {
        eq_totals<NC, NS>(P, c, T);
#pragma unroll (NC > 0 ? NC : 1)
        for (int j = 0; j < nc; ++j) {
            const float x = (float)log10(T[j]);
            const float lo = M.in_lo[j], hi = M.in_hi[j];
            const float sx = 2.f * (x - lo) / (hi - lo) - 1.f;
            if (!(fabsf(sx) <= 1.f + M.range_margin)) in_range = false;
            row[j] = sx;
        }
    }
    __syncwarp();
    float y[2][4];
#pragma unroll
    for (int tile = 0; tile < 2; ++tile) {
        uint32_t A[4];
        load_a_tile(ws + tile * 256, lane, A);
        mlp_tile_forward(M, A, lane, y);
        __syncwarp();
        store_d_tile(ws + tile * 256, lane, y);  // overwrite the tile's inputs with its outputs
        __syncwarp();
    }
    if (!active) return false;
    // the surrogate's log10 species; its components' values start a short Newton polish
    double x[EQ_NC(NC)];
#pragma unroll (NS > 0 ? NS : 1)
    for (int i = 0; i < ns; ++i) {
        const float lo = M.out_lo[i], hi = M.out_hi[i];
        e[i] = (double)lo + ((double)row[i] + 1.0) * 0.5 * (double)(hi - lo);
    }
#pragma unroll (NC > 0 ? NC : 1)
    for (int j = 0; j < nc; ++j) x[j] = P.comp[j] >= 0 ? eq_pick<NS>(e, P.comp[j], ns) : -7.0;
    *it_used = 0;
    if (!in_range) {
#pragma unroll (NC > 0 ? NC : 1)
        for (int j = 0; j < nc; ++j) x0_out[j] = x[j];
        return false;
    }
    eq_solve_nr<NC, NS>(P, c, e, it_used, x, M.polish);
#pragma unroll (NC > 0 ? NC : 1)
    for (int j = 0; j < nc; ++j) x0_out[j] = x[j];
    if (!check) return true;
    double worst = 0;
#pragma unroll (NC > 0 ? NC : 1)
    for (int j = 0; j < nc; ++j) {
        double v = -T[j];
#pragma unroll (NS > 0 ? NS : 1)
        for (int i = 0; i < ns; ++i)
            if (P.eq[i]) v = fma(P.S[i * CLB_MAX_COMPONENTS + j], e[i], v);
        worst = fmax(worst, fabs(v) / fmax(T[j], EQ_MIN_C));
    }
    return worst <= (double)M.resid_tol;
}

// The speciation step on the populations the last transport step wrote. Warps walk 32
// consecutive nodes at a time so the surrogate's tensor-core tiles see converged warps.
template <typename TS, int NC, int NS>
__global__ void __launch_bounds__(128) k_speciate_step(TS* __restrict__ g, TS* __restrict__ glink,
                                                       double* __restrict__ imm, const SparseView S, const AdeParams A,
                                                       const SpecParams P, int odd, int64_t k_west_end,
                                                       int64_t k_east_begin, const MlpView M, int mode,
                                                       unsigned long long* __restrict__ stats) {
    __shared__ float wsm[4][32 * 16];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const bool use_mlp = (mode == CLB_SPEC_MLP || mode == CLB_SPEC_MLP_NR);
    unsigned long long n_solve = 0, n_conv = 0, n_sur = 0, n_fb = 0, n_it = 0;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t base = ((int64_t)blockIdx.x * (blockDim.x >> 5) + wib) * 32; base < S.K; base += nwarps * 32) {
        const int64_t k = base + lane;
        const bool active = k < S.K && k >= k_west_end && k < k_east_begin && A.react[S.code[k]];
        double c[EQ_NS(NS)], e[EQ_NS(NS)];
        const int ns = NS > 0 ? NS : P.ns;
        if (active) {
            // species by species (the gathers stay a loop; the values go to c by selects)
#pragma unroll 1
            for (int i = 0; i < ns; ++i) {
                const int si = P.ispec[i];
                double v;
                if (A.slot[si] >= 0) {
                    const int m = A.slot[si];
                    TS* f = g + (int64_t)m * S.SS;
                    TS* lk = glink + (int64_t)m * S.SS;
                    v = ade_sigma<TS>();
                    for (int q = 0; q < 7; ++q) v += ldd(out_slot7(S, f, lk, (int)k, q, odd));
                } else {
                    v = imm[(int64_t)si * A.g.N + S.node[k]];
                }
                eq_put<NS>(c, i, fmax(v, EQ_MIN_C));
            }
        }
        bool done = false;
        double xs[EQ_NC(NC)];
        int pit = 0;
        if (use_mlp) {  // warp-uniform
            done = mlp_warp_speciate<NC, NS>(M, P, active, c, e, mode == CLB_SPEC_MLP_NR, wsm[wib], xs, &pit);
            if (active) { if (done) ++n_sur; else ++n_fb; }
        }
        if (!active) continue;
        ++n_solve;
        n_it += pit;
        if (done) {
            ++n_conv;
        } else {
            // Newton-Raphson fallback, from where the surrogate's polish stopped when there was one
            int it = 0;
            if (eq_solve_nr<NC, NS>(P, c, e, &it, (use_mlp && pit > 0) ? xs : nullptr, -1)) ++n_conv;
            n_it += it;
        }
#pragma unroll 1
        for (int i = 0; i < ns; ++i) {
            const double ci = eq_pick<NS>(c, i, ns);
            double dC = eq_pick<NS>(e, i, ns) - ci;
            const double cap = fmax(1e-9, 0.1 * fabs(ci));
            if (fabs(dC) > cap) dC = dC > 0 ? cap : -cap;
            if (ci + dC < 1e-20) dC = 1e-20 - ci;
            if (!(fabs(dC) > THRD)) continue;
            const int si = P.ispec[i];
            if (A.slot[si] >= 0) {
                const int m = A.slot[si];
                TS* f = g + (int64_t)m * S.SS;
                TS* lk = glink + (int64_t)m * S.SS;
                for (int q = 0; q < 7; ++q) {
                    TS* p = out_slot7(S, f, lk, (int)k, q, odd);
                    const double v = ldd(p) + q7w(q) * dC;
                    if constexpr (std::is_same<TS, __half>::value) *p = to_half(v);
                    else *p = (TS)v;
                }
            } else {
                imm[(int64_t)si * A.g.N + S.node[k]] += dC;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        n_solve += __shfl_down_sync(0xffffffffu, n_solve, o);
        n_conv += __shfl_down_sync(0xffffffffu, n_conv, o);
        n_sur += __shfl_down_sync(0xffffffffu, n_sur, o);
        n_fb += __shfl_down_sync(0xffffffffu, n_fb, o);
        n_it += __shfl_down_sync(0xffffffffu, n_it, o);
    }
    if (lane == 0 && n_solve) {
        atomicAdd(&stats[0], n_solve);
        atomicAdd(&stats[1], n_conv);
        atomicAdd(&stats[2], n_sur);
        atomicAdd(&stats[3], n_fb);
        atomicAdd(&stats[4], n_it);
    }
}

// ------------------------------------------------------------------ host side

clb_status speciation_setup(clb_handle* h, const clb_speciation_desc* d) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (d->n_species < 1 || d->n_species > CLB_MAX_EQ_SPECIES || d->n_species > h->S)
        return fail(h, CLB_INVALID_ARG, "tableau species must be the first species of the handle");
    if (d->n_components < 1 || d->n_components > CLB_MAX_COMPONENTS)
        return fail(h, CLB_INVALID_ARG, "component count out of range");
    if (!(d->tolerance > 0) || d->max_iterations < 1) return fail(h, CLB_INVALID_ARG, "bad solver settings");
    static_assert(sizeof(SpecParams) <= sizeof(((clb_handle*)nullptr)->sp_storage), "SpecParams storage");
    SpecParams& P = CLB_SP(h);
    std::memset(&P, 0, sizeof(P));
    P.ns = d->n_species;
    P.nc = d->n_components;
    P.tol = d->tolerance;
    P.max_it = d->max_iterations;
    for (int i = 0; i < P.ns; ++i) {
        P.logK[i] = d->logK[i];
        bool part = false;
        for (int j = 0; j < P.nc; ++j) {
            P.S[i * CLB_MAX_COMPONENTS + j] = d->stoich[i][j];
            if (std::fabs(d->stoich[i][j]) > 1e-10) part = true;
        }
        P.eq[i] = part ? 1 : 0;
        P.ispec[i] = h->u2i[i];
    }
    for (int j = 0; j < P.nc; ++j) {
        const int cs = d->component_species[j];
        if (cs >= P.ns) return fail(h, CLB_INVALID_ARG, "component species outside the tableau");
        P.comp[j] = cs;
    }
    if (!h->d_spec_stats) {
        cudaError_t e = cudaMalloc(&h->d_spec_stats, sizeof(unsigned long long) * 8);
        if (e != cudaSuccess) return cuda_check(h, e, "speciation counters");
    }
    cudaMemsetAsync(h->d_spec_stats, 0, sizeof(unsigned long long) * 8, h->stream);
    h->spec_ready = true;
    return cuda_check(h, cudaGetLastError(), "speciation setup");
}

template <typename TS, int NC, int NS>
static int launch_speciate(clb_handle* h, int grid, const SparseView& S, const MlpView& M, int odd) {
    k_speciate_step<TS, NC, NS><<<grid, 128, 0, h->stream>>>((TS*)h->d_g, (TS*)h->d_glink, h->d_imm, S, h->ap,
                                                            CLB_SP(h), odd, h->ade_west_end, h->ade_east_begin, M,
                                                            h->spec_mode, h->d_spec_stats);
    return 0;
}

clb_status speciation_step(clb_handle* h) {
    if (!h->spec_ready || h->spec_mode == CLB_SPEC_OFF) return CLB_OK;
    if ((h->spec_mode == CLB_SPEC_MLP || h->spec_mode == CLB_SPEC_MLP_NR) && !h->mlp_ready)
        return fail(h, CLB_NOT_INITIALIZED, "surrogate speciation needs a trained network");
    const int odd = (int)((h->ade_iters - 1) & 1);  // parity of the step just taken
    const SparseView S = view_of(h->ade_sp);
    const int grid = h->num_sms * 4;
    const MlpView M = mlp_view(h);
    ++h->launches;
    switch (h->ade_prec) {
#define CLB_SPEC_F64(NC, NS) launch_speciate<double, NC, NS>(h, grid, S, M, odd)
#define CLB_SPEC_F32(NC, NS) launch_speciate<float, NC, NS>(h, grid, S, M, odd)
#define CLB_SPEC_F16(NC, NS) launch_speciate<__half, NC, NS>(h, grid, S, M, odd)
        case CLB_F64: CLB_EQ_SHAPES(CLB_SP(h), CLB_SPEC_F64); break;
        case CLB_F32: CLB_EQ_SHAPES(CLB_SP(h), CLB_SPEC_F32); break;
        default: CLB_EQ_SHAPES(CLB_SP(h), CLB_SPEC_F16); break;
#undef CLB_SPEC_F64
#undef CLB_SPEC_F32
#undef CLB_SPEC_F16
    }
    return cuda_check(h, cudaGetLastError(), "speciation step");
}

clb_status speciation_solve(clb_handle* h, const double* cin, int n, double* cout, int* iters) {
    if (!h->spec_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_speciation_setup first");
    if (n <= 0) return CLB_OK;
    const size_t bytes = sizeof(double) * (size_t)n * CLB_SP(h).ns;
    double *di = nullptr, *dout = nullptr;
    int* dit = nullptr;
    cudaError_t e = cudaMalloc(&di, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&dout, bytes);
    if (e == cudaSuccess && iters) e = cudaMalloc(&dit, sizeof(int) * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(di, cin, bytes, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
#define CLB_EQB(NC, NS) launch_eq_batch<NC, NS>(CLB_SP(h), di, dout, dit, n, h->num_sms, h->stream)
        CLB_EQ_SHAPES(CLB_SP(h), CLB_EQB);
#undef CLB_EQB
        e = cudaMemcpyAsync(cout, dout, bytes, cudaMemcpyDeviceToHost, h->stream);
    }
    if (e == cudaSuccess && iters) e = cudaMemcpyAsync(iters, dit, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(di);
    cudaFree(dout);
    cudaFree(dit);
    return cuda_check(h, e, "speciation solve");
}

// device-resident batch solve (used by the surrogate's training-data generator)
clb_status speciation_solve_device(clb_handle* h, const double* d_in, int n, double* d_out) {
#define CLB_EQB(NC, NS) launch_eq_batch<NC, NS>(CLB_SP(h), d_in, d_out, nullptr, n, h->num_sms, h->stream)
    CLB_EQ_SHAPES(CLB_SP(h), CLB_EQB);
#undef CLB_EQB
    return cuda_check(h, cudaGetLastError(), "speciation batch");
}

clb_status speciation_stats(clb_handle* h, clb_speciation_stats* out) {
    std::memset(out, 0, sizeof(*out));
    if (!h->d_spec_stats) return CLB_OK;
    unsigned long long v[8];
    cudaError_t e = cudaMemcpyAsync(v, h->d_spec_stats, sizeof(v), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_check(h, e, "speciation counters");
    out->solves = (int64_t)v[0];
    out->converged = (int64_t)v[1];
    out->surrogate_used = (int64_t)v[2];
    out->fallbacks = (int64_t)v[3];
    out->iterations = (int64_t)v[4];
    return CLB_OK;
}


// =====================================================================================
//                    SURROGATE: data from Newton-Raphson solves, training
// =====================================================================================
// Parameter blob layout (FP32 master copy, same layout for the Adam moments and gradients):
//   W1 [64][16], b1 [64], W2 [64][64], b2 [64], W3 [16][64], b3 [16]
constexpr int P_W1 = 0, P_B1 = P_W1 + MLP_H * MLP_IN, P_W2 = P_B1 + MLP_H, P_B2 = P_W2 + MLP_H * MLP_H,
              P_W3 = P_B2 + MLP_H, P_B3 = P_W3 + MLP_OUT * MLP_H, P_N = P_B3 + MLP_OUT;
// BF16 operand copies: W1, W2, W3 as stored (forward), then W2 and W3 transposed (backward)
constexpr int BF_W1 = 0, BF_W2 = BF_W1 + MLP_H * MLP_IN, BF_W3 = BF_W2 + MLP_H * MLP_H,
              BF_W2T = BF_W3 + MLP_OUT * MLP_H, BF_W3T = BF_W2T + MLP_H * MLP_H, BF_N = BF_W3T + MLP_H * MLP_OUT;
// per-block partial gradients of a training launch: P_N values then the block's squared error
constexpr int PART_STRIDE = P_N + 1;

MlpView mlp_view(clb_handle* h) {
    MlpView M;
    std::memset(&M, 0, sizeof(M));
    if (!h->d_mlp) return M;
    const float* pf = h->d_mlp;
    const __nv_bfloat16* pb = static_cast<const __nv_bfloat16*>(h->d_mlp_bf16);
    M.w1b = pb;
    M.w2b = pb + MLP_H * MLP_IN;
    M.w3b = pb + MLP_H * MLP_IN + MLP_H * MLP_H;
    M.w2t = pb + BF_W2T;
    M.w3t = pb + BF_W3T;
    M.b1 = pf + P_B1;
    M.b2 = pf + P_B2;
    M.b3 = pf + P_B3;
    const float* sc = pf + 4 * P_N;  // scaling after params, m, v, grad
    M.in_lo = sc;
    M.in_hi = sc + 16;
    M.out_lo = sc + 32;
    M.out_hi = sc + 48;
    M.nc = CLB_SP(h).nc;
    M.ns = CLB_SP(h).ns;
    M.range_margin = h->mlp_margin;
    M.resid_tol = h->mlp_resid_tol;
    M.polish = h->mlp_polish;
    return M;
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// species states with log10 c uniform in [lo_i, hi_i]
__global__ void k_mlp_sample(int ns, int n, uint64_t seed, const double* __restrict__ lo, const double* __restrict__ hi,
                             double* __restrict__ c) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (int64_t)n * ns; t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % ns);
        const double u = (double)(mix64(seed ^ mix64((uint64_t)t)) >> 11) * (1.0 / 9007199254740992.0);
        c[t] = exp10(lo[i] + (hi[i] - lo[i]) * u);
    }
}

// Training states from the run itself: species of randomly chosen open voxels (x = 1..nx-2),
// each scaled by 10^u, u uniform in [-jitter, jitter].
template <typename TS>
__global__ void k_mlp_sample_field(const TS* __restrict__ g, const TS* __restrict__ glink,
                                   const double* __restrict__ imm, const SparseView S, const AdeParams A,
                                   const SpecParams P, int odd, int64_t k_lo, int64_t k_hi, int n, uint64_t seed,
                                   double jitter, double* __restrict__ c) {
    const Geom G = A.g;
    double init[7];  // an untouched slot: the equilibrium at 1
    for (int i = 0; i < 7; ++i) init[i] = q7w(i) * (1.0 - ade_sigma<TS>());
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        uint64_t hsh = mix64(seed ^ mix64(0x5DEECE66DULL + (uint64_t)t));
        int64_t k = k_lo + (int64_t)(hsh % (uint64_t)(k_hi - k_lo));
        for (int tries = 0; tries < 16 && !A.react[S.code[k]]; ++tries) {
            hsh = mix64(hsh);
            k = k_lo + (int64_t)(hsh % (uint64_t)(k_hi - k_lo));
        }
        const int64_t nd = S.node[k];
        for (int i = 0; i < P.ns; ++i) {
            const int si = P.ispec[i];
            double v;
            if (A.slot[si] >= 0) {
                const int m = A.slot[si];
                double pop[7];
                natural<TS, double, 7>(S, G, g + (int64_t)m * S.SS, glink + (int64_t)m * S.SS, nd, odd, init, pop);
                v = ade_sigma<TS>();
                for (int q = 0; q < 7; ++q) v += pop[q];
            } else {
                v = imm[(int64_t)si * G.N + nd];
            }
            hsh = mix64(hsh + 0x9E3779B97F4A7C15ULL);
            const double u = (double)(hsh >> 11) * (1.0 / 9007199254740992.0);
            c[(int64_t)t * P.ns + i] = fmax(v, 1e-30) * exp10(jitter * (2.0 * u - 1.0));
        }
    }
}

// X = log10 totals of the sampled state, Y = log10 of its equilibrium species. A state with a
// total that is not positive (clamped to 1e-30 by the species model, no meaningful root) is
// marked by a NaN in X[.][0] and dropped from the training set.
__global__ void k_mlp_xy(const SpecParams P, int n, const double* __restrict__ cin, const double* __restrict__ ceq,
                         float* __restrict__ X, float* __restrict__ Y) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        double ci[CLB_MAX_EQ_SPECIES], T[CLB_MAX_COMPONENTS];
        for (int i = 0; i < P.ns; ++i) ci[i] = cin[(int64_t)t * P.ns + i];
        bool valid = true;
        for (int j = 0; j < P.nc; ++j) {
            double raw = 0;
            for (int i = 0; i < P.ns; ++i) if (P.eq[i]) raw += P.S[i * CLB_MAX_COMPONENTS + j] * ci[i];
            if (!(raw > 0)) valid = false;
        }
        eq_totals<0, 0>(P, ci, T);
        for (int q = 0; q < MLP_IN; ++q) X[(int64_t)t * MLP_IN + q] = q < P.nc ? (float)log10(T[q]) : 0.f;
        if (!valid) X[(int64_t)t * MLP_IN] = __int_as_float(0x7fc00000);
        for (int q = 0; q < MLP_OUT; ++q) Y[(int64_t)t * MLP_OUT + q] = q < P.ns ? (float)log10(ceq[(int64_t)t * P.ns + q]) : 0.f;
    }
}

__global__ void k_mlp_scale(int n, int width, int used, float* __restrict__ Z, const float* __restrict__ lo,
                            const float* __restrict__ hi) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (int64_t)n * width; t += (int64_t)gridDim.x * blockDim.x) {
        const int q = (int)(t % width);
        Z[t] = q < used ? 2.f * (Z[t] - lo[q]) / (hi[q] - lo[q]) - 1.f : 0.f;
    }
}

// the BF16 operand copy of FP32 parameter q (a weight), plain and, for W2 and W3, transposed
__device__ __forceinline__ void mlp_bf16_store(__nv_bfloat16* b, int q, float v) {
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    if (q < P_B1) {
        b[BF_W1 + q - P_W1] = h;
    } else if (q >= P_W2 && q < P_B2) {
        const int jj = (q - P_W2) / MLP_H, ii = (q - P_W2) % MLP_H;  // W2[j][i]
        b[BF_W2 + q - P_W2] = h;
        b[BF_W2T + ii * MLP_H + jj] = h;
    } else if (q >= P_W3 && q < P_B3) {
        const int o = (q - P_W3) / MLP_H, jj = (q - P_W3) % MLP_H;   // W3[o][j]
        b[BF_W3 + q - P_W3] = h;
        b[BF_W3T + jj * MLP_OUT + o] = h;
    }
}

__global__ void k_mlp_to_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ b) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P_N; q += gridDim.x * blockDim.x) mlp_bf16_store(b, q, p[q]);
}

// One minibatch chunk of 128 samples per block (4 warps, 32 rows each): forward on the tensor
// cores, mean-squared error on the scaled outputs, backward on the tensor cores too -- every GEMM
// of the backward pass (dH2 = dY W3, dH1 = dZ2 W2 per warp's rows; dW3 = dY^T H2, dW2 = dZ2^T H1,
// dW1 = dZ1^T X over the block's 128 rows) as mma.sync m16n8k16 with BF16 operands and FP32
// accumulation; bias gradients as FP32 column sums. The block writes its gradient and its squared
// error to its own row of `part` (PART_STRIDE floats); the optimiser kernel sums the rows in
// block order, so training is deterministic. rows[] selects the samples (a shuffled index list);
// count = samples in the minibatch.
constexpr int TR_ROWS = 128;

// A fragment (m16 x k16) of the transpose of a row-major [rows][ld] float matrix Z: rows of the
// fragment are Z's columns c0.., its k are Z's rows k0.. (BF16 pairs along k)
__device__ __forceinline__ void load_at(const float* Z, int ld, int k0, int c0, int lane, uint32_t (&A)[4]) {
    const int g = lane >> 2, t = lane & 3;
    const float* p = Z + (k0 + 2 * t) * ld + c0 + g;
    A[0] = pack_bf16(p[0], p[ld]);
    A[1] = pack_bf16(p[8], p[ld + 8]);
    A[2] = pack_bf16(p[8 * ld], p[9 * ld]);
    A[3] = pack_bf16(p[8 * ld + 8], p[9 * ld + 8]);
}

// B fragment (k16 x n8) of a row-major [rows][ld] float matrix Z read as B[k][n] = Z[k0 + k][n0 + n]
__device__ __forceinline__ void load_bz(const float* Z, int ld, int k0, int n0, int lane, uint32_t& b0, uint32_t& b1) {
    const int g = lane >> 2, t = lane & 3;
    const float* p = Z + (k0 + 2 * t) * ld + n0 + g;
    b0 = pack_bf16(p[0], p[ld]);
    b1 = pack_bf16(p[8 * ld], p[9 * ld]);
}

// D fragment of an m16 x n8 tile (rows m0.., cols n0..) into out[row * ld + col]
__device__ __forceinline__ void store_d(float* out, int ld, int m0, int n0, int lane, const float (&d)[4]) {
    const int g = lane >> 2, t = lane & 3;
    out[(m0 + g) * ld + n0 + 2 * t] = d[0];
    out[(m0 + g) * ld + n0 + 2 * t + 1] = d[1];
    out[(m0 + g + 8) * ld + n0 + 2 * t] = d[2];
    out[(m0 + g + 8) * ld + n0 + 2 * t + 1] = d[3];
}

__global__ void __launch_bounds__(128) k_mlp_train(const MlpView M, const float* __restrict__ X,
                                                   const float* __restrict__ Y, const int* __restrict__ rows,
                                                   int count, float inv_norm, float* __restrict__ part) {
    extern __shared__ float tsm[];
    float* xs = tsm;                          // [128][16]
    float* h1 = xs + TR_ROWS * 16;            // [128][64]
    float* h2 = h1 + TR_ROWS * 64;            // [128][64]
    float* dy = h2 + TR_ROWS * 64;            // [128][16]
    float* d2 = dy + TR_ROWS * 16;            // [128][64]  dL/d(pre-activation of layer 2)
    float* d1 = d2 + TR_ROWS * 64;            // [128][64]  dL/d(pre-activation of layer 1)
    __shared__ float wsum[4];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int r0 = blockIdx.x * TR_ROWS;
    for (int q = tid; q < TR_ROWS * 16; q += blockDim.x) {
        const int r = q >> 4;
        xs[q] = (r0 + r < count) ? X[(int64_t)rows[r0 + r] * MLP_IN + (q & 15)] : 0.f;
    }
    __syncthreads();
    float lsum = 0.f;
    const int g = lane >> 2, t = lane & 3;
    for (int tile = 0; tile < 2; ++tile) {
        const int tr = w * 32 + tile * 16;  // first row of the tile within the block
        uint32_t A[4];
        load_a_tile(xs + tr * 16, lane, A);
        float y[2][4], a1[8][4], a2[8][4];
        mlp_tile_forward(M, A, lane, y, a1, a2);
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            store_d(h1, 64, tr, nt * 8, lane, a1[nt]);
            store_d(h2, 64, tr, nt * 8, lane, a2[nt]);
        }
        float dyv[2][4];
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int row = tr + g + ((q & 2) ? 8 : 0), col = nt * 8 + 2 * t + (q & 1);
                const bool live = (r0 + row < count) && col < M.ns;
                const float target = live ? Y[(int64_t)rows[r0 + row] * MLP_OUT + col] : 0.f;
                const float diff = live ? (y[nt][q] - target) : 0.f;
                lsum += diff * diff;
                dyv[nt][q] = 2.f * diff * inv_norm;
            }
        store_d(dy, 16, tr, 0, lane, dyv[0]);
        store_d(dy, 16, tr, 8, lane, dyv[1]);
        __syncwarp();
        // dH2 = dY (16 x 16) W3 (16 x 64); dZ2 = dH2 (1 - h2^2), kept as the next GEMM's A
        load_a_tile(dy + tr * 16, lane, A);
        uint32_t A2[4][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float d[4] = {0.f, 0.f, 0.f, 0.f};
            uint32_t b0, b1;
            load_b(M.w3t, MLP_OUT, nt, 0, lane, b0, b1);
            mma_bf16(d, A, b0, b1);
#pragma unroll
            for (int q = 0; q < 4; ++q) d[q] *= 1.f - a2[nt][q] * a2[nt][q];
            store_d(d2, 64, tr, nt * 8, lane, d);
            const int kt = nt >> 1, hi = nt & 1;
            A2[kt][0 + 2 * hi] = pack_bf16(d[0], d[1]);
            A2[kt][1 + 2 * hi] = pack_bf16(d[2], d[3]);
        }
        // dH1 = dZ2 (16 x 64) W2 (64 x 64); dZ1 = dH1 (1 - h1^2)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) {
                uint32_t b0, b1;
                load_b(M.w2t, MLP_H, nt, kt, lane, b0, b1);
                mma_bf16(d, A2[kt], b0, b1);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) d[q] *= 1.f - a1[nt][q] * a1[nt][q];
            store_d(d1, 64, tr, nt * 8, lane, d);
        }
    }
    __syncthreads();
    float* out = part + (int64_t)blockIdx.x * PART_STRIDE;
    // weight gradients over the block's 128 rows (K = 128: 8 k-steps). Warp w: rows w*16.. of
    // dW2 (64 x 64) and dW1 (64 x 16), columns w*16.. of dW3 (16 x 64).
    {
        float acc[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
        for (int kt = 0; kt < TR_ROWS / 16; ++kt) {
            uint32_t A[4];
            load_at(d2, 64, kt * 16, w * 16, lane, A);
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                uint32_t b0, b1;
                load_bz(h1, 64, kt * 16, nt * 8, lane, b0, b1);
                mma_bf16(acc[nt], A, b0, b1);
            }
        }
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) store_d(out + P_W2, 64, w * 16, nt * 8, lane, acc[nt]);
    }
    {
        float acc[2][4];
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
        for (int kt = 0; kt < TR_ROWS / 16; ++kt) {
            uint32_t A[4];
            load_at(d1, 64, kt * 16, w * 16, lane, A);
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                uint32_t b0, b1;
                load_bz(xs, 16, kt * 16, nt * 8, lane, b0, b1);
                mma_bf16(acc[nt], A, b0, b1);
            }
        }
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) store_d(out + P_W1, 16, w * 16, nt * 8, lane, acc[nt]);
    }
    {
        float acc[2][4];
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
        for (int kt = 0; kt < TR_ROWS / 16; ++kt) {
            uint32_t A[4];
            load_at(dy, 16, kt * 16, 0, lane, A);
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                uint32_t b0, b1;
                load_bz(h2, 64, kt * 16, w * 16 + nt * 8, lane, b0, b1);
                mma_bf16(acc[nt], A, b0, b1);
            }
        }
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) store_d(out + P_W3, 64, 0, w * 16 + nt * 8, lane, acc[nt]);
    }
    // bias gradients: column sums in row order
    for (int c = tid; c < 2 * MLP_H + MLP_OUT; c += blockDim.x) {
        float sum = 0.f;
        if (c < MLP_H) {
            for (int r = 0; r < TR_ROWS; ++r) sum += d1[r * 64 + c];
            out[P_B1 + c] = sum;
        } else if (c < 2 * MLP_H) {
            for (int r = 0; r < TR_ROWS; ++r) sum += d2[r * 64 + c - MLP_H];
            out[P_B2 + c - MLP_H] = sum;
        } else {
            for (int r = 0; r < TR_ROWS; ++r) sum += dy[r * 16 + c - 2 * MLP_H];
            out[P_B3 + c - 2 * MLP_H] = sum;
        }
    }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
    if (lane == 0) wsum[w] = lsum;
    __syncthreads();
    if (tid == 0) out[P_N] = (wsum[0] + wsum[1]) + (wsum[2] + wsum[3]);
}

// Adam on the block-order sum of the partial gradients, with the BF16 operand copies refreshed;
// one thread adds the launch's squared errors to loss_acc[0] in block order.
__global__ void k_mlp_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ part, int nb, float lr, float b1, float b2, float eps, float c1,
                           float c2, __nv_bfloat16* __restrict__ bf, float* __restrict__ loss_acc) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q <= P_N; q += gridDim.x * blockDim.x) {
        float gq = 0.f;
        for (int b = 0; b < nb; ++b) gq += part[(int64_t)b * PART_STRIDE + q];
        if (q == P_N) {
            loss_acc[0] += gq;
            continue;
        }
        const float mq = b1 * m[q] + (1.f - b1) * gq;
        const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
        m[q] = mq;
        v[q] = vq;
        const float pq = p[q] - lr * (mq / c1) / (sqrtf(vq / c2) + eps);
        p[q] = pq;
        mlp_bf16_store(bf, q, pq);
    }
}

// the block-order sum of the partial gradients (the gradient check's view)
__global__ void k_mlp_grad_sum(const float* __restrict__ part, int nb, float* __restrict__ grad) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q <= P_N; q += gridDim.x * blockDim.x) {
        float gq = 0.f;
        for (int b = 0; b < nb; ++b) gq += part[(int64_t)b * PART_STRIDE + q];
        grad[q] = gq;
    }
}

// forward only: squared error on scaled outputs, summed
__global__ void __launch_bounds__(128) k_mlp_eval(const MlpView M, const float* __restrict__ X,
                                                  const float* __restrict__ Y, int first, int count,
                                                  float* __restrict__ block_loss) {
    __shared__ float xs[4][32 * 16];
    __shared__ float wsum[4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    float lsum = 0.f;
    for (int base = (blockIdx.x * 4 + w) * 32; base < count; base += gridDim.x * 128) {
        for (int q = lane; q < 32 * 16; q += 32) {
            const int r = q >> 4;
            xs[w][q] = (base + r < count) ? X[(int64_t)(first + base + r) * MLP_IN + (q & 15)] : 0.f;
        }
        __syncwarp();
        for (int tile = 0; tile < 2; ++tile) {
            uint32_t A[4];
            load_a_tile(xs[w] + tile * 256, lane, A);
            float y[2][4];
            mlp_tile_forward(M, A, lane, y);
            for (int nt = 0; nt < 2; ++nt)
                for (int q = 0; q < 4; ++q) {
                    const int row = base + tile * 16 + g + ((q & 2) ? 8 : 0), col = nt * 8 + 2 * t + (q & 1);
                    if (row < count && col < M.ns) {
                        const float d = y[nt][q] - Y[(int64_t)(first + row) * MLP_OUT + col];
                        lsum += d * d;
                    }
                }
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
    if (lane == 0) wsum[w] = lsum;
    __syncthreads();
    if (threadIdx.x == 0) block_loss[blockIdx.x] = (wsum[0] + wsum[1]) + (wsum[2] + wsum[3]);
}

// surrogate prediction of species for raw concentration inputs (the speciation step's view)
__global__ void __launch_bounds__(128) k_mlp_predict(const MlpView M, const SpecParams P, const double* __restrict__ cin,
                                                     int n, double* __restrict__ cout, int* __restrict__ accepted,
                                                     int check) {
    __shared__ float wsm[4][32 * 16];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = (blockIdx.x * 4 + w) * 32; base < n; base += gridDim.x * 128) {
        const int tix = base + lane;
        const bool active = tix < n;
        double c[CLB_MAX_EQ_SPECIES], e[CLB_MAX_EQ_SPECIES];
        if (active)
            for (int i = 0; i < P.ns; ++i) c[i] = fmax(cin[(int64_t)tix * P.ns + i], EQ_MIN_C);
        double xs[CLB_MAX_COMPONENTS];
        int pit = 0;
        const bool ok = mlp_warp_speciate<0, 0>(M, P, active, c, e, check != 0, wsm[w], xs, &pit);
        if (active) {
            for (int i = 0; i < P.ns; ++i) cout[(int64_t)tix * P.ns + i] = e[i];
            if (accepted) accepted[tix] = ok ? 1 : 0;
        }
    }
}

// ------------------------------------------------------------------ host side (surrogate)

static clb_status mlp_alloc(clb_handle* h) {
    if (h->d_mlp) return CLB_OK;
    cudaError_t e = cudaMalloc(&h->d_mlp, sizeof(float) * (4 * P_N + 64));
    if (e == cudaSuccess) e = cudaMalloc(&h->d_mlp_bf16, sizeof(__nv_bfloat16) * BF_N);
    if (e != cudaSuccess) return cuda_check(h, e, "surrogate parameters");
    cudaMemsetAsync(h->d_mlp, 0, sizeof(float) * (4 * P_N + 64), h->stream);
    return CLB_OK;
}

static void mlp_refresh_bf16(clb_handle* h) {
    k_mlp_to_bf16<<<(P_N + 255) / 256, 256, 0, h->stream>>>(h->d_mlp, static_cast<__nv_bfloat16*>(h->d_mlp_bf16));
}

// Glorot-uniform initial weights from a seeded xorshift64* stream, zero biases
static void mlp_init_params(clb_handle* h, uint64_t seed, std::vector<float>& p) {
    p.assign(P_N, 0.f);
    uint64_t s = seed ? seed : 1;
    auto uni = [&]() {
        s ^= s >> 12; s ^= s << 25; s ^= s >> 27;
        return (double)((s * 2685821657736338717ULL) >> 11) / 9007199254740992.0;
    };
    auto fill = [&](int off, int rows, int cols, int used_rows, int used_cols) {
        const double a = std::sqrt(6.0 / (double)(used_rows + used_cols));
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c)
                p[off + r * cols + c] = (r < used_rows && c < used_cols) ? (float)(a * (2.0 * uni() - 1.0)) : 0.f;
    };
    fill(P_W1, MLP_H, MLP_IN, MLP_H, CLB_SP(h).nc);
    fill(P_W2, MLP_H, MLP_H, MLP_H, MLP_H);
    fill(P_W3, MLP_OUT, MLP_H, CLB_SP(h).ns, MLP_H);
}

clb_status surrogate_train(clb_handle* h, const clb_surrogate_train_desc* d, clb_surrogate_report* rep) {
    if (!h->spec_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_speciation_setup first");
    const int ns = CLB_SP(h).ns, nc = CLB_SP(h).nc, n = d->n_samples;
    if (n < 256 || d->epochs < 1 || d->batch < TR_ROWS) return fail(h, CLB_INVALID_ARG, "bad training settings");
    clb_status st = mlp_alloc(h);
    if (st != CLB_OK) return st;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, h->stream);
    // ---- data: sampled species states, their equilibria by Newton-Raphson on the GPU
    double *dlo = nullptr, *dhi = nullptr, *cin = nullptr, *ceq = nullptr;
    float *X = nullptr, *Y = nullptr, *loss = nullptr, *rng = nullptr;
    int* rows = nullptr;
    cudaError_t e = cudaMalloc(&dlo, sizeof(double) * ns);
    if (e == cudaSuccess) e = cudaMalloc(&dhi, sizeof(double) * ns);
    if (e == cudaSuccess) e = cudaMalloc(&cin, sizeof(double) * (size_t)n * ns);
    if (e == cudaSuccess) e = cudaMalloc(&ceq, sizeof(double) * (size_t)n * ns);
    if (e == cudaSuccess) e = cudaMalloc(&X, sizeof(float) * (size_t)n * MLP_IN);
    if (e == cudaSuccess) e = cudaMalloc(&Y, sizeof(float) * (size_t)n * MLP_OUT);
    if (e == cudaSuccess) e = cudaMalloc(&loss, sizeof(float) * 4);
    const int part_blocks = (d->batch + TR_ROWS - 1) / TR_ROWS, eval_blocks = h->num_sms * 2;
    float *part = nullptr, *eval_part = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&part, sizeof(float) * (size_t)part_blocks * PART_STRIDE);
    if (e == cudaSuccess) e = cudaMalloc(&eval_part, sizeof(float) * eval_blocks);
    if (e == cudaSuccess) e = cudaMalloc(&rows, sizeof(int) * (size_t)n);
    auto cleanup = [&]() {
        cudaFree(dlo); cudaFree(dhi); cudaFree(cin); cudaFree(ceq); cudaFree(X); cudaFree(Y);
        cudaFree(loss); cudaFree(rows); cudaFree(rng); cudaFree(part); cudaFree(eval_part);
        cudaEventDestroy(t0); cudaEventDestroy(t1);
    };
    if (e != cudaSuccess) { cleanup(); return cuda_check(h, e, "training buffers"); }
    cudaMemcpyAsync(dlo, d->log_c_lo, sizeof(double) * ns, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(dhi, d->log_c_hi, sizeof(double) * ns, cudaMemcpyHostToDevice, h->stream);
    if (d->source == 1) {
        if (h->ade_east_begin <= h->ade_west_end) { cleanup(); return fail(h, CLB_INVALID_ARG, "no interior voxels"); }
        const SparseView Sv = view_of(h->ade_sp);
        const int odd = (int)(h->ade_iters & 1);
        const int gs = h->num_sms * 8;
        switch (h->ade_prec) {
            case CLB_F64: k_mlp_sample_field<double><<<gs, 128, 0, h->stream>>>((const double*)h->d_g, (const double*)h->d_glink, h->d_imm, Sv, h->ap, CLB_SP(h), odd, h->ade_west_end, h->ade_east_begin, n, d->seed, d->jitter, cin); break;
            case CLB_F32: k_mlp_sample_field<float><<<gs, 128, 0, h->stream>>>((const float*)h->d_g, (const float*)h->d_glink, h->d_imm, Sv, h->ap, CLB_SP(h), odd, h->ade_west_end, h->ade_east_begin, n, d->seed, d->jitter, cin); break;
            default: k_mlp_sample_field<__half><<<gs, 128, 0, h->stream>>>((const __half*)h->d_g, (const __half*)h->d_glink, h->d_imm, Sv, h->ap, CLB_SP(h), odd, h->ade_west_end, h->ade_east_begin, n, d->seed, d->jitter, cin); break;
        }
    } else {
        k_mlp_sample<<<h->num_sms * 8, 256, 0, h->stream>>>(ns, n, d->seed, dlo, dhi, cin);
    }
    speciation_solve_device(h, cin, n, ceq);
    k_mlp_xy<<<h->num_sms * 8, 128, 0, h->stream>>>(CLB_SP(h), n, cin, ceq, X, Y);
    // ---- mapminmax ranges over the data
    std::vector<float> hx((size_t)n * MLP_IN), hy((size_t)n * MLP_OUT);
    cudaMemcpyAsync(hx.data(), X, sizeof(float) * hx.size(), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(hy.data(), Y, sizeof(float) * hy.size(), cudaMemcpyDeviceToHost, h->stream);
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { cleanup(); return cuda_check(h, e, "training data"); }
    // drop states without a meaningful root, then upload the compacted set
    int nv = 0;
    for (int r = 0; r < n; ++r) {
        if (std::isnan(hx[(size_t)r * MLP_IN])) continue;
        if (nv != r) {
            std::copy(&hx[(size_t)r * MLP_IN], &hx[(size_t)r * MLP_IN] + MLP_IN, &hx[(size_t)nv * MLP_IN]);
            std::copy(&hy[(size_t)r * MLP_OUT], &hy[(size_t)r * MLP_OUT] + MLP_OUT, &hy[(size_t)nv * MLP_OUT]);
        }
        ++nv;
    }
    if (nv < 2 * TR_ROWS) { cleanup(); return fail(h, CLB_INVALID_ARG, "too few sampled states have positive totals"); }
    const int n_all = n;
    (void)n_all;
    cudaMemcpyAsync(X, hx.data(), sizeof(float) * (size_t)nv * MLP_IN, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(Y, hy.data(), sizeof(float) * (size_t)nv * MLP_OUT, cudaMemcpyHostToDevice, h->stream);
    const int nkeep = nv;
    float sc[64];
    for (int q = 0; q < 16; ++q) { sc[q] = 1e30f; sc[16 + q] = -1e30f; sc[32 + q] = 1e30f; sc[48 + q] = -1e30f; }
    for (int r = 0; r < nkeep; ++r) {
        for (int q = 0; q < nc; ++q) { const float v = hx[(size_t)r * MLP_IN + q]; sc[q] = std::min(sc[q], v); sc[16 + q] = std::max(sc[16 + q], v); }
        for (int q = 0; q < ns; ++q) { const float v = hy[(size_t)r * MLP_OUT + q]; sc[32 + q] = std::min(sc[32 + q], v); sc[48 + q] = std::max(sc[48 + q], v); }
    }
    for (int q = 0; q < 16; ++q) {
        if (q >= nc || !(sc[16 + q] > sc[q])) { sc[q] = -1.f; sc[16 + q] = 1.f; }
        if (q >= ns || !(sc[48 + q] > sc[32 + q])) { sc[32 + q] = sc[32 + q] < 1e29f ? sc[32 + q] - 1.f : -1.f; sc[48 + q] = sc[32 + q] + 2.f; }
    }
    float* dsc = h->d_mlp + 4 * P_N;
    cudaMemcpyAsync(dsc, sc, sizeof(sc), cudaMemcpyHostToDevice, h->stream);
    k_mlp_scale<<<h->num_sms * 8, 256, 0, h->stream>>>(nkeep, MLP_IN, nc, X, dsc, dsc + 16);
    k_mlp_scale<<<h->num_sms * 8, 256, 0, h->stream>>>(nkeep, MLP_OUT, ns, Y, dsc + 32, dsc + 48);
    // ---- parameters
    std::vector<float> p0;
    mlp_init_params(h, d->seed ^ 0x5eedULL, p0);
    float* P = h->d_mlp;
    float* Mm = P + P_N;
    float* V = P + 2 * P_N;
    cudaMemcpyAsync(P, p0.data(), sizeof(float) * P_N, cudaMemcpyHostToDevice, h->stream);
    cudaMemsetAsync(Mm, 0, sizeof(float) * 3 * P_N, h->stream);
    mlp_refresh_bf16(h);
    h->mlp_ready = true;
    // ---- training: shuffled minibatches, Adam, early stop on the held-out part
    const int n_val = std::max(TR_ROWS, (int)(d->val_fraction * nkeep));
    const int n_tr = nkeep - n_val;
    const size_t smem = sizeof(float) * TR_ROWS * (16 + 64 + 64 + 16 + 64 + 64);
    cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    std::vector<int> perm(n_tr);
    for (int q = 0; q < n_tr; ++q) perm[q] = q;
    uint64_t rs = d->seed ? d->seed : 7;
    auto rnd = [&]() { rs ^= rs >> 12; rs ^= rs << 25; rs ^= rs >> 27; return rs * 2685821657736338717ULL; };
    std::vector<float> best((size_t)P_N);
    float best_val = 1e30f, last_train = 0.f;
    int since = 0, epoch = 0, step = 0;
    const float b1 = 0.9f, b2 = 0.999f;
    for (epoch = 0; epoch < d->epochs; ++epoch) {
        for (int q = n_tr - 1; q > 0; --q) std::swap(perm[q], perm[(int)(rnd() % (uint64_t)(q + 1))]);
        cudaMemcpyAsync(rows, perm.data(), sizeof(int) * n_tr, cudaMemcpyHostToDevice, h->stream);
        cudaMemsetAsync(loss, 0, sizeof(float) * 4, h->stream);
        for (int s0 = 0; s0 < n_tr; s0 += d->batch) {
            const int cnt = std::min(d->batch, n_tr - s0);
            const MlpView Mv = mlp_view(h);
            const int nb = (cnt + TR_ROWS - 1) / TR_ROWS;
            k_mlp_train<<<nb, 128, smem, h->stream>>>(Mv, X, Y, rows + s0, cnt, 1.f / (float)(cnt * ns), part);
            ++step;
            const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
            // learning rate decays by 5 % per epoch
            const float lr = (float)d->learning_rate * std::pow(0.95f, (float)epoch);
            k_mlp_adam<<<(P_N + 256) / 256, 256, 0, h->stream>>>(P, Mm, V, part, nb, lr, b1, b2, 1e-8f, c1, c2,
                                                                   static_cast<__nv_bfloat16*>(h->d_mlp_bf16), loss);
        }
        k_mlp_eval<<<eval_blocks, 128, 0, h->stream>>>(mlp_view(h), X, Y, n_tr, n_val, eval_part);
        float l[4];
        std::vector<float> ev((size_t)eval_blocks);
        cudaMemcpyAsync(l, loss, sizeof(l), cudaMemcpyDeviceToHost, h->stream);
        cudaMemcpyAsync(ev.data(), eval_part, sizeof(float) * eval_blocks, cudaMemcpyDeviceToHost, h->stream);
        e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) { cleanup(); return cuda_check(h, e, "training"); }
        double vsum = 0;
        for (float x : ev) vsum += x;  // block order: deterministic
        last_train = l[0] / (float)((size_t)n_tr * ns);
        const float val = (float)(vsum / (double)((size_t)n_val * ns));
        if (val < best_val) {
            best_val = val;
            since = 0;
            cudaMemcpy(best.data(), P, sizeof(float) * P_N, cudaMemcpyDeviceToHost);
        } else if (++since >= d->patience) {
            ++epoch;
            break;
        }
    }
    cudaMemcpyAsync(P, best.data(), sizeof(float) * P_N, cudaMemcpyHostToDevice, h->stream);
    mlp_refresh_bf16(h);
    cudaEventRecord(t1, h->stream);
    e = cudaStreamSynchronize(h->stream);
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    if (rep) {
        rep->train_mse = last_train;
        rep->val_mse = best_val;
        rep->epochs = epoch;
        rep->steps = step;
        rep->seconds = ms * 1e-3;
        rep->n_train = n_tr;
        rep->n_val = n_val;
    }
    cleanup();
    return cuda_check(h, e, "training");
}

clb_status surrogate_predict(clb_handle* h, const double* cin, int n, double* cout, int* accepted, int check) {
    if (!h->mlp_ready) return fail(h, CLB_NOT_INITIALIZED, "no trained surrogate");
    if (n <= 0) return CLB_OK;
    const size_t bytes = sizeof(double) * (size_t)n * CLB_SP(h).ns;
    double *di = nullptr, *dout = nullptr;
    int* da = nullptr;
    cudaError_t e = cudaMalloc(&di, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&dout, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&da, sizeof(int) * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(di, cin, bytes, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        k_mlp_predict<<<std::max(1, std::min(h->num_sms * 4, (n + 127) / 128)), 128, 0, h->stream>>>(mlp_view(h), CLB_SP(h), di, n, dout, da, check);
        e = cudaMemcpyAsync(cout, dout, bytes, cudaMemcpyDeviceToHost, h->stream);
    }
    if (e == cudaSuccess && accepted) e = cudaMemcpyAsync(accepted, da, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(di);
    cudaFree(dout);
    cudaFree(da);
    return cuda_check(h, e, "surrogate predict");
}

// Loss and gradient of the current network on given scaled samples (for the gradient check).
clb_status surrogate_gradient(clb_handle* h, const float* X, const float* Y, int n, float* grad, float* loss) {
    if (!h->mlp_ready) return fail(h, CLB_NOT_INITIALIZED, "no surrogate parameters");
    if (n < 1) return fail(h, CLB_INVALID_ARG, "no samples");
    const int nb = (n + TR_ROWS - 1) / TR_ROWS;
    float *dx = nullptr, *dy = nullptr, *dp = nullptr, *dg = nullptr;
    int* dr = nullptr;
    cudaError_t e = cudaMalloc(&dx, sizeof(float) * (size_t)n * MLP_IN);
    if (e == cudaSuccess) e = cudaMalloc(&dy, sizeof(float) * (size_t)n * MLP_OUT);
    if (e == cudaSuccess) e = cudaMalloc(&dp, sizeof(float) * (size_t)nb * PART_STRIDE);
    if (e == cudaSuccess) e = cudaMalloc(&dg, sizeof(float) * PART_STRIDE);
    if (e == cudaSuccess) e = cudaMalloc(&dr, sizeof(int) * n);
    std::vector<int> r(n);
    for (int q = 0; q < n; ++q) r[q] = q;
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, X, sizeof(float) * (size_t)n * MLP_IN, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dy, Y, sizeof(float) * (size_t)n * MLP_OUT, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dr, r.data(), sizeof(int) * n, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        const size_t smem = sizeof(float) * TR_ROWS * (16 + 64 + 64 + 16 + 64 + 64);
        cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_mlp_train<<<nb, 128, smem, h->stream>>>(mlp_view(h), dx, dy, dr, n, 1.f / (float)(n * CLB_SP(h).ns), dp);
        k_mlp_grad_sum<<<(P_N + 256) / 256, 256, 0, h->stream>>>(dp, nb, dg);
        e = cudaMemcpyAsync(grad, dg, sizeof(float) * P_N, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(loss, dg + P_N, sizeof(float), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
    cudaFree(dx); cudaFree(dy); cudaFree(dp); cudaFree(dg); cudaFree(dr);
    return cuda_check(h, e, "surrogate gradient");
}

clb_status surrogate_params(clb_handle* h, float* out, const float* in, float* scaling_out, const float* scaling_in) {
    clb_status st = mlp_alloc(h);
    if (st != CLB_OK) return st;
    cudaError_t e = cudaSuccess;
    if (in) e = cudaMemcpyAsync(h->d_mlp, in, sizeof(float) * P_N, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && scaling_in)
        e = cudaMemcpyAsync(h->d_mlp + 4 * P_N, scaling_in, sizeof(float) * 64, cudaMemcpyHostToDevice, h->stream);
    if (in || scaling_in) { mlp_refresh_bf16(h); h->mlp_ready = true; }
    if (e == cudaSuccess && out) e = cudaMemcpyAsync(out, h->d_mlp, sizeof(float) * P_N, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess && scaling_out)
        e = cudaMemcpyAsync(scaling_out, h->d_mlp + 4 * P_N, sizeof(float) * 64, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return cuda_check(h, e, "surrogate parameters");
}

int surrogate_param_count() { return P_N; }

}  // namespace clb
