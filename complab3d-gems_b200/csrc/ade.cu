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
// Layout: mobile species populations g[m][7][N] of the storage type (m = rank of the species
// among the mobile ones), AA in-place pattern as in flow.cu; immobile species and biomass
// are FP64 scalar fields; the advection velocity u[3][N] in the arithmetic type.
// Algorithmic bytes per node update: 2*7*sizeof(storage) per mobile species, plus the
// velocity (3*sizeof(arith)) and the material byte shared by all species.
#include "clb_internal.cuh"

#include <algorithm>
#include <cstring>

namespace clb {

constexpr int ADE_THREADS = 256;

template <typename TS, typename TC, bool ODD>
__device__ __forceinline__ void load7(const TS* __restrict__ f, int64_t N, const Geom& G, int64_t n, int x, int y,
                                      int z, TC (&g)[7]) {
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        if (!ODD || i == 0) {
            g[i] = ld<TS, TC>(f + (int64_t)i * N + n);
        } else {
            const int cx = q7cx(i), cy = q7cy(i), cz = q7cz(i);
            const bool in = (cx == 0 || ((unsigned)(x - cx) < (unsigned)G.nx)) &&
                            (cy == 0 || ((unsigned)(y - cy) < (unsigned)G.ny)) &&
                            (cz == 0 || ((unsigned)(z - cz) < (unsigned)G.nz));
            const int64_t off = (int64_t)cx * G.plane + cy * G.nz + cz;
            g[i] = in ? ld<TS, TC>(f + (int64_t)q7opp(i) * N + n - off) : ld<TS, TC>(f + (int64_t)i * N + n);
        }
    }
}

template <typename TS, typename TC, bool ODD>
__device__ __forceinline__ void store7(TS* __restrict__ f, int64_t N, const Geom& G, int64_t n, int x, int y, int z,
                                       const TC (&o)[7]) {
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        if (!ODD || i == 0) {
            st<TS, TC>(f + (int64_t)q7opp(i) * N + n, o[i]);
        } else {
            const int cx = q7cx(i), cy = q7cy(i), cz = q7cz(i);
            const bool in = (cx == 0 || ((unsigned)(x + cx) < (unsigned)G.nx)) &&
                            (cy == 0 || ((unsigned)(y + cy) < (unsigned)G.ny)) &&
                            (cz == 0 || ((unsigned)(z + cz) < (unsigned)G.nz));
            const int64_t off = (int64_t)cx * G.plane + cy * G.nz + cz;
            if (in) st<TS, TC>(f + (int64_t)i * N + n + off, o[i]);
            else st<TS, TC>(f + (int64_t)q7opp(i) * N + n, o[i]);
        }
    }
}

// Rate laws (clb_law). C, B are the floored concentrations / biomasses.
__device__ __forceinline__ void eval_rates(const AdeParams& P, const double* C, const double* B, double* R,
                                           double* RB) {
    for (int s = 0; s < P.S; ++s) R[s] = 0.0;
    for (int m = 0; m < P.M; ++m) RB[m] = 0.0;
    switch (P.law) {
        case CLB_LAW_DECAY:
            for (int s = 0; s < P.S; ++s) R[s] = -P.prm[s] * C[s];
            break;
        case CLB_LAW_MONOD:
            for (int s = 0; s < P.S; ++s) R[s] = -P.prm[s] * C[s] / (P.prm[P.S + s] + C[s]);
            break;
        case CLB_LAW_DUAL_MONOD: {
            const double mu = P.prm[0], ks = P.prm[1], Y = P.prm[2], kd = P.prm[3];
            for (int m = 0; m < P.M; ++m) {
                const int a = 1 + m;
                if (a >= P.S) break;
                const double Bm = B[m];
                if (Bm <= 0.0) continue;
                const double growth = mu * (C[0] / (ks + C[0])) * (C[a] / (ks + C[a])) * Bm;
                RB[m] += growth - kd * Bm;
                R[0] -= growth / Y;
                R[a] -= growth / Y;
            }
            break;
        }
        default:
            break;
    }
}

template <typename TS, typename TC, bool ODD, int NM>
__global__ void __launch_bounds__(ADE_THREADS)
    k_ade_aa(TS* __restrict__ g, double* __restrict__ imm, double* __restrict__ bio, const TC* __restrict__ u,
             const int32_t* __restrict__ list, int64_t nlist, const int8_t* __restrict__ mat,
             const double* __restrict__ neu, const AdeParams P, int n_mobile, const int* __restrict__ mob_species) {
    const Geom G = P.g;
    const int64_t N = G.N;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nlist; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = list[k];
        int x, y, z;
        decode(G, n, x, y, z);
        const int code = mat[n];
        const int dyn = P.dyn[code];
        const bool west = (x == 0), east = (x == G.nx - 1);
        TC pop[NM][7];
        TC rb[NM];
        bool act[NM];
#pragma unroll
        for (int m = 0; m < NM; ++m) {
            act[m] = false;
            rb[m] = 0;
            if (m >= n_mobile) continue;
            const int s = mob_species[m];
            if ((west && P.ltype[s] == CLB_CLOSED) || (east && P.rtype[s] == CLB_CLOSED)) continue;  // bounce-back
            act[m] = true;
            const TS* base = g + (int64_t)m * 7 * N;
            load7<TS, TC, ODD>(base, N, G, n, x, y, z, pop[m]);
            if ((west || east) && dyn != ADE_NONE) {
                // AdvectionDiffusionBoundaryDynamics: the one inward population makes the
                // node's density equal to the stored value
                const int type = west ? P.ltype[s] : P.rtype[s];
                double rs;
                if (type == CLB_DIRICHLET) rs = west ? P.lbc[s] : P.rbc[s];
                else rs = neu[((int64_t)s * 2 + (west ? 0 : 1)) * G.plane + (n - (int64_t)x * G.plane)];
                const int miss = west ? 4 : 1;
                TC sum = 0;
#pragma unroll
                for (int i = 0; i < 7; ++i)
                    if (i != miss) sum += pop[m][i];
                pop[m][miss] = (TC)(rs - 1.0) - sum;
            }
            TC r = 0;
#pragma unroll
            for (int i = 0; i < 7; ++i) r += pop[m][i];
            rb[m] = r;
        }
        // ---- kinetics (x = 1..nx-2, mask neither solid nor wall)
        double dC[CLB_MAX_SPECIES];
        for (int s = 0; s < P.S; ++s) dC[s] = 0.0;
        if (P.law != CLB_LAW_NONE && !west && !east && P.react[code]) {
            double C[CLB_MAX_SPECIES], R[CLB_MAX_SPECIES], B[CLB_MAX_MICROBES], RB[CLB_MAX_MICROBES];
            for (int s = 0; s < P.S; ++s) {
                double c;
                const int m = P.slot[s];
                if (m >= 0) {
                    c = 0.0;
#pragma unroll
                    for (int mm = 0; mm < NM; ++mm)
                        if (mm == m) c = (double)rb[mm] + 1.0;
                } else {
                    c = imm[(int64_t)s * N + n];
                }
                C[s] = c < THRD ? 0.0 : c;
            }
            for (int mb = 0; mb < P.M; ++mb) {
                const double b = bio[(int64_t)mb * N + n];
                B[mb] = b < THRD ? 0.0 : b;
            }
            eval_rates(P, C, B, R, RB);
            for (int s = 0; s < P.S; ++s) {
                double d = R[s] * P.dt;
                if (!(d > THRD || d < -THRD)) continue;
                if (d + C[s] < 0.0) d = -C[s];
                if (!(d > THRD || d < -THRD)) continue;
                if (P.slot[s] >= 0) dC[s] = d;
                else imm[(int64_t)s * N + n] += d;
            }
            for (int mb = 0; mb < P.M; ++mb) {
                double d = RB[mb] * P.dt;
                if (!(d > THRD || d < -THRD)) continue;
                if (d + B[mb] < 0.0) d = -B[mb];
                bio[(int64_t)mb * N + n] += d;
            }
        }
        // ---- collide, deposit, stream
        const TC ux = u[n], uy = u[N + n], uz = u[2 * N + n];
#pragma unroll
        for (int m = 0; m < NM; ++m) {
            if (!act[m]) continue;
            const int s = mob_species[m];
            TC o[7];
            if (dyn == ADE_NONE) {
#pragma unroll
                for (int i = 0; i < 7; ++i) o[i] = pop[m][i];
            } else {
                const TC w = (TC)(dyn == ADE_BIO ? P.wbio[s] : P.wpore[s]);
                const TC omw = (TC)1 - w;
                const TC rho = rb[m] + (TC)1;
                const TC jx = rho * ux, jy = rho * uy, jz = rho * uz;
                const TC d = (TC)dC[s];
#pragma unroll
                for (int i = 0; i < 7; ++i) {
                    const TC cj = (TC)q7cx(i) * jx + (TC)q7cy(i) * jy + (TC)q7cz(i) * jz;
                    o[i] = pop[m][i] * omw + w * ((TC)q7w(i) * (rb[m] + (TC)4 * cj));
                    o[i] += (TC)q7w(i) * d;
                }
            }
            store7<TS, TC, ODD>(g + (int64_t)m * 7 * N, N, G, n, x, y, z, o);
        }
    }
}

// The stored density of every Neumann plane node: the density of its inner neighbour as
// it stands before the step (FlatAdiabaticBoundaryFunctional3D after the previous stream).
// A node whose inner neighbour is not a fluid node keeps its previous value.
template <typename TS, typename TC, bool ODD>
__global__ void k_ade_neumann(const TS* __restrict__ g, const int8_t* __restrict__ mat, double* __restrict__ neu,
                              const AdeParams P, int s, int m, int side) {
    const Geom G = P.g;
    const int xb = side == 0 ? 0 : G.nx - 1, xi = side == 0 ? 1 : G.nx - 2;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < G.plane; p += gridDim.x * blockDim.x) {
        const int y = p / G.nz, z = p - y * G.nz;
        const int64_t nb = (int64_t)xb * G.plane + p, ni = (int64_t)xi * G.plane + p;
        const int db = P.dyn[mat[nb]], di = P.dyn[mat[ni]];
        if (!(db == ADE_PORE || db == ADE_BIO) || !(di == ADE_PORE || di == ADE_BIO)) continue;
        TC pop[7];
        load7<TS, TC, ODD>(g + (int64_t)m * 7 * G.N, G.N, G, ni, xi, y, z, pop);
        double r = 1.0;
        for (int i = 0; i < 7; ++i) r += (double)pop[i];
        neu[((int64_t)s * 2 + side) * G.plane + p] = r;
    }
}

template <typename TS>
__global__ void k_ade_init(TS* __restrict__ g, int64_t N, int n_mobile, const double* __restrict__ c0m) {
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
        for (int m = 0; m < n_mobile; ++m) {
            double c = c0m[m];
            if (c < THRD && c > -THRD) c = 0.0;
            for (int i = 0; i < 7; ++i) {
                double v = q7w(i) * (c - 1.0);
                if constexpr (std::is_same<TS, __half>::value) g[((int64_t)m * 7 + i) * N + n] = __double2half(v);
                else g[((int64_t)m * 7 + i) * N + n] = (TS)v;
            }
        }
    }
}

// Natural-layout incoming populations of one mobile species (parity rule), as FP64.
template <typename TS>
__global__ void k_ade_get_pops(const TS* __restrict__ g, const Geom G, int odd, double* __restrict__ out) {
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < G.N; n += (int64_t)gridDim.x * blockDim.x) {
        int x, y, z;
        decode(G, n, x, y, z);
        double v[7];
        if constexpr (std::is_same<TS, double>::value) {
            if (odd) load7<TS, double, true>(g, G.N, G, n, x, y, z, v);
            else load7<TS, double, false>(g, G.N, G, n, x, y, z, v);
        } else {
            float h[7];
            if (odd) load7<TS, float, true>(g, G.N, G, n, x, y, z, h);
            else load7<TS, float, false>(g, G.N, G, n, x, y, z, h);
            for (int i = 0; i < 7; ++i) v[i] = h[i];
        }
        for (int i = 0; i < 7; ++i) out[(int64_t)i * G.N + n] = v[i];
    }
}

template <typename TS>
__global__ void k_ade_set_pops(TS* __restrict__ g, const Geom G, int odd, const double* __restrict__ in) {
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < G.N; n += (int64_t)gridDim.x * blockDim.x) {
        int x, y, z;
        decode(G, n, x, y, z);
        for (int i = 0; i < 7; ++i) {
            int64_t slot = (int64_t)i * G.N + n;
            if (odd && i != 0) {
                const int cx = q7cx(i), cy = q7cy(i), cz = q7cz(i);
                const bool inb = ((unsigned)(x - cx) < (unsigned)G.nx) && ((unsigned)(y - cy) < (unsigned)G.ny) &&
                                 ((unsigned)(z - cz) < (unsigned)G.nz);
                const int64_t off = (int64_t)cx * G.plane + cy * G.nz + cz;
                if (inb) slot = (int64_t)q7opp(i) * G.N + n - off;
            }
            double v = in[(int64_t)i * G.N + n];
            if constexpr (std::is_same<TS, __half>::value) g[slot] = __double2half(v);
            else g[slot] = (TS)v;
        }
    }
}

// Per-block FP64 partials of the live fields: for each species the sum of concentration over
// open voxels of x=1..nx-2, the node content sum (sum of populations + 1 over every node),
// min, max; biomass sums; non-finite count.
template <typename TS>
__global__ void k_ade_reduce(const TS* __restrict__ g, const double* __restrict__ imm,
                             const double* __restrict__ bio, const int8_t* __restrict__ mat, const AdeParams P,
                             int n_mobile, const int* __restrict__ mob_species, int odd, double* __restrict__ part,
                             int nq) {
    const Geom G = P.g;
    // part layout per block: [S total][S content][S min][S max][M bio][1 nonfinite][1 open]
    extern __shared__ double shq[];
    for (int q = threadIdx.x; q < nq; q += blockDim.x) shq[q] = 0.0;
    const int S = P.S, M = P.M;
    for (int s = threadIdx.x; s < S; s += blockDim.x) {
        shq[2 * S + s] = 1e300;
        shq[3 * S + s] = -1e300;
    }
    __syncthreads();
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < G.N; n += (int64_t)gridDim.x * blockDim.x) {
        int x, y, z;
        decode(G, n, x, y, z);
        const int code = mat[n];
        const bool inner = (x >= 1 && x <= G.nx - 2);
        const bool open = inner && P.react[code] && P.dyn[code] != ADE_BB;
        if (open) atomicAdd(&shq[4 * S + M + 1], 1.0);
        for (int s = 0; s < S; ++s) {
            double c, content;
            const int m = P.slot[s];
            if (m >= 0) {
                double v[7];
                if constexpr (std::is_same<TS, double>::value) {
                    if (odd) load7<TS, double, true>(g + (int64_t)m * 7 * G.N, G.N, G, n, x, y, z, v);
                    else load7<TS, double, false>(g + (int64_t)m * 7 * G.N, G.N, G, n, x, y, z, v);
                } else {
                    float h[7];
                    if (odd) load7<TS, float, true>(g + (int64_t)m * 7 * G.N, G.N, G, n, x, y, z, h);
                    else load7<TS, float, false>(g + (int64_t)m * 7 * G.N, G.N, G, n, x, y, z, h);
                    for (int i = 0; i < 7; ++i) v[i] = h[i];
                }
                content = 1.0;
                for (int i = 0; i < 7; ++i) content += v[i];
                c = content;
            } else {
                c = imm[(int64_t)s * G.N + n];
                content = c;
            }
            atomicAdd(&shq[S + s], content);
            if (open) {
                atomicAdd(&shq[s], c);
                if (!isfinite(c)) atomicAdd(&shq[4 * S + M], 1.0);
                // min / max through CAS on shared doubles
                double cur = shq[2 * S + s];
                while (c < cur) {
                    unsigned long long old = atomicCAS((unsigned long long*)&shq[2 * S + s],
                                                       __double_as_longlong(cur), __double_as_longlong(c));
                    if (old == (unsigned long long)__double_as_longlong(cur)) break;
                    cur = __longlong_as_double(old);
                }
                cur = shq[3 * S + s];
                while (c > cur) {
                    unsigned long long old = atomicCAS((unsigned long long*)&shq[3 * S + s],
                                                       __double_as_longlong(cur), __double_as_longlong(c));
                    if (old == (unsigned long long)__double_as_longlong(cur)) break;
                    cur = __longlong_as_double(old);
                }
            }
        }
        if (inner)
            for (int mb = 0; mb < M; ++mb) atomicAdd(&shq[4 * S + mb], bio[(int64_t)mb * G.N + n]);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nq; q += blockDim.x) part[(int64_t)blockIdx.x * nq + q] = shq[q];
}

// ------------------------------------------------------------------ host side

static size_t esize(int prec) { return prec == CLB_F64 ? 8 : (prec == CLB_F32 ? 4 : 2); }
static size_t usize(int prec) { return prec == CLB_F64 ? 8 : 4; }

void ade_free(clb_handle* h) {
    cudaFree(h->d_g); h->d_g = nullptr;
    cudaFree(h->d_imm); h->d_imm = nullptr;
    cudaFree(h->d_bio); h->d_bio = nullptr;
    cudaFree(h->d_u); h->d_u = nullptr;
    cudaFree(h->d_ade_list); h->d_ade_list = nullptr;
    cudaFree(h->d_neu); h->d_neu = nullptr;
    h->ade_ready = false;
}

static int* mob_table(clb_handle* h) {
    // device copy of the mobile-species table lives after the neumann buffer
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
    std::vector<int> mob;
    std::vector<double> c0m;
    for (int s = 0; s < S; ++s) {
        P.mobile[s] = sp[s].mobile ? 1 : 0;
        P.slot[s] = -1;
        if (sp[s].mobile) { P.slot[s] = (int)mob.size(); mob.push_back(s); c0m.push_back(sp[s].c0); }
        P.ltype[s] = sp[s].left_type;
        P.rtype[s] = sp[s].right_type;
        P.lbc[s] = sp[s].left_bc;
        P.rbc[s] = sp[s].right_bc;
        P.wpore[s] = sp[s].omega_pore;
        P.wbio[s] = sp[s].omega_biofilm;
        P.c0[s] = sp[s].c0;
    }
    h->S = S;
    h->n_mobile = (int)mob.size();
    if (h->n_mobile > 16) return fail(h, CLB_INVALID_ARG, "at most 16 mobile species");
    h->M = 0;
    h->ade_prec = d.ade_precision;

    int8_t cls[MAX_CODES];
    for (int c = 0; c < MAX_CODES; ++c) cls[c] = (P.dyn[c] != ADE_BB);
    std::vector<int32_t> list = build_list(h, cls);
    const size_t N = (size_t)h->g.N;
    cudaError_t e;
    if ((e = cudaMalloc(&h->d_g, esize(h->ade_prec) * 7 * N * std::max(1, h->n_mobile))) != cudaSuccess)
        return cuda_check(h, e, "species populations");
    if ((e = cudaMalloc(&h->d_imm, sizeof(double) * N * S)) != cudaSuccess) return cuda_check(h, e, "immobile fields");
    if ((e = cudaMalloc(&h->d_u, usize(h->ade_prec) * 3 * N)) != cudaSuccess) return cuda_check(h, e, "velocity");
    if ((e = cudaMalloc(&h->d_ade_list, sizeof(int32_t) * std::max<size_t>(1, list.size()))) != cudaSuccess)
        return cuda_check(h, e, "ade list");
    if ((e = cudaMalloc(&h->d_neu, sizeof(double) * S * 2 * h->g.plane + sizeof(int) * 16)) != cudaSuccess)
        return cuda_check(h, e, "boundary store");
    h->n_ade_list = (int64_t)list.size();
    if (!list.empty())
        cudaMemcpyAsync(h->d_ade_list, list.data(), sizeof(int32_t) * list.size(), cudaMemcpyHostToDevice, h->stream);
    cudaMemsetAsync(h->d_u, 0, usize(h->ade_prec) * 3 * N, h->stream);
    // immobile species: uniform c0 (initial_concentration applies to the whole domain)
    std::vector<double> immh(N);
    for (int s = 0; s < S; ++s) {
        if (sp[s].mobile) continue;
        std::fill(immh.begin(), immh.end(), sp[s].c0);
        cudaMemcpy(h->d_imm + (size_t)s * N, immh.data(), sizeof(double) * N, cudaMemcpyHostToDevice);
    }
    // stored boundary densities: Dirichlet value, else c0 (lattice.initialize() runs the
    // Neumann processor once on the equilibrium field)
    std::vector<double> neu((size_t)S * 2 * h->g.plane);
    for (int s = 0; s < S; ++s)
        for (int side = 0; side < 2; ++side) {
            int t = side == 0 ? sp[s].left_type : sp[s].right_type;
            double v = t == CLB_DIRICHLET ? (side == 0 ? sp[s].left_bc : sp[s].right_bc) : sp[s].c0;
            std::fill(neu.begin() + ((size_t)s * 2 + side) * h->g.plane,
                      neu.begin() + ((size_t)s * 2 + side + 1) * h->g.plane, v);
        }
    cudaMemcpy(h->d_neu, neu.data(), sizeof(double) * neu.size(), cudaMemcpyHostToDevice);
    int mt[16] = {0};
    for (size_t k = 0; k < mob.size(); ++k) mt[k] = mob[k];
    cudaMemcpy(mob_table(h), mt, sizeof(mt), cudaMemcpyHostToDevice);
    double* dc0 = nullptr;
    if (!c0m.empty()) {
        cudaMalloc(&dc0, sizeof(double) * c0m.size());
        cudaMemcpy(dc0, c0m.data(), sizeof(double) * c0m.size(), cudaMemcpyHostToDevice);
        const int grid = h->num_sms * 8;
        switch (h->ade_prec) {
            case CLB_F64: k_ade_init<double><<<grid, 256, 0, h->stream>>>((double*)h->d_g, h->g.N, h->n_mobile, dc0); break;
            case CLB_F32: k_ade_init<float><<<grid, 256, 0, h->stream>>>((float*)h->d_g, h->g.N, h->n_mobile, dc0); break;
            default: k_ade_init<__half><<<grid, 256, 0, h->stream>>>((__half*)h->d_g, h->g.N, h->n_mobile, dc0); break;
        }
        cudaStreamSynchronize(h->stream);
        cudaFree(dc0);
    }
    h->ade_iters = 0;
    h->ade_grid = h->num_sms * 4;
    h->ade_ready = true;
    return cuda_check(h, cudaGetLastError(), "ade init");
}

clb_status ade_set_kinetics(clb_handle* h, int law, const double* prm, int nprm, double dt) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (nprm < 0 || nprm > 4 * CLB_MAX_SPECIES) return fail(h, CLB_INVALID_ARG, "too many kinetics parameters");
    if (law < 0 || law > CLB_LAW_DUAL_MONOD) return fail(h, CLB_INVALID_ARG, "unknown rate law");
    AdeParams& P = h->ap;
    P.law = law;
    std::memset(P.prm, 0, sizeof(P.prm));
    for (int k = 0; k < nprm; ++k) P.prm[k] = prm[k];
    P.dt = dt;
    return CLB_OK;
}

clb_status ade_set_biomass(clb_handle* h, int M, const double* b) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (M < 0 || M > CLB_MAX_MICROBES) return fail(h, CLB_INVALID_ARG, "microbe count out of range");
    cudaFree(h->d_bio);
    h->d_bio = nullptr;
    h->M = M;
    h->ap.M = M;
    if (M == 0) return CLB_OK;
    cudaError_t e = cudaMalloc(&h->d_bio, sizeof(double) * M * (size_t)h->g.N);
    if (e != cudaSuccess) return cuda_check(h, e, "biomass");
    e = cudaMemcpy(h->d_bio, b, sizeof(double) * M * (size_t)h->g.N, cudaMemcpyHostToDevice);
    return cuda_check(h, e, "biomass copy");
}

template <typename TS, typename TC, bool ODD>
static void launch_ade_t(clb_handle* h) {
    const int grid = h->ade_grid;
    const int nm = h->n_mobile;
    TS* g = (TS*)h->d_g;
    const TC* u = (const TC*)h->d_u;
    int* mt = mob_table(h);
#define CLB_ADE(NM)                                                                                        \
    k_ade_aa<TS, TC, ODD, NM><<<grid, ADE_THREADS, 0, h->stream>>>(g, h->d_imm, h->d_bio, u, h->d_ade_list, \
                                                                  h->n_ade_list, h->d_mat, h->d_neu, h->ap, nm, mt)
    if (nm <= 1) CLB_ADE(1);
    else if (nm <= 2) CLB_ADE(2);
    else if (nm <= 4) CLB_ADE(4);
    else if (nm <= 8) CLB_ADE(8);
    else CLB_ADE(16);
#undef CLB_ADE
}

template <typename TS, typename TC, bool ODD>
static void launch_neumann(clb_handle* h) {
    for (int s = 0; s < h->S; ++s) {
        const int m = h->ap.slot[s];
        if (m < 0) continue;
        for (int side = 0; side < 2; ++side) {
            int t = side == 0 ? h->ap.ltype[s] : h->ap.rtype[s];
            if (t != CLB_NEUMANN) continue;
            k_ade_neumann<TS, TC, ODD><<<std::max(1, std::min(h->num_sms * 2, (h->g.plane + 255) / 256)), 256, 0,
                                         h->stream>>>((const TS*)h->d_g, h->d_mat, h->d_neu, h->ap, s, m, side);
        }
    }
}

static void refresh_neumann(clb_handle* h) {
    const bool odd = (h->ade_iters & 1) != 0;
    switch (h->ade_prec) {
        case CLB_F64: if (odd) launch_neumann<double, double, true>(h); else launch_neumann<double, double, false>(h); break;
        case CLB_F32: if (odd) launch_neumann<float, float, true>(h); else launch_neumann<float, float, false>(h); break;
        default: if (odd) launch_neumann<__half, float, true>(h); else launch_neumann<__half, float, false>(h); break;
    }
}

clb_status ade_step(clb_handle* h, int n) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (h->M > 0 && h->d_bio == nullptr) return fail(h, CLB_INVALID_ARG, "biomass missing");
    for (int k = 0; k < n; ++k) {
        const bool odd = (h->ade_iters & 1) != 0;
        switch (h->ade_prec) {
            case CLB_F64:
                if (odd) { launch_neumann<double, double, true>(h); launch_ade_t<double, double, true>(h); }
                else { launch_neumann<double, double, false>(h); launch_ade_t<double, double, false>(h); }
                break;
            case CLB_F32:
                if (odd) { launch_neumann<float, float, true>(h); launch_ade_t<float, float, true>(h); }
                else { launch_neumann<float, float, false>(h); launch_ade_t<float, float, false>(h); }
                break;
            default:
                if (odd) { launch_neumann<__half, float, true>(h); launch_ade_t<__half, float, true>(h); }
                else { launch_neumann<__half, float, false>(h); launch_ade_t<__half, float, false>(h); }
                break;
        }
        h->ade_iters += 1;
    }
    return cuda_check(h, cudaGetLastError(), "ade step");
}

clb_status ade_couple(clb_handle* h) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (!h->flow_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_flow_init first");
    return flow_velocity(h, h->d_u, h->ade_prec == CLB_F64 ? 0 : 1, false);
}

clb_status ade_populations(clb_handle* h, int s, double* host) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (s < 0 || s >= h->S || h->ap.slot[s] < 0) return fail(h, CLB_INVALID_ARG, "not a mobile species");
    const int m = h->ap.slot[s];
    double* buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, sizeof(double) * 7 * (size_t)h->g.N);
    if (e != cudaSuccess) return cuda_check(h, e, "population buffer");
    const int odd = (int)(h->ade_iters & 1);
    const int grid = h->num_sms * 8;
    const size_t off = (size_t)m * 7 * h->g.N;
    switch (h->ade_prec) {
        case CLB_F64: k_ade_get_pops<double><<<grid, 256, 0, h->stream>>>((const double*)h->d_g + off, h->g, odd, buf); break;
        case CLB_F32: k_ade_get_pops<float><<<grid, 256, 0, h->stream>>>((const float*)h->d_g + off, h->g, odd, buf); break;
        default: k_ade_get_pops<__half><<<grid, 256, 0, h->stream>>>((const __half*)h->d_g + off, h->g, odd, buf); break;
    }
    e = cudaMemcpyAsync(host, buf, sizeof(double) * 7 * (size_t)h->g.N, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(buf);
    return cuda_check(h, e, "population copy");
}

clb_status ade_set_populations(clb_handle* h, int s, const double* host) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (s < 0 || s >= h->S || h->ap.slot[s] < 0) return fail(h, CLB_INVALID_ARG, "not a mobile species");
    const int m = h->ap.slot[s];
    double* buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, sizeof(double) * 7 * (size_t)h->g.N);
    if (e != cudaSuccess) return cuda_check(h, e, "population buffer");
    cudaMemcpy(buf, host, sizeof(double) * 7 * (size_t)h->g.N, cudaMemcpyHostToDevice);
    const int odd = (int)(h->ade_iters & 1);
    const int grid = h->num_sms * 8;
    const size_t off = (size_t)m * 7 * h->g.N;
    switch (h->ade_prec) {
        case CLB_F64: k_ade_set_pops<double><<<grid, 256, 0, h->stream>>>((double*)h->d_g + off, h->g, odd, buf); break;
        case CLB_F32: k_ade_set_pops<float><<<grid, 256, 0, h->stream>>>((float*)h->d_g + off, h->g, odd, buf); break;
        default: k_ade_set_pops<__half><<<grid, 256, 0, h->stream>>>((__half*)h->d_g + off, h->g, odd, buf); break;
    }
    e = cudaStreamSynchronize(h->stream);
    cudaFree(buf);
    return cuda_check(h, e, "set populations");
}

// computeDensity: BGK nodes of a Dirichlet / Neumann plane report the stored value; every
// other node the sum of its populations + 1; immobile species their field.
clb_status ade_density(clb_handle* h, int s, double* host) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (s < 0 || s >= h->S) return fail(h, CLB_INVALID_ARG, "species index out of range");
    const size_t N = (size_t)h->g.N;
    if (h->ap.slot[s] < 0) {
        cudaError_t e = cudaMemcpy(host, h->d_imm + (size_t)s * N, sizeof(double) * N, cudaMemcpyDeviceToHost);
        return cuda_check(h, e, "immobile copy");
    }
    // the Neumann planes' stored values as the reference holds them after the last stream
    refresh_neumann(h);
    std::vector<double> pops(7 * N);
    clb_status st = ade_populations(h, s, pops.data());
    if (st != CLB_OK) return st;
    std::vector<double> neu((size_t)2 * h->g.plane);
    cudaMemcpy(neu.data(), h->d_neu + (size_t)s * 2 * h->g.plane, sizeof(double) * neu.size(), cudaMemcpyDeviceToHost);
    const AdeParams& P = h->ap;
    for (size_t n = 0; n < N; ++n) {
        const int x = (int)(n / h->g.plane);
        const int p = (int)(n - (size_t)x * h->g.plane);
        const int dyn = P.dyn[(uint8_t)h->h_mat[n]];
        const bool bgk = dyn == ADE_PORE || dyn == ADE_BIO;
        if (bgk && x == 0 && P.ltype[s] != CLB_CLOSED) {
            host[n] = P.ltype[s] == CLB_DIRICHLET ? P.lbc[s] : neu[p];
            continue;
        }
        if (bgk && x == h->g.nx - 1 && P.rtype[s] != CLB_CLOSED) {
            host[n] = P.rtype[s] == CLB_DIRICHLET ? P.rbc[s] : neu[h->g.plane + p];
            continue;
        }
        double r = 1.0;
        for (int i = 0; i < 7; ++i) r += pops[(size_t)i * N + n];
        host[n] = r;
    }
    return CLB_OK;
}

clb_status ade_biomass(clb_handle* h, int m, double* host) {
    if (!h->ade_ready || m < 0 || m >= h->M) return fail(h, CLB_INVALID_ARG, "no such biomass field");
    cudaError_t e = cudaMemcpy(host, h->d_bio + (size_t)m * h->g.N, sizeof(double) * h->g.N, cudaMemcpyDeviceToHost);
    return cuda_check(h, e, "biomass copy");
}

clb_status ade_velocity(clb_handle* h, double* host) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    const size_t N = (size_t)h->g.N;
    if (h->ade_prec == CLB_F64) return cuda_check(h, cudaMemcpy(host, h->d_u, 8 * 3 * N, cudaMemcpyDeviceToHost), "u");
    std::vector<float> tmp(3 * N);
    cudaError_t e = cudaMemcpy(tmp.data(), h->d_u, 4 * 3 * N, cudaMemcpyDeviceToHost);
    for (size_t k = 0; k < 3 * N; ++k) host[k] = tmp[k];
    return cuda_check(h, e, "u");
}

clb_status ade_reduce(clb_handle* h, clb_stats* out) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    std::memset(out, 0, sizeof(*out));
    const int S = h->S, M = h->M;
    const int nq = 4 * S + M + 2;
    const int grid = h->num_sms * 2;
    double* part = nullptr;
    cudaError_t e = cudaMalloc(&part, sizeof(double) * nq * grid);
    if (e != cudaSuccess) return cuda_check(h, e, "reduce buffer");
    const int odd = (int)(h->ade_iters & 1);
    int* mt = mob_table(h);
    const size_t sh = sizeof(double) * nq;
    switch (h->ade_prec) {
        case CLB_F64: k_ade_reduce<double><<<grid, 256, sh, h->stream>>>((const double*)h->d_g, h->d_imm, h->d_bio, h->d_mat, h->ap, h->n_mobile, mt, odd, part, nq); break;
        case CLB_F32: k_ade_reduce<float><<<grid, 256, sh, h->stream>>>((const float*)h->d_g, h->d_imm, h->d_bio, h->d_mat, h->ap, h->n_mobile, mt, odd, part, nq); break;
        default: k_ade_reduce<__half><<<grid, 256, sh, h->stream>>>((const __half*)h->d_g, h->d_imm, h->d_bio, h->d_mat, h->ap, h->n_mobile, mt, odd, part, nq); break;
    }
    std::vector<double> hp((size_t)nq * grid);
    e = cudaMemcpyAsync(hp.data(), part, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(part);
    if (e != cudaSuccess) return cuda_check(h, e, "reduce");
    for (int s = 0; s < S; ++s) { out->min_c[s] = 1e300; out->max_c[s] = -1e300; }
    for (int b = 0; b < grid; ++b) {
        const double* q = &hp[(size_t)b * nq];
        for (int s = 0; s < S; ++s) {
            out->total[s] += q[s];
            out->content[s] += q[S + s];
            out->min_c[s] = std::min(out->min_c[s], q[2 * S + s]);
            out->max_c[s] = std::max(out->max_c[s], q[3 * S + s]);
        }
        for (int mb = 0; mb < M; ++mb) out->biomass[mb] += q[4 * S + mb];
        out->nonfinite += (int64_t)q[4 * S + M];
        out->open_voxels += (int64_t)q[4 * S + M + 1];
    }
    out->ade_iterations = h->ade_iters;
    return CLB_OK;
}

}  // namespace clb
