// geometry_update.cu -- precipitation sealing and dissolution reopening of voxels, and the
// dissolution of sealed mineral voxels into their open neighbours.
//
// Reference behaviour:
//   precipNodeConversion3D (precipitationVOP.hh:166-227), applied on Box3D(1, nx-2, ...) every
//     update interval (complab.cpp:3139-3146): a voxel whose mask is neither solid nor wall and whose
//     precipitate reached max_precipRho takes the precipitate's material code (the solid code) and
//     the precipitate phase stamp;
//   dissolNodeConversion3D (dissolutionVOP.hh:745-810): a stamped voxel whose mineral fell below
//     reopen_fraction x full_density becomes pore again and loses its stamp;
//   updateSoluteSolidDynamics3D (complab3d_processors_part2.hh:585-647): the species lattices switch
//     the voxel between BounceBack and advection-diffusion BGK and keep its populations;
//   updateNsLatticesDynamics3D (:748-818) skips voxels whose mask is the solid code, so on the flow
//     lattice a sealed voxel keeps its dynamics; `seal_flow` instead makes it bounce-back (or a
//     permeable IncBGK) and re-solves the flow, which is what the precipitation header describes;
//   surfaceDissolutionKinetics3D (dissolutionVOP.hh:379-605) and dissolutionGather3D (:608-742),
//     run inside the abiotic block of every transport step (complab.cpp:2496-2525).
//
// Design. A sealed voxel stays a node of the compacted species (and flow) layout; only its
// material code changes. The fused AA step skips a bounce-back node, which on AA slots is exactly
// the bounce-back collision, so the voxel keeps its populations for as long as it is sealed and
// resumes with them when it reopens, as Palabos' cells do. No relayout is needed.
//
// Dissolution runs as two small passes ahead of each fused step, over lists rebuilt whenever the
// geometry changes: the park pass over sealed voxels (rate from the water of the open face
// neighbours, the mineral debit, one product share per open face), and the gather pass over open
// voxels next to a sealed one, which recomputes their abiotic increment, adds the shares with the
// headroom clamp and hands the total to the fused step (AdeExtra). The concentrations both passes
// read are the ones the reference's processors see: the start-of-step density plus the step's
// biotic increment (post_biotic).
#include "kinetics.cuh"

#include <algorithm>
#include <cstring>

namespace clb {

constexpr int SEALED_FLOW_CODE = MAX_CODES - 1;  // flow-lattice material of a sealed voxel (seal_flow)
constexpr int GU_THREADS = 128;

static const int DLOC[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
__constant__ int c_dloc[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

// ------------------------------------------------------------------ node conversion kernels

// precipNodeConversion3D over the species lattice's nodes of x = 1..nx-2
__global__ void k_seal(int8_t* __restrict__ code, int8_t* __restrict__ mat, uint8_t* __restrict__ stamp,
                       const double* __restrict__ mineral, const SparseView S, const AdeParams P, int64_t k_lo,
                       int64_t k_hi, double full, int8_t pcode, unsigned int* __restrict__ count) {
    for (int64_t k = k_lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < k_hi; k += (int64_t)gridDim.x * blockDim.x) {
        if (!P.react[code[k]]) continue;
        const int64_t n = S.node[k];
        if (mineral[n] >= full) {
            code[k] = pcode;
            mat[n] = pcode;
            stamp[n] = 1;
            atomicAdd(count, 1u);
        }
    }
}

// dissolNodeConversion3D
__global__ void k_reopen(int8_t* __restrict__ code, int8_t* __restrict__ mat, uint8_t* __restrict__ stamp,
                         const double* __restrict__ mineral, const SparseView S, int64_t k_lo, int64_t k_hi,
                         double limit, int8_t pore, unsigned int* __restrict__ count) {
    for (int64_t k = k_lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < k_hi; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = S.node[k];
        if (!stamp[n]) continue;
        if (mineral[n] < limit) {
            code[k] = pore;
            mat[n] = pore;
            stamp[n] = 0;
            atomicAdd(count, 1u);
        }
    }
}

// the flow lattice's code of every flow node from its dense material map
__global__ void k_flow_codes(int8_t* __restrict__ code, const int32_t* __restrict__ node, int64_t K,
                             const int8_t* __restrict__ mat) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x)
        code[k] = mat[node[k]];
}

// ------------------------------------------------------------------ dissolution passes

// surfaceDissolutionKinetics3D over the sealed list. park[s][j]: the share of species s one open
// face of sealed voxel j receives this step (0: none).
template <typename TS, typename TC>
__global__ void k_dissolve_park(const TS* __restrict__ g, const TS* __restrict__ glink, double* __restrict__ imm,
                                const double* __restrict__ bio, const int8_t* __restrict__ mat, const SparseView S,
                                const AdeParams P, int n_mobile, const int32_t* __restrict__ seal, int64_t ns,
                                int64_t cap, int odd, double* __restrict__ park) {
    const Geom G = P.g;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < ns; j += (int64_t)gridDim.x * blockDim.x) {
        for (int s = 0; s < P.S; ++s) park[(int64_t)s * cap + j] = 0.0;
        const int64_t n = S.node[seal[j]];
        const double mineral = imm[(int64_t)P.sM * G.N + n];
        if (!(mineral > THRD)) continue;
        int x, y, z;
        decode(G, n, x, y, z);
        int64_t open[6];
        int no = 0;
        for (int d = 0; d < 6; ++d) {
            const int X = x + c_dloc[d][0], Y = y + c_dloc[d][1], Z = z + c_dloc[d][2];
            if (X < 1 || X > G.nx - 2 || Y < 0 || Y > G.ny - 1 || Z < 0 || Z > G.nz - 1) continue;
            const int64_t m = (int64_t)X * G.plane + (int64_t)Y * G.nz + Z;
            if (!P.react[mat[m]]) continue;
            open[no++] = m;
        }
        if (no == 0 && P.dis_surf) continue;
        double water[CLB_MAX_SPECIES], Cn[CLB_MAX_SPECIES], subsR[CLB_MAX_SPECIES];
        for (int s = 0; s < CLB_MAX_SPECIES; ++s) water[s] = 0.0;
        if (no > 0) {
            for (int q = 0; q < no; ++q) {
                post_biotic<TS, TC>(P, S, g, glink, imm, bio, n_mobile, open[q], odd, Cn);
                for (int s = 0; s < P.S; ++s) water[s] += Cn[s];
            }
            for (int s = 0; s < P.S; ++s) water[s] /= (double)no;
        }
        for (int s = 0; s < P.S; ++s)
            if (water[s] < 0.0) water[s] = 0.0;
        double mR;
        dissol_rate(P, water, mineral, subsR, mR);
        if (!(mR < 0.0)) continue;
        double dM = mR * P.dt;
        double scale = 1.0;
        const double maxRemove = 0.5 * mineral;  // MAX_DISSOL_FRACTION
        if (-dM > maxRemove) scale = maxRemove / (-dM);
        dM *= scale;
        if (!(-dM > THRD)) continue;
        imm[(int64_t)P.sM * G.N + n] += dM;
        if (no == 0) continue;
        for (int s = 0; s < P.S; ++s) {
            if (s == P.sM) continue;
            const double rel = subsR[s] * P.dt * scale;
            if (fabs(rel) <= THRD) continue;
            const double share = rel / (double)no;
            park[(int64_t)s * cap + j] = share;
            // update_abiotic_rxnLattices applies an immobile species' increment in a solid voxel too
            if (s >= n_mobile && (share > THRD || share < -THRD)) imm[(int64_t)s * G.N + n] += share;
        }
    }
}

// dissolutionGather3D over the open voxels next to sealed ones, with their own abiotic increment:
// xdc[s][i] is the node's whole abiotic-block increment of species s.
template <typename TS, typename TC>
__global__ void k_dissolve_gather(const TS* __restrict__ g, const TS* __restrict__ glink,
                                  const double* __restrict__ imm, const double* __restrict__ bio, const SparseView S,
                                  const AdeParams P, int n_mobile, const int32_t* __restrict__ gath,
                                  const int32_t* __restrict__ gath_nb, int64_t ng, int64_t gcap,
                                  const uint8_t* __restrict__ iface, const double* __restrict__ park, int64_t scap,
                                  int odd, double* __restrict__ xdc) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += (int64_t)gridDim.x * blockDim.x) {
        const int k = gath[i];
        const int64_t n = S.node[k];
        double Craw[CLB_MAX_SPECIES], tot[CLB_MAX_SPECIES];
        post_biotic<TS, TC>(P, S, g, glink, imm, bio, n_mobile, n, odd, Craw);
        for (int s = 0; s < CLB_MAX_SPECIES; ++s) tot[s] = 0.0;
        if (P.law2 != CLB_LAW_NONE && (!P.surf || iface[k])) {
            double C[CLB_MAX_SPECIES], R[CLB_MAX_SPECIES];
            for (int s = 0; s < CLB_MAX_SPECIES; ++s) C[s] = s < P.S ? (Craw[s] < THRD ? 0.0 : Craw[s]) : 0.0;
            eval_rates2<CLB_MAX_SPECIES>(P, C, R);
            for (int s = 0; s < P.S; ++s) {
                double d = R[s] * P.dt;
                if (!(d > THRD || d < -THRD)) continue;
                if (d + C[s] < 0.0) d = -C[s];
                if (!(d > THRD || d < -THRD)) continue;
                tot[s] = d;
            }
        }
        for (int d = 0; d < 6; ++d) {
            const int j = gath_nb[i * 6 + d];
            if (j < 0) continue;
            for (int s = 0; s < P.S; ++s) {
                if (s == P.sM) continue;
                const double share = park[(int64_t)s * scap + j];
                if (fabs(share) <= 1e-14) continue;
                double give = share;
                if (give < 0.0) {
                    // a consumed reactant may not take more than the voxel holds
                    const double have = Craw[s];
                    const double head = (have > 0.0 ? have : 0.0) + tot[s];
                    if (give + head < 0.0) give = -head;
                    if (give > 0.0) give = 0.0;
                }
                if (!(fabs(give) > 1e-14)) continue;
                tot[s] += give;
            }
        }
        for (int s = 0; s < P.S; ++s) xdc[(int64_t)s * gcap + i] = tot[s];
    }
}

// ------------------------------------------------------------------ host side

void precip_free(clb_handle* h) {
    cudaFree(h->d_stamp); h->d_stamp = nullptr;
    cudaFree(h->d_count); h->d_count = nullptr;
    cudaFree(h->d_iface); h->d_iface = nullptr;
    cudaFree(h->d_seal); h->d_seal = nullptr;
    cudaFree(h->d_gath); h->d_gath = nullptr;
    cudaFree(h->d_gath_nb); h->d_gath_nb = nullptr;
    cudaFree(h->d_xidx); h->d_xidx = nullptr;
    cudaFree(h->d_park); h->d_park = nullptr;
    cudaFree(h->d_xdc); h->d_xdc = nullptr;
    h->n_seal = h->seal_cap = h->n_gath = h->gath_cap = 0;
    h->prc_ready = false;
    h->ap.dis_on = 0;
}

AdeExtra ade_extra(clb_handle* h) {
    AdeExtra X;
    X.iface = h->d_iface;
    X.xidx = h->d_xidx;
    X.xdc = h->d_xdc;
    X.ng = h->gath_cap;
    return X;
}

static clb_status grow(clb_handle* h, void** p, size_t bytes, const char* what) {
    cudaFree(*p);
    *p = nullptr;
    cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    return e == cudaSuccess ? CLB_OK : cuda_check(h, e, what);
}

// Surface gate, sealed list, gather list and the row index of every species node, from the
// host material map and the stamp field.
clb_status geometry_refresh(clb_handle* h) {
    if (!h->ade_ready) return CLB_OK;
    {
        clb_status st = host_mat_sync(h);
        if (st != CLB_OK) return st;
    }
    const AdeParams& P = h->ap;
    const Geom G = h->g;
    const int64_t K = h->ade_sp.K;
    const bool need_iface = P.law2 != CLB_LAW_NONE && P.surf;
    const bool need_lists = P.law2 != CLB_LAW_NONE || P.dis_on;
    if (!need_iface && !need_lists) return CLB_OK;
    std::vector<int32_t> node((size_t)K);
    cudaError_t e = cudaMemcpy(node.data(), h->ade_sp.node, sizeof(int32_t) * K, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_check(h, e, "node list");
    std::vector<uint8_t> stamp((size_t)G.N, 0);
    if (h->d_stamp) {
        e = cudaMemcpy(stamp.data(), h->d_stamp, (size_t)G.N, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_check(h, e, "stamp field");
    }
    const std::vector<int8_t>& mat = h->h_mat;
    auto open = [&](int64_t n) { return P.react[(uint8_t)mat[n] & 127] != 0; };
    std::vector<uint8_t> iface((size_t)std::max<int64_t>(K, 1), 0);
    std::vector<int32_t> xidx((size_t)std::max<int64_t>(K, 1), -1);
    std::vector<int32_t> seal, gath, gnb;
    std::vector<int32_t> seal_row;
    if (P.dis_on) seal_row.assign((size_t)G.N, -1);
    for (int64_t k = 0; k < K; ++k) {
        const int64_t n = node[k];
        const int x = (int)(n / G.plane), r = (int)(n - (int64_t)x * G.plane), y = r / G.nz, z = r - y * G.nz;
        for (int d = 0; d < 6; ++d) {
            const int X = x + DLOC[d][0], Y = y + DLOC[d][1], Z = z + DLOC[d][2];
            if (X < 0 || Y < 0 || Z < 0 || X >= G.nx || Y >= G.ny || Z >= G.nz) continue;
            if (!open((int64_t)X * G.plane + (int64_t)Y * G.nz + Z)) iface[k] = 1;
        }
        if (P.dis_on && stamp[n] && x >= 1 && x <= G.nx - 2) {
            seal_row[n] = (int32_t)seal.size();
            seal.push_back((int32_t)k);
        }
    }
    if (P.dis_on)
        for (int64_t k = 0; k < K; ++k) {
            const int64_t n = node[k];
            const int x = (int)(n / G.plane), r = (int)(n - (int64_t)x * G.plane), y = r / G.nz, z = r - y * G.nz;
            if (x < 1 || x > G.nx - 2 || !open(n)) continue;
            int32_t nb[6];
            bool any = false;
            for (int d = 0; d < 6; ++d) {
                nb[d] = -1;
                const int X = x + DLOC[d][0], Y = y + DLOC[d][1], Z = z + DLOC[d][2];
                if (X < 1 || X > G.nx - 2 || Y < 0 || Y > G.ny - 1 || Z < 0 || Z > G.nz - 1) continue;
                const int64_t m = (int64_t)X * G.plane + (int64_t)Y * G.nz + Z;
                if (seal_row[m] >= 0) { nb[d] = seal_row[m]; any = true; }
            }
            if (!any) continue;
            xidx[k] = (int32_t)gath.size();
            gath.push_back((int32_t)k);
            gnb.insert(gnb.end(), nb, nb + 6);
        }
    clb_status st;
    if (!h->d_iface) {
        if ((st = grow(h, (void**)&h->d_iface, (size_t)std::max<int64_t>(K, 1), "surface gate")) != CLB_OK) return st;
        if ((st = grow(h, (void**)&h->d_xidx, sizeof(int32_t) * std::max<int64_t>(K, 1), "gather index")) != CLB_OK) return st;
    }
    cudaMemcpy(h->d_iface, iface.data(), iface.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_xidx, xidx.data(), sizeof(int32_t) * xidx.size(), cudaMemcpyHostToDevice);
    const int S = h->S;
    if ((int64_t)seal.size() > h->seal_cap || !h->d_seal) {
        h->seal_cap = std::max<int64_t>((int64_t)seal.size() * 2, 256);
        if ((st = grow(h, (void**)&h->d_seal, sizeof(int32_t) * h->seal_cap, "sealed list")) != CLB_OK) return st;
        if ((st = grow(h, (void**)&h->d_park, sizeof(double) * S * h->seal_cap, "parked shares")) != CLB_OK) return st;
    }
    if ((int64_t)gath.size() > h->gath_cap || !h->d_gath) {
        h->gath_cap = std::max<int64_t>((int64_t)gath.size() * 2, 256);
        if ((st = grow(h, (void**)&h->d_gath, sizeof(int32_t) * h->gath_cap, "gather list")) != CLB_OK) return st;
        if ((st = grow(h, (void**)&h->d_gath_nb, sizeof(int32_t) * 6 * h->gath_cap, "gather list")) != CLB_OK) return st;
        if ((st = grow(h, (void**)&h->d_xdc, sizeof(double) * S * h->gath_cap, "gathered increments")) != CLB_OK) return st;
    }
    h->n_seal = (int64_t)seal.size();
    h->n_gath = (int64_t)gath.size();
    if (!seal.empty()) cudaMemcpy(h->d_seal, seal.data(), sizeof(int32_t) * seal.size(), cudaMemcpyHostToDevice);
    if (!gath.empty()) {
        cudaMemcpy(h->d_gath, gath.data(), sizeof(int32_t) * gath.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(h->d_gath_nb, gnb.data(), sizeof(int32_t) * gnb.size(), cudaMemcpyHostToDevice);
    }
    return cuda_check(h, cudaGetLastError(), "geometry lists");
}

template <typename TS, typename TC>
static void launch_dissolution(clb_handle* h) {
    const int odd = (int)(h->ade_iters & 1);
    const SparseView S = view_of(h->ade_sp);
    const TS* g = (const TS*)h->d_g;
    const TS* gl = (const TS*)h->d_glink;
    h->launches += (h->n_seal > 0) + (h->n_gath > 0);
    if (h->n_seal > 0)
        k_dissolve_park<TS, TC><<<(int)std::min<int64_t>((h->n_seal + GU_THREADS - 1) / GU_THREADS, h->num_sms * 4),
                                  GU_THREADS, 0, h->stream>>>(g, gl, h->d_imm, h->d_bio, h->d_mat, S, h->ap,
                                                              h->n_mobile, h->d_seal, h->n_seal, h->seal_cap, odd,
                                                              h->d_park);
    if (h->n_gath > 0)
        k_dissolve_gather<TS, TC><<<(int)std::min<int64_t>((h->n_gath + GU_THREADS - 1) / GU_THREADS, h->num_sms * 4),
                                    GU_THREADS, 0, h->stream>>>(g, gl, h->d_imm, h->d_bio, S, h->ap, h->n_mobile,
                                                                h->d_gath, h->d_gath_nb, h->n_gath, h->gath_cap,
                                                                h->d_iface, h->d_park, h->seal_cap, odd, h->d_xdc);
}

clb_status dissolution_pre_step(clb_handle* h) {
    if (h->M > 0 && h->d_bio == nullptr) return fail(h, CLB_INVALID_ARG, "biomass missing");
    switch (h->ade_prec) {
        case CLB_F64: launch_dissolution<double, double>(h); break;
        case CLB_F32: launch_dissolution<float, float>(h); break;
        default: launch_dissolution<__half, float>(h); break;
    }
    return CLB_OK;
}

clb_status precip_setup(clb_handle* h, const clb_precip_desc* d) {
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    const int S = h->S;
    if (d->mineral_species < 0 || d->mineral_species >= S) return fail(h, CLB_INVALID_ARG, "mineral species index");
    const int mi = h->u2i[d->mineral_species];
    if (h->ap.slot[mi] >= 0) return fail(h, CLB_INVALID_ARG, "the mineral must be an immobile species");
    if (!(d->full_density > 0)) return fail(h, CLB_INVALID_ARG, "full_density must be positive");
    int pcode = d->precip_code < 0 ? h->d.solid_code : d->precip_code;
    if (pcode < 0 || pcode >= MAX_CODES) return fail(h, CLB_INVALID_ARG, "no material code for sealed voxels");
    if (h->ap.dyn[pcode] != ADE_BB || h->ap.react[pcode])
        return fail(h, CLB_INVALID_ARG, "the precipitate code must be the solid or the bounce-back code");
    int pore = d->pore_code < 0 ? (h->d.n_pore_codes > 0 ? h->d.pore_codes[0] : 2) : d->pore_code;
    if (d->dissolution) {
        if (!(d->reopen_fraction >= 0 && d->reopen_fraction < 1))
            return fail(h, CLB_INVALID_ARG, "reopen_fraction must lie in [0, 1)");
        if (pore < 0 || pore >= MAX_CODES || !h->ap.react[pore] || h->ap.dyn[pore] == ADE_BB)
            return fail(h, CLB_INVALID_ARG, "the reopened voxel's code must be an open material");
        if (d->dissolution_law < CLB_DISSOL_NONE || d->dissolution_law > CLB_DISSOL_MINERAL)
            return fail(h, CLB_INVALID_ARG, "unknown dissolution law");
    }
    if (d->seal_flow) {
        clb_status hs = host_mat_sync(h);
        if (hs != CLB_OK) return hs;
        for (int64_t n = 0; n < h->g.N; ++n)
            if ((uint8_t)h->h_mat[n] == SEALED_FLOW_CODE)
                return fail(h, CLB_INVALID_ARG, "seal_flow reserves material code 127");
        if (!h->flow_ready) return fail(h, CLB_NOT_INITIALIZED, "seal_flow needs clb_flow_init first");
    }
    h->prc = *d;
    h->prc.precip_code = pcode;
    h->prc.pore_code = pore;
    AdeParams& P = h->ap;
    P.sM = mi;
    P.dis_on = d->dissolution ? 1 : 0;
    P.dis_law = d->dissolution_law;
    P.dis_surf = d->dissolution_surface_only ? 1 : 0;
    std::memset(P.dprm, 0, sizeof(P.dprm));
    if (P.dis_law == CLB_DISSOL_FIRST_ORDER) {
        P.dprm[0] = d->dissolution_params[0];
        const int hs = (int)d->dissolution_params[1];
        if (hs >= S) return fail(h, CLB_INVALID_ARG, "dissolution law: species index out of range");
        P.dprm[1] = hs >= 0 ? h->u2i[hs] : -1;
        for (int i = 0; i < S; ++i) P.dprm[2 + i] = d->dissolution_params[2 + h->i2u[i]];
    } else if (P.dis_law == CLB_DISSOL_MINERAL) {
        P.dprm[0] = d->dissolution_params[0];
        P.dprm[1] = d->dissolution_params[1];
        for (int i = 0; i < S; ++i) P.dprm[2 + i] = d->dissolution_params[2 + h->i2u[i]];
    }
    cudaError_t e = cudaSuccess;
    if (!h->d_stamp) {
        e = cudaMalloc(&h->d_stamp, (size_t)h->g.N);
        if (e == cudaSuccess) e = cudaMemsetAsync(h->d_stamp, 0, (size_t)h->g.N, h->stream);
    }
    if (e == cudaSuccess && !h->d_count) e = cudaMalloc(&h->d_count, sizeof(unsigned int) * 4);
    if (e != cudaSuccess) return cuda_check(h, e, "precipitation state");
    if (d->seal_flow) {
        FlowParams& F = h->fp;
        const double omega = 1.0 / h->d.tau;
        const double r = d->seal_perm_ratio;
        F.dyn[SEALED_FLOW_CODE] = r > 1e-14 ? DYN_BGK : DYN_BB;
        F.omega[SEALED_FLOW_CODE] = r > 1e-14 ? 1.0 / (r * (1.0 / omega - 0.5) + 0.5) : 0.0;
    }
    h->prc_ready = true;
    return geometry_refresh(h);
}

// Re-derive the flow lattice's dynamics from the species' map: sealed voxels take
// SEALED_FLOW_CODE, everything else its current material.
static clb_status flow_follow(clb_handle* h) {
    const int64_t N = h->g.N;
    std::vector<uint8_t> stamp((size_t)N);
    cudaError_t e = cudaMemcpy(stamp.data(), h->d_stamp, (size_t)N, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_check(h, e, "stamp field");
    h->h_mat_flow = h->h_mat;
    for (int64_t n = 0; n < N; ++n)
        if (stamp[n]) h->h_mat_flow[n] = (int8_t)SEALED_FLOW_CODE;
    if (!h->d_mat_flow) {
        e = cudaMalloc(&h->d_mat_flow, (size_t)N);
        if (e != cudaSuccess) return cuda_check(h, e, "flow material map");
    }
    e = cudaMemcpy(h->d_mat_flow, h->h_mat_flow.data(), (size_t)N, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_check(h, e, "flow material map");
    ++h->launches;
    k_flow_codes<<<h->num_sms * 4, 256, 0, h->stream>>>(h->flow_sp.code, h->flow_sp.node, h->flow_sp.K, h->d_mat_flow);
    int64_t nbgk = 0;
    for (int64_t n = 0; n < N; ++n) nbgk += h->fp.dyn[(uint8_t)h->h_mat_flow[n] & 127] == DYN_BGK;
    h->fp.n_bgk = nbgk;
    return cuda_check(h, cudaGetLastError(), "flow codes");
}

clb_status geometry_update(clb_handle* h, int* sealed, int* reopened) {
    if (!h->prc_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_precip_setup first");
    const AdeParams& P = h->ap;
    const double* mineral = h->d_imm + (size_t)P.sM * h->g.N;
    const SparseView S = view_of(h->ade_sp);
    const int64_t lo = h->ade_west_end, hi = h->ade_east_begin;  // x = 1..nx-2
    const int grid = h->num_sms * 4;
    // the Neumann planes' stored densities belong to the last stream, with the map before the change
    ade_refresh_neumann(h);
    cudaMemsetAsync(h->d_count, 0, sizeof(unsigned int) * 4, h->stream);
    h->launches += 1 + (h->prc.dissolution ? 1 : 0);
    k_seal<<<grid, 256, 0, h->stream>>>(h->ade_sp.code, h->d_mat, h->d_stamp, mineral, S, P, lo, hi,
                                        h->prc.full_density, (int8_t)h->prc.precip_code, h->d_count);
    if (h->prc.dissolution)
        k_reopen<<<grid, 256, 0, h->stream>>>(h->ade_sp.code, h->d_mat, h->d_stamp, mineral, S, lo, hi,
                                              h->prc.reopen_fraction * h->prc.full_density,
                                              (int8_t)h->prc.pore_code, h->d_count + 1);
    unsigned int cnt[4] = {0, 0, 0, 0};
    cudaError_t e = cudaMemcpyAsync(cnt, h->d_count, sizeof(cnt), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_check(h, e, "geometry update");
    if (sealed) *sealed = (int)cnt[0];
    if (reopened) *reopened = (int)cnt[1];
    if (cnt[0] == 0 && cnt[1] == 0) return CLB_OK;
    h->ca_full = true;  // the automaton's next mask pass looks at the whole changed map
    if (!h->d_mat_flow) {
        // from now on the flow lattice has a map of its own: the one before the first change
        h->h_mat_flow = h->h_mat;
        e = cudaMalloc(&h->d_mat_flow, (size_t)h->g.N);
        if (e == cudaSuccess)
            e = cudaMemcpy(h->d_mat_flow, h->h_mat_flow.data(), (size_t)h->g.N, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_check(h, e, "flow material map");
    }
    e = cudaMemcpy(h->h_mat.data(), h->d_mat, (size_t)h->g.N, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_check(h, e, "material copy");
    h->h_mat_stale = false;
    clb_status st = geometry_refresh(h);
    if (st != CLB_OK) return st;
    if (h->prc.seal_flow && h->flow_ready) {
        st = flow_follow(h);
        if (st != CLB_OK) return st;
        int it = 0;
        st = flow_solve(h, h->prc.flow_max_iterations, h->prc.flow_eps, &it, true);
        if (st != CLB_OK && st != CLB_NOT_CONVERGED) return st;
        const clb_status cs = ade_couple(h);
        if (cs != CLB_OK) return cs;
        return st;
    }
    return CLB_OK;
}

}  // namespace clb
