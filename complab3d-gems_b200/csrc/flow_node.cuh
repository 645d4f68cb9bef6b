// flow_node.cuh -- one node of the D3Q19 AA step (collision, pressure planes, the even step's
// own-slot access and the odd step's neighbour-row gathers and scatters). Shared by the
// single-domain flow steps (flow.cu) and the batched steps of many domains, so every path runs
// the same per-node arithmetic.
#pragma once

#include "sparse.cuh"

namespace clb {

template <typename TC>
__device__ __forceinline__ TC feq19(int i, TC rb, TC jx, TC jy, TC jz, TC jsq) {
    TC cj = (TC)q19cx(i) * jx + (TC)q19cy(i) * jy + (TC)q19cz(i) * jz;
    return (TC)q19w(i) * (rb + (TC)3 * cj + (TC)1.5 * ((TC)3 * cj * cj - jsq));
}

// Palabos' regularized density boundary on the x planes (direction 0, orientation o):
// j_x = o (rb_0 + 2 rb_n - rb), j_y = j_z = 0, Pi_neq from the known populations with the
// off-equilibrium parts of the normal ones counted twice, then f_i = feq_i + fneq_i(Pi).
template <typename TC>
__device__ __forceinline__ void regularize19(TC (&g)[19], int orient, TC rb) {
    TC r0 = 0, rn = 0;
#pragma unroll
    for (int i = 0; i < 19; ++i) {
        if (q19cx(i) == 0) r0 += g[i];
        else if (q19cx(i) == orient) rn += g[i];
    }
    const TC jx = (TC)orient * (r0 + (TC)2 * rn - rb);
    const TC jsq = jx * jx;
    TC pxx = 0, pxy = 0, pxz = 0, pyy = 0, pyz = 0, pzz = 0;
#pragma unroll
    for (int i = 1; i < 19; ++i) {
        const int cx = q19cx(i);
        if (cx == -orient) continue;
        const TC fac = (cx == 0) ? (TC)1 : (TC)2;
        const TC fneq = fac * (g[i] - feq19<TC>(i, rb, jx, (TC)0, (TC)0, jsq));
        pxx += (TC)(q19cx(i) * q19cx(i)) * fneq;
        pxy += (TC)(q19cx(i) * q19cy(i)) * fneq;
        pxz += (TC)(q19cx(i) * q19cz(i)) * fneq;
        pyy += (TC)(q19cy(i) * q19cy(i)) * fneq;
        pyz += (TC)(q19cy(i) * q19cz(i)) * fneq;
        pzz += (TC)(q19cz(i) * q19cz(i)) * fneq;
    }
    const TC third = (TC)1 / (TC)3;
#pragma unroll
    for (int i = 0; i < 19; ++i) {
        const TC cx = q19cx(i), cy = q19cy(i), cz = q19cz(i);
        TC s = (cx * cx - third) * pxx + (cy * cy - third) * pyy + (cz * cz - third) * pzz +
               (TC)2 * (cx * cy * pxy + cx * cz * pxz + cy * cz * pyz);
        g[i] = feq19<TC>(i, rb, jx, (TC)0, (TC)0, jsq) + (TC)q19w(i) * (TC)4.5 * s;
    }
}


// IncBGK collision of one node in place, in opposite-pair form: for the pair (i, opp(i)) with
// cj = c_i . j, feq = t (rb - 1.5 |j|^2 + 4.5 cj^2) +- 3 t cj. Written out per direction so no
// term is multiplied by a zero velocity component (IEEE-strict code cannot fold 0 * x away).
// Returns |j|^2.
template <typename TC>
__device__ __forceinline__ TC bgk19(TC (&g)[19], TC w) {
    const TC rb = (((g[0] + g[1]) + (g[2] + g[3])) + ((g[4] + g[5]) + (g[6] + g[7]))) +
                  (((g[8] + g[9]) + (g[10] + g[11])) + ((g[12] + g[13]) + (g[14] + g[15]))) + ((g[16] + g[17]) + g[18]);
    const TC jx = ((g[10] + g[13]) + (g[14] + g[15]) + g[16]) - ((g[1] + g[4]) + (g[5] + g[6]) + g[7]);
    const TC jy = ((g[5] + g[11]) + (g[13] + g[17]) + g[18]) - ((g[2] + g[4]) + (g[8] + g[9]) + g[14]);
    const TC jz = ((g[7] + g[9]) + (g[12] + g[15]) + g[17]) - ((g[3] + g[6]) + (g[8] + g[16]) + g[18]);
    const TC jsq = jx * jx + jy * jy + jz * jz;
    const TC omw = (TC)1 - w;
    const TC base = rb - (TC)1.5 * jsq;
    const TC t1 = (TC)(1.0 / 18.0), t2 = (TC)(1.0 / 36.0);
    g[0] = omw * g[0] + w * ((TC)(1.0 / 3.0) * base);
#define CLB_PAIR(I, CJ, T)                                          \
    {                                                               \
        const TC cj = (CJ);                                         \
        const TC sym = (T) * (base + (TC)4.5 * cj * cj);            \
        const TC asym = (T) * ((TC)3 * cj);                         \
        g[I] = omw * g[I] + w * (sym + asym);                       \
        g[I + 9] = omw * g[I + 9] + w * (sym - asym);               \
    }
    CLB_PAIR(1, -jx, t1)
    CLB_PAIR(2, -jy, t1)
    CLB_PAIR(3, -jz, t1)
    CLB_PAIR(4, -jx - jy, t2)
    CLB_PAIR(5, -jx + jy, t2)
    CLB_PAIR(6, -jx - jz, t2)
    CLB_PAIR(7, -jx + jz, t2)
    CLB_PAIR(8, -jy - jz, t2)
    CLB_PAIR(9, -jy + jz, t2)
#undef CLB_PAIR
    return jsq;
}


// The per-node metadata a step reads before the populations (loaded one node ahead by the
// single-domain step so its latency overlaps the previous node's work).
struct FlowMeta {
    int code;
    uint32_t m0, m1;
    int4 dv;
};

template <bool ODD>
__device__ __forceinline__ FlowMeta flow_meta(const SparseView& S, int64_t k) {
    FlowMeta M;
    M.code = S.code[k];
    M.m0 = S.meta[2 * k];
    if (ODD) {
        M.m1 = S.meta[2 * k + 1];
        M.dv = *reinterpret_cast<const int4*>(S.dres + 8 * k);
    } else {
        M.m1 = 0;
        M.dv = make_int4(0, 0, 0, 0);
    }
    return M;
}

// Odd-step geometry of node k from its metadata: the compact index bases of its 8 neighbour rows
// (rb), the directions whose neighbour is a wall or outside the box (blk) and the row-parity bits.
struct OddRows {
    int rb[8];
    uint32_t blk, rbit;
};

__device__ __forceinline__ OddRows odd_rows(const SparseView& S, int64_t k, const FlowMeta& M) {
    OddRows R;
    const int t = (int)(k >> 8);
    R.blk = (M.m0 | M.m1) & 0x7FFFFu;  // wall or outside the box: the node's own opposite slot
    R.rbit = M.m1 >> 19;
    const int4 dv = M.dv;
    const int* tb = S.tdb + 8 * t;
    R.rb[0] = (int)k + tb[0] + (int16_t)(dv.x & 0xFFFF);
    R.rb[1] = (int)k + tb[1] + (int16_t)((uint32_t)dv.x >> 16);
    R.rb[2] = (int)k + tb[2] + (int16_t)(dv.y & 0xFFFF);
    R.rb[3] = (int)k + tb[3] + (int16_t)((uint32_t)dv.y >> 16);
    R.rb[4] = (int)k + tb[4] + (int16_t)(dv.z & 0xFFFF);
    R.rb[5] = (int)k + tb[5] + (int16_t)((uint32_t)dv.z >> 16);
    R.rb[6] = (int)k + tb[6] + (int16_t)(dv.w & 0xFFFF);
    R.rb[7] = (int)k + tb[7] + (int16_t)((uint32_t)dv.w >> 16);
    return R;
}

// storage slot (row offset + index) an odd step reads incoming population i of node k from
__device__ __forceinline__ uint32_t odd_src(int i, int64_t k, const OddRows& R, uint32_t K32) {
    if (i == 0) return (uint32_t)k;
    const int cx = q19cx(i), cy = q19cy(i), cz = q19cz(i), oi = q19opp(i);
    if ((R.blk >> oi) & 1u) return (uint32_t)(i * K32) + (uint32_t)k;
    int src;
    if (cx == 0 && cy == 0) src = (int)k - cz;
    else {
        const int s8 = row8(-cx, -cy);
        src = (cz == 0) ? R.rb[s8] : (-cz > 0 ? R.rb[s8] + (int)((R.rbit >> s8) & 1u) : R.rb[s8] - 1);
    }
    return (uint32_t)(oi * K32) + (uint32_t)src;
}

// storage slot an odd step writes outgoing population i of node k to
__device__ __forceinline__ uint32_t odd_dst(int i, int64_t k, const OddRows& R, uint32_t K32) {
    if (i == 0) return (uint32_t)k;
    const int cx = q19cx(i), cy = q19cy(i), cz = q19cz(i), oi = q19opp(i);
    if ((R.blk >> i) & 1u) return (uint32_t)(oi * K32) + (uint32_t)k;
    int dst;
    if (cx == 0 && cy == 0) dst = (int)k + cz;
    else {
        const int s8 = row8(cx, cy);
        dst = (cz == 0) ? R.rb[s8] : (cz > 0 ? R.rb[s8] + (int)((R.rbit >> s8) & 1u) : R.rb[s8] - 1);
    }
    return (uint32_t)(i * K32) + (uint32_t)dst;
}

// One node of the AA step (the flow lattice's collide-and-stream at compact index k); returns
// the node's |u|^2 when it is a BGK node (for the stored average energy), else 0. Shared by the
// single-domain step and the batched step of many domains.
template <typename TS, typename TC, bool ODD, typename FP>
__device__ __forceinline__ double flow_node_m(TS* __restrict__ f, TS* __restrict__ link, const SparseView& S, const FP& P,
                                              int64_t k, int64_t k_west_end, int64_t k_east_begin, const FlowMeta& M) {
    const uint32_t K32 = (uint32_t)S.KS;  // row stride; 19 KS < 2^31 is checked when the layout is built
    double e = 0.0;
    const int code = M.code;
    // a stored bounce-back node (a voxel sealed by precipitation): the identity on AA slots
    if (P.dyn[code] == DYN_BB) return 0.0;
    TC g[19];
    uint32_t ad[19];
    uint32_t wm = 0;
    int lb = 0;
    if (!ODD) {
        // own slots; a wall link (a, i) takes its incoming opp(i) from its even-step slot X
        // and its odd-step slot Y = f[opp(i)][a] is written back unchanged (whole sectors)
        const uint32_t m0 = M.m0;
        wm = m0 & 0x7FFFFu;
        lb = S.tlb[(int)(k >> 8)] + (int)(m0 >> 19);
#pragma unroll
        for (int i = 0; i < 19; ++i) g[i] = ld<TS, TC>(f + (uint32_t)(i * K32) + k);
        if (wm) {
#pragma unroll
            for (int i = 1; i < 19; ++i) {
                if (!((wm >> i) & 1u)) continue;
                const int oi = q19opp(i);
                st<TS, TC>(f + (uint32_t)(oi * K32) + k, g[oi]);
                g[oi] = ld<TS, TC>(link + lb + __popc(wm & ((1u << i) - 1u)));
            }
        }
    } else {
        // an in-place permutation: incoming i is read from slot ad[i], outgoing opp(i) goes back there
        const OddRows R = odd_rows(S, k, M);
#pragma unroll
        for (int i = 0; i < 19; ++i) {
            ad[i] = odd_src(i, k, R, K32);
            g[i] = ld<TS, TC>(f + ad[i]);
        }
    }
    if (P.dyn[code] == DYN_BGK) {
        if (k < k_west_end) regularize19<TC>(g, -1, (TC)(P.rho_w - 1.0));
        else if (k >= k_east_begin) regularize19<TC>(g, 1, (TC)(P.rho_e - 1.0));
        e = (double)bgk19<TC>(g, (TC)P.omega[code]);
    }
    if (!ODD) {
#pragma unroll
        for (int i = 0; i < 19; ++i) {
            if ((wm >> i) & 1u) st<TS, TC>(link + lb + __popc(wm & ((1u << i) - 1u)), g[i]);
            else st<TS, TC>(f + (uint32_t)(q19opp(i) * K32) + k, g[i]);
        }
    } else {
#pragma unroll
        for (int i = 0; i < 19; ++i) st<TS, TC>(f + ad[q19opp(i)], g[i]);
    }
    return e;
}

template <typename TS, typename TC, bool ODD, typename FP>
__device__ __forceinline__ double flow_node(TS* __restrict__ f, TS* __restrict__ link, const SparseView& S, const FP& P,
                                            int64_t k, int64_t k_west_end, int64_t k_east_begin) {
    return flow_node_m<TS, TC, ODD>(f, link, S, P, k, k_west_end, k_east_begin, flow_meta<ODD>(S, k));
}

}  // namespace clb
