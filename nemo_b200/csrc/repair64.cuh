// repair64.cuh -- positivity repair of one element held in shared memory (FP64, rare path).
#pragma once

#include "common.cuh"
#include "euler_fp64.cuh"
#include "mhd_phys.cuh"

namespace nemo {

// dgfv_repair_3d (source/kernel/mcfv/3d/kernel_validate_mod.f90:159-272) with N_NODES = 4: if a
// node is inadmissible, squeeze 2x2x2 tiles of node means towards their mean in steps of
// repair_decr until the tile means are admissible, first on the 8 octants (2^3 nodes each), then
// node by node inside each octant.  su holds the tile's state [5][EPC][64]; one thread per element.
template <int EPC>
__device__ __noinline__ bool repair_elem(double* su, int el, const OpConsts& k) {
    constexpr int V = 5;
    auto at = [&](int v, int p) -> double& { return su[(v * EPC + el) * NP + p]; };
    auto node_ok = [&](int p) {
        double q[5];
        for (int v = 0; v < V; ++v) q[v] = at(v, p);
        return isvalid64(q, k);
    };
    bool ok = true;
    for (int p = 0; p < NP; ++p) ok = ok && node_ok(p);
    if (ok) return true;
    for (int level = 1; level <= 2; ++level) {
        int mm = 1 << (level - 1), nn = 1 << (2 - level);
        double ws = 1.0 / (double)(nn * nn * nn);
        for (int r = 0; r < mm; ++r)
            for (int pp = 0; pp < mm; ++pp)
                for (int q = 0; q < mm; ++q) {
                    double tiles[8][V], means[V];
                    for (int t = 0; t < 8; ++t)
                        for (int v = 0; v < V; ++v) tiles[t][v] = 0.0;
                    for (int v = 0; v < V; ++v)
                        for (int kk = 0; kk < 2; ++kk)
                            for (int jj = 0; jj < 2; ++jj)
                                for (int ii = 0; ii < 2; ++ii)
                                    for (int kx = (2 * r + kk) * nn; kx < (2 * r + kk + 1) * nn; ++kx)
                                        for (int jx = (2 * pp + jj) * nn; jx < (2 * pp + jj + 1) * nn; ++jx)
                                            for (int ix = (2 * q + ii) * nn; ix < (2 * q + ii + 1) * nn; ++ix) {
                                                int t = ii + 2 * (jj + 2 * kk);
                                                tiles[t][v] = tiles[t][v] + ws * at(v, nidx(ix, jx, kx));
                                            }
                    bool tv = true;
                    for (int t = 0; t < 8; ++t) tv = tv && isvalid64(tiles[t], k);
                    if (tv) continue;
                    for (int v = 0; v < V; ++v) {
                        double s = 0.0;
                        for (int t = 0; t < 8; ++t) s = s + tiles[t][v];
                        means[v] = 0.125 * s;
                    }
                    double hiles[8][V];
                    for (int t = 0; t < 8; ++t)
                        for (int v = 0; v < V; ++v) hiles[t][v] = tiles[t][v] - means[v];
                    double squeeze = 1.0;
                    while (squeeze > 0.0) {
                        squeeze = fmax(0.0, squeeze - k.repair_decr);
                        for (int t = 0; t < 8; ++t)
                            for (int v = 0; v < V; ++v) tiles[t][v] = means[v] + squeeze * hiles[t][v];
                        bool tv2 = true;
                        for (int t = 0; t < 8; ++t) tv2 = tv2 && isvalid64(tiles[t], k);
                        if (tv2) break;
                    }
                    for (int v = 0; v < V; ++v)
                        for (int kx = 2 * r * nn; kx < (2 * r + 2) * nn; ++kx)
                            for (int jx = 2 * pp * nn; jx < (2 * pp + 2) * nn; ++jx)
                                for (int ix = 2 * q * nn; ix < (2 * q + 2) * nn; ++ix) {
                                    int p = nidx(ix, jx, kx);
                                    at(v, p) = means[v] + squeeze * (at(v, p) - means[v]);
                                }
                }
    }
    ok = true;
    for (int p = 0; p < NP; ++p) ok = ok && node_ok(p);
    return ok;
}


// The same repair done by the element's 16 threads together (a half-warp that calls it as a whole),
// for V variables and an admissibility test valid(q):
// no per-thread tile arrays, so it inlines without a call frame.  Level 1 squeezes the 8 octants
// (lanes 0..7, one octant each); level 2 squeezes the 8 nodes of each octant (lanes 0..7 and 8..15
// take one octant each, four rounds).  Each lane sums its tile in the serial routine's node order,
// the means run over the tiles in tile order, and all lanes of a block take the same squeeze steps.
template <int EPC, int V, typename Valid>
__device__ __forceinline__ bool repair_coop16(double* su, int el, int lane, double decr, Valid valid) {
    auto at = [&](int v, int p) -> double& { return su[(v * EPC + el) * NP + p]; };
    const unsigned half = threadIdx.x & 16;
#pragma unroll 1
    for (int level = 1; level <= 2; ++level) {
        const int rounds = level == 1 ? 1 : 4;
#pragma unroll 1
        for (int rd = 0; rd < rounds; ++rd) {
            const int grp = lane >> 3, t = lane & 7;
            const bool use = level == 2 || grp == 0;
            const unsigned gm = 0xffu << (half + 8 * grp);   // the 8 lanes of this block
            const int ii = t & 1, jj = (t >> 1) & 1, kk = t >> 2;
            // block origin (level 2: octant (q, pp, r) = blk bits) and the tile's node range
            const int blk = level == 1 ? 0 : 2 * rd + grp;
            const int q = blk & 1, pp = (blk >> 1) & 1, r = blk >> 2;
            const int nn = level == 1 ? 2 : 1;
            const int i0 = level == 1 ? 2 * ii : 2 * q + ii;
            const int j0 = level == 1 ? 2 * jj : 2 * pp + jj;
            const int k0 = level == 1 ? 2 * kk : 2 * r + kk;
            const double ws = level == 1 ? 0.125 : 1.0;
            double tile[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                double acc = 0.0;
                if (use)
                    for (int kx = k0; kx < k0 + nn; ++kx)
                        for (int jx = j0; jx < j0 + nn; ++jx)
                            for (int ix = i0; ix < i0 + nn; ++ix) acc = acc + ws * at(v, nidx(ix, jx, kx));
                tile[v] = acc;
            }
            if (!use) continue;
            const bool bad = !valid(tile);
            if (__ballot_sync(gm, bad) == 0u) continue;   // the block's tiles are admissible
            double mean[V], hile[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                double sum = 0.0;
#pragma unroll
                for (int tt = 0; tt < 8; ++tt) sum = sum + __shfl_sync(gm, tile[v], (int)(half + 8 * grp) + tt);
                mean[v] = 0.125 * sum;
                hile[v] = tile[v] - mean[v];
            }
            double squeeze = 1.0;
#pragma unroll 1
            while (squeeze > 0.0) {
                squeeze = fmax(0.0, squeeze - decr);
                double tv[V];
#pragma unroll
                for (int v = 0; v < V; ++v) tv[v] = mean[v] + squeeze * hile[v];
                if (__ballot_sync(gm, !valid(tv)) == 0u) break;
            }
            for (int kx = k0; kx < k0 + nn; ++kx)
                for (int jx = j0; jx < j0 + nn; ++jx)
                    for (int ix = i0; ix < i0 + nn; ++ix) {
                        const int p = nidx(ix, jx, kx);
#pragma unroll
                        for (int v = 0; v < V; ++v) at(v, p) = mean[v] + squeeze * (at(v, p) - mean[v]);
                    }
        }
        __syncwarp(0xffffu << half);
    }
    bool ok = true;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const int p = lane + 16 * m;
        double qv[V];
#pragma unroll
        for (int v = 0; v < V; ++v) qv[v] = at(v, p);
        ok = ok && valid(qv);
    }
    return __ballot_sync(0xffffu << half, !ok) == 0u;
}

template <int EPC>
__device__ __forceinline__ bool repair_elem16(double* su, int el, int lane, const OpConsts& k) {
    return repair_coop16<EPC, 5>(su, el, lane, k.repair_decr, [&](const double* q) { return isvalid64(q, k); });
}

template <int EPC>
__device__ __forceinline__ bool repair_elem16_mhd(double* su, int el, int lane, const OpConsts& k) {
    return repair_coop16<EPC, 9>(su, el, lane, k.repair_decr,
                                 [&](const double* q) { return m_isvalid<double>(q, k.kappa, k.mu0); });
}

// The same repair for the 9 GLM-MHD variables (MHD pressure in the admissibility check).
template <int EPC>
__device__ __noinline__ bool repair_elem_mhd(double* su, int el, const OpConsts& k) {
    constexpr int V = 9;
    auto at = [&](int v, int p) -> double& { return su[(v * EPC + el) * NP + p]; };
    auto node_ok = [&](int p) {
        double q[9];
        for (int v = 0; v < V; ++v) q[v] = at(v, p);
        return m_isvalid(q, k.kappa, k.mu0);
    };
    bool ok = true;
    for (int p = 0; p < NP; ++p) ok = ok && node_ok(p);
    if (ok) return true;
    for (int level = 1; level <= 2; ++level) {
        int mm = 1 << (level - 1), nn = 1 << (2 - level);
        double ws = 1.0 / (double)(nn * nn * nn);
        for (int r = 0; r < mm; ++r)
            for (int pp = 0; pp < mm; ++pp)
                for (int q = 0; q < mm; ++q) {
                    double tiles[8][V], means[V];
                    for (int t = 0; t < 8; ++t)
                        for (int v = 0; v < V; ++v) tiles[t][v] = 0.0;
                    for (int v = 0; v < V; ++v)
                        for (int kk = 0; kk < 2; ++kk)
                            for (int jj = 0; jj < 2; ++jj)
                                for (int ii = 0; ii < 2; ++ii)
                                    for (int kx = (2 * r + kk) * nn; kx < (2 * r + kk + 1) * nn; ++kx)
                                        for (int jx = (2 * pp + jj) * nn; jx < (2 * pp + jj + 1) * nn; ++jx)
                                            for (int ix = (2 * q + ii) * nn; ix < (2 * q + ii + 1) * nn; ++ix) {
                                                int t = ii + 2 * (jj + 2 * kk);
                                                tiles[t][v] = tiles[t][v] + ws * at(v, nidx(ix, jx, kx));
                                            }
                    bool tv = true;
                    for (int t = 0; t < 8; ++t) tv = tv && m_isvalid(tiles[t], k.kappa, k.mu0);
                    if (tv) continue;
                    for (int v = 0; v < V; ++v) {
                        double s = 0.0;
                        for (int t = 0; t < 8; ++t) s = s + tiles[t][v];
                        means[v] = 0.125 * s;
                    }
                    double hiles[8][V];
                    for (int t = 0; t < 8; ++t)
                        for (int v = 0; v < V; ++v) hiles[t][v] = tiles[t][v] - means[v];
                    double squeeze = 1.0;
                    while (squeeze > 0.0) {
                        squeeze = fmax(0.0, squeeze - k.repair_decr);
                        for (int t = 0; t < 8; ++t)
                            for (int v = 0; v < V; ++v) tiles[t][v] = means[v] + squeeze * hiles[t][v];
                        bool tv2 = true;
                        for (int t = 0; t < 8; ++t) tv2 = tv2 && m_isvalid(tiles[t], k.kappa, k.mu0);
                        if (tv2) break;
                    }
                    for (int v = 0; v < V; ++v)
                        for (int kx = 2 * r * nn; kx < (2 * r + 2) * nn; ++kx)
                            for (int jx = 2 * pp * nn; jx < (2 * pp + 2) * nn; ++jx)
                                for (int ix = 2 * q * nn; ix < (2 * q + 2) * nn; ++ix) {
                                    int p = nidx(ix, jx, kx);
                                    at(v, p) = means[v] + squeeze * (at(v, p) - means[v]);
                                }
                }
    }
    ok = true;
    for (int p = 0; p < NP; ++p) ok = ok && node_ok(p);
    return ok;
}


}  // namespace nemo
