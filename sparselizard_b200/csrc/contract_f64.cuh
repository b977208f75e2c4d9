// FP64 element-matrix contraction on the FP64 tensor cores (DMMA).
//
// The element matrices of one group are K[e][p] = sum_q M[p][q] C[q][e]
// (src/formulation/contribution.cpp:200-210 with densemat::multiply,
// src/densemat.cpp:228-310), M[(i,j)][(t,g)] = T_t[o][i][g] * D_t[o][j][g].
// Here the product is computed as K^T = C^T M^T, element rows by entry
// columns, with mma.sync.m16n8k8.f64 (FP64 operands, FP64 accumulation; the
// FP64 tensor path of sm_100a -- tcgen05 has no FP64 kind).
//
//  * M^T of every orientation is built once per group and form
//    (k_build_mt, [norient][Qpad][rpad], zero outside Q x nrows) and stays
//    resident; its columns are the group's computed rows: every entry, or,
//    for the mirrored forms, the rows of a row map (upper triangle of a
//    symmetric group, or every entry of a group whose transposed partner is
//    written by the same launch).
//  * A block computes 64 elements x BP rows (BP = 128 or 64, picked per group
//    shape by timing); 8 warps of 32 x BP/4 (2 x BP/32 MMA tiles of 16 x 8).
//    K advances 16 at a time through a 3-stage cp.async ring of C^T and M^T
//    tiles in shared memory (rows padded to 68 and BP + 4 doubles so that the
//    fragment loads of a half-warp hit distinct banks).
//  * Fragments are stored straight to global memory: each value at its
//    entry, and for the mirrored forms also at its mirror entry (same matrix
//    or the partner's).
#pragma once

#include "engine_internal.h"

#include <cstdint>

namespace slgpu {

constexpr int kMmaBE = 64;    // elements per block
constexpr int kMmaBPMax = 128;  // most rows (entries) per block; M^T rows are padded to it
constexpr int kMmaBQ = 16;    // (term, Gauss point) pairs per stage
constexpr int kMmaStages = 3;
constexpr int kMmaCS = kMmaBE + 4;  // C^T tile row stride (doubles)
template <int BP>
struct MmaShape {
    static constexpr int MS = BP + 4;  // M^T tile row stride (doubles)
    static constexpr int StageDoubles = kMmaBQ * (kMmaCS + MS);
    static constexpr size_t Smem = (size_t)kMmaStages * StageDoubles * sizeof(double);
    static constexpr int NT = BP / 32;  // 8-row MMA tiles per warp
};

struct BuildMtParams {
    const double* tables;
    const int64_t* tab_off;
    const int32_t* term_tf;
    const int32_t* term_dof;
    const int2* rowmap;  // nullptr: row r is entry r
    int nterms, ngp, ntf, ndof, norient, nrows, Qpad, rpad;
    double* Mt;          // [norient][Qpad][rpad]
};

// M^T[o][q][r] = T_t[o][i][g] * D_t[o][j][g] for q = t*ngp + g < Q and
// r < nrows (entry p = i*ndof + j of row r), 0 elsewhere.
__global__ void k_build_mt(BuildMtParams p)
{
    const int64_t n = (int64_t)p.norient * p.Qpad * p.rpad;
    const int Q = p.nterms * p.ngp;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(idx % p.rpad);
        const int64_t oq = idx / p.rpad;
        const int q = (int)(oq % p.Qpad);
        const int o = (int)(oq / p.Qpad);
        double v = 0.0;
        if (q < Q && r < p.nrows) {
            const int pe = p.rowmap != nullptr ? p.rowmap[r].x : r;
            const int t = q / p.ngp, g = q - t * p.ngp;
            const int i = pe / p.ndof, j = pe - i * p.ndof;
            const double tv = p.tables[p.tab_off[p.term_tf[t]] + ((int64_t)o * p.ntf + i) * p.ngp + g];
            const int dt = p.term_dof[t];
            const double dv = dt >= 0 ? p.tables[p.tab_off[dt] + ((int64_t)o * p.ndof + j) * p.ngp + g] : 1.0;
            v = tv * dv;
        }
        p.Mt[idx] = v;
    }
}

struct MmaParams {
    const double* Mt;    // [norient][Qpad][rpad]
    const double* C;     // [Q][nelem]
    const Tile* tiles;   // orientation-uniform element runs of at most 64
    const int2* rowmap;  // nullptr: row r is entry r
    int Q, Qpad, rpad, nrows, P;
    int nrt;             // row tiles (rpad / BP)
    int mirror;          // 0 none, 1 mirror entry of the same matrix, 2 mirror entry of out2
    int64_t nelem;
    double* out;         // [nelem][P]
    double* out2;        // partner's [nelem][P] (mirror == 2)
};

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
}

__device__ __forceinline__ void cp_async16(double* dst, const double* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void dmma_16x8x8(double (&c)[4], const double (&a)[4], const double (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

template <int BP>
__global__ void __launch_bounds__(256, 2) k_contract_f64mma(MmaParams p)
{
    using Sh = MmaShape<BP>;
    constexpr int NT = Sh::NT;
    extern __shared__ double sm_mma[];
    const int rt = (int)(blockIdx.x % p.nrt);
    const Tile tile = p.tiles[blockIdx.x / p.nrt];
    const int r0 = rt * BP;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const int we = warp >> 2, wr = warp & 3;  // warp's 32 elements and BP/4 rows
    const double* Mt = p.Mt + (int64_t)tile.orient * p.Qpad * p.rpad + r0;
    const int nchunks = p.Qpad / kMmaBQ;

    auto stage_C = [&](int s) { return sm_mma + (int64_t)s * Sh::StageDoubles; };
    auto stage_M = [&](int s) { return sm_mma + (int64_t)s * Sh::StageDoubles + kMmaBQ * kMmaCS; };
    auto load = [&](int chunk, int s) {
        const int q0 = chunk * kMmaBQ;
        double* Cs = stage_C(s);
        double* Ms = stage_M(s);
#pragma unroll
        for (int k = 0; k < (kMmaBQ * kMmaBE) / 256; k++) {
            const int idx = tid + 256 * k;
            const int row = idx / kMmaBE, col = idx % kMmaBE;
            const bool valid = q0 + row < p.Q && col < tile.ne;
            const double* src = valid ? p.C + (int64_t)(q0 + row) * p.nelem + tile.e0 + col : p.C;
            cp_async8(Cs + row * kMmaCS + col, src, valid);
        }
#pragma unroll
        for (int k = 0; k < (kMmaBQ * BP) / (2 * 256); k++) {
            const int idx = tid + 256 * k;
            const int row = idx / (BP / 2), c2 = idx % (BP / 2);
            cp_async16(Ms + row * Sh::MS + 2 * c2, Mt + (int64_t)(q0 + row) * p.rpad + 2 * c2);
        }
    };

    double acc[2][NT][4];
#pragma unroll
    for (int m = 0; m < 2; m++)
#pragma unroll
        for (int n = 0; n < NT; n++)
#pragma unroll
            for (int k = 0; k < 4; k++) acc[m][n][k] = 0.0;

    // Prologue: the first kMmaStages - 1 chunks in flight (one commit group each).
#pragma unroll
    for (int s = 0; s < kMmaStages - 1; s++) {
        if (s < nchunks)
            load(s, s);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    for (int c = 0; c < nchunks; c++) {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(kMmaStages - 2) : "memory");
        __syncthreads();  // chunk c landed for every thread; chunk c-1's stage is free
        const int nxt = c + kMmaStages - 1;
        if (nxt < nchunks)
            load(nxt, nxt % kMmaStages);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        const double* Cs = stage_C(c % kMmaStages);
        const double* Ms = stage_M(c % kMmaStages);
#pragma unroll
        for (int ks = 0; ks < kMmaBQ; ks += 8) {
            double a[2][4], b[NT][2];
#pragma unroll
            for (int m = 0; m < 2; m++) {
                const int e = we * 32 + m * 16 + gid;
                a[m][0] = Cs[(ks + tig) * kMmaCS + e];
                a[m][1] = Cs[(ks + tig) * kMmaCS + e + 8];
                a[m][2] = Cs[(ks + tig + 4) * kMmaCS + e];
                a[m][3] = Cs[(ks + tig + 4) * kMmaCS + e + 8];
            }
#pragma unroll
            for (int n = 0; n < NT; n++) {
                const int r = wr * (8 * NT) + n * 8 + gid;
                b[n][0] = Ms[(ks + tig) * Sh::MS + r];
                b[n][1] = Ms[(ks + tig + 4) * Sh::MS + r];
            }
#pragma unroll
            for (int m = 0; m < 2; m++)
#pragma unroll
                for (int n = 0; n < NT; n++) dmma_16x8x8(acc[m][n], a[m], b[n]);
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");

    // Fragment (m, n): rows e = base + gid (+8), columns r = base + 2 tig (+1).
#pragma unroll
    for (int m = 0; m < 2; m++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int e = we * 32 + m * 16 + gid + 8 * h;
            if (e >= tile.ne)
                continue;
            double* orow = p.out + (int64_t)(tile.e0 + e) * p.P;
            double* mrow = (p.mirror == 2 ? p.out2 : p.out) + (int64_t)(tile.e0 + e) * p.P;
#pragma unroll
            for (int n = 0; n < NT; n++)
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    const int r = r0 + wr * (8 * NT) + n * 8 + 2 * tig + k;
                    if (r >= p.nrows)
                        continue;
                    const double v = acc[m][n][2 * h + k];
                    if (p.rowmap == nullptr) {
                        orow[r] = v;
                    } else {
                        const int2 mp = p.rowmap[r];
                        orow[mp.x] = v;
                        if (p.mirror == 2 || mp.y != mp.x)
                            mrow[mp.y] = v;
                    }
                }
        }
}

}  // namespace slgpu
