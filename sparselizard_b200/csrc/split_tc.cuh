// Split-precision element contraction on the sm_100a tensor cores.
//
// V[e][p] = sum_q M[p][q] C[q][e] is evaluated with FP64 operands cut into
// 7-bit integer slices (Ozaki scheme):
//   M[p][q] = 2^E_p   sum_a m_a[p][q] 2^-7a      (row exponent E_p, a = 1..S)
//   C[q][e] = 2^F_e   sum_b c_b[q][e] 2^-7b      (column exponent F_e)
//   V[e][p] ~ 2^(E_p+F_e) sum_{a+b <= L} 2^-7(a+b) sum_q m_a c_b
// Each sum_q m_a c_b is an INT8 x INT8 product summed exactly in INT32 by
// tcgen05.mma (kind::i8); all pairs with the same level l = a+b accumulate
// in the same TMEM accumulator (still exact: at most S products of
// |m c| <= 127^2 per q).  The epilogue recombines the levels in FP64.
//
// Operands live in global memory in the interleaved K-major layout that the
// UMMA "no swizzle" canonical form expects, so that one 3D TMA box lands in
// shared memory ready for the descriptors:
//   slices[s][chunk][row][16 bytes],  chunk = q / 16.
// A core matrix (8 rows x 16 bytes) is 128 contiguous bytes; 8-row groups are
// SBO = 128 bytes apart and 16-byte K chunks LBO = rows*16 bytes apart.
#pragma once

#include "engine_internal.h"

#include <cstdint>

namespace slgpu {

constexpr int kSplitM = 128;     // element-matrix entries per tile (TMEM lanes)
constexpr int kSplitN = 64;      // elements per tile (= kTileE)
constexpr int kSplitKStage = 4;  // 16-byte K chunks per pipeline stage (64 bytes of K)
constexpr int kSplitMaxS = 7;    // slices per operand (levels 2..8 fit 448 TMEM columns)

struct SplitParams {
    int S;          // slices per operand
    int L;          // highest level kept (pairs with a + b <= L)
    int nchunkA;    // Qpad / 16
    int nkstage;    // Qpad / 128
    int P, Ppad, norient;
    int64_t nelem, Epad;
    const Tile* tiles;
    const int32_t* rowexp;  // [norient][Ppad]
    const int32_t* colexp;  // [nelem]
    double* out;            // [nelem][P]
    unsigned int* error;    // set on a timed-out wait
};

// ---------------------------------------------------------------- slicing

// Row slices of M for one orientation: block per row p, threads over q.
// M[p][q] = T_t[o][i][g] * D_t[o][j][g] as in the FP64 contraction.
struct RowSliceParams {
    const double* tables;
    const int64_t* tab_off;
    const int32_t* term_tf;
    const int32_t* term_dof;
    int nterms, ngp, ntf, ndof, norient, S, Qpad, Ppad;
    int8_t* slices;   // [S][norient][Qpad/16][Ppad][16]
    int32_t* rowexp;  // [norient][Ppad]
};

__device__ __forceinline__ double m_entry(const RowSliceParams& p, int o, int pe, int q)
{
    const int Q = p.nterms * p.ngp;
    if (q >= Q || pe >= p.ntf * p.ndof)
        return 0.0;
    const int t = q / p.ngp, g = q - t * p.ngp;
    const int i = pe / p.ndof, j = pe - i * p.ndof;
    const double tv = p.tables[p.tab_off[p.term_tf[t]] + ((int64_t)o * p.ntf + i) * p.ngp + g];
    const int dt = p.term_dof[t];
    const double dv = dt >= 0 ? p.tables[p.tab_off[dt] + ((int64_t)o * p.ndof + j) * p.ngp + g] : 1.0;
    return tv * dv;
}

// Splits x (|x| < 1 after scaling) into S signed 7-bit integers by repeated
// truncation; every step is exact in FP64.
__device__ __forceinline__ void split7(double x, int S, int8_t* out)
{
    for (int s = 0; s < S; s++) {
        const double y = x * 128.0;
        const double m = trunc(y);
        out[s] = (int8_t)m;
        x = y - m;
    }
}

__global__ void k_slice_rows(RowSliceParams p)
{
    const int pe = blockIdx.x, o = blockIdx.y;
    __shared__ double red[256];
    double mx = 0;
    for (int q = threadIdx.x; q < p.Qpad; q += blockDim.x) mx = fmax(mx, fabs(m_entry(p, o, pe, q)));
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    int ex = 0;
    if (red[0] > 0)
        frexp(red[0], &ex);  // red[0] = f * 2^ex, f in [0.5, 1)
    if (threadIdx.x == 0)
        p.rowexp[(int64_t)o * p.Ppad + pe] = ex;
    const int nchunk = p.Qpad / 16;
    for (int q = threadIdx.x; q < p.Qpad; q += blockDim.x) {
        int8_t sl[kSplitMaxS];
        split7(ldexp(m_entry(p, o, pe, q), -ex), p.S, sl);
        for (int s = 0; s < p.S; s++)
            p.slices[((((int64_t)s * p.norient + o) * nchunk + q / 16) * p.Ppad + pe) * 16 + (q & 15)] = sl[s];
    }
}

// Column slices of C: thread per element; C[q][e] read coalesced over e,
// 16-byte chunks written coalesced over e.
struct ColSliceParams {
    const double* C;  // [Q][nelem]
    int Q, Qpad, S;
    int64_t nelem, Epad;
    int8_t* slices;   // [S][Qpad/16][Epad][16]
    int32_t* colexp;  // [nelem]
};

template <int S>
__global__ void k_slice_cols(ColSliceParams p)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= p.nelem)
        return;
    double mx = 0;
    for (int q = 0; q < p.Q; q++) mx = fmax(mx, fabs(p.C[(int64_t)q * p.nelem + e]));
    int ex = 0;
    if (mx > 0)
        frexp(mx, &ex);
    p.colexp[e] = ex;
    const int nchunk = p.Qpad / 16;
    uint4* out = reinterpret_cast<uint4*>(p.slices);
    for (int c = 0; c < nchunk; c++) {
        uint32_t w[S][4];
#pragma unroll
        for (int s = 0; s < S; s++)
#pragma unroll
            for (int k = 0; k < 4; k++) w[s][k] = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int q = c * 16 + k;
            double x = q < p.Q ? ldexp(p.C[(int64_t)q * p.nelem + e], -ex) : 0.0;
#pragma unroll
            for (int s = 0; s < S; s++) {
                const double y = x * 128.0;
                const double m = trunc(y);
                w[s][k >> 2] |= (uint32_t)(uint8_t)(int8_t)m << (8 * (k & 3));
                x = y - m;
            }
        }
#pragma unroll
        for (int s = 0; s < S; s++) out[((int64_t)s * nchunk + c) * p.Epad + e] = make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
    }
}

// ---------------------------------------------------------------- PTX helpers

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Bounded wait for the phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < (1u << 22); it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done)
            return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

// UMMA shared-memory descriptor, K-major, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor for kind::i8: S32 accumulate, signed A and B,
// both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t umma_idesc_i8(int M, int N)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
          "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ---------------------------------------------------------------- contraction

// Shared memory: two pipeline stages; each holds every A slice (128 rows x
// 64 bytes = 8 KB) and every B slice (64 rows x 64 bytes = 4 KB) of one
// 64-byte K stage, plus barriers and the TMEM address.
struct SplitSmem {
    alignas(1024) int8_t A[2][kSplitMaxS][kSplitKStage][kSplitM][16];
    alignas(1024) int8_t B[2][kSplitMaxS][kSplitKStage][kSplitN][16];
    alignas(8) uint64_t full[2];
    uint64_t mma_done[2];
    uint32_t tmem;
    int failed;
    int colexp[kSplitN];
};
constexpr size_t kSplitSmemBytes = sizeof(SplitSmem) + 1024;

// One CTA = one (128 entries x 64 elements) tile; 128 threads (4 warps).
// Thread 0 issues TMA and MMA; warp 0 owns the TMEM allocation; all warps
// run the epilogue (warp w reads TMEM lanes 32w..32w+31).
//
// Pipeline: stage ks (64 bytes of K) loads all S A slices and S B slices into
// buffer ks&1 under one barrier; stage ks+1 is loaded while the MMAs of stage
// ks run, once the MMAs that last read its buffer (stage ks-1) have completed
// (tcgen05.commit on mma_done[buffer]).  Every wait is bounded: on timeout the
// CTA records the failure, skips its epilogue, frees its TMEM and returns.
__global__ void __launch_bounds__(128, 1) k_contract_split(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                                                           SplitParams p)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    SplitSmem& sm = *reinterpret_cast<SplitSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5;
    const Tile tile = p.tiles[blockIdx.y];
    const int p0 = blockIdx.x * kSplitM;
    const uint32_t ncols = 512;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem)), "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&sm.full[0], 1);
        mbar_init(&sm.full[1], 1);
        mbar_init(&sm.mma_done[0], 1);
        mbar_init(&sm.mma_done[1], 1);
        sm.failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (tid < kSplitN) {
        const int64_t e = tile.e0 + tid;
        sm.colexp[tid] = (tid < tile.ne && e < p.nelem) ? p.colexp[e] : 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem;

    if (tid == 0) {
        const uint32_t idesc = umma_idesc_i8(kSplitM, kSplitN);
        const uint32_t lboA = kSplitM * 16, lboB = kSplitN * 16, sbo = 128;
        const int amax = min(p.S, p.L - 1);
        const uint32_t stage_bytes = (uint32_t)(p.S * kSplitKStage * (kSplitM + kSplitN) * 16);
        uint32_t ph_full[2] = {0, 0}, ph_mma[2] = {0, 0};
        bool pending[2] = {false, false};
        bool ok = true;
        auto issue = [&](int ks) {
            const int buf = ks & 1;
            mbar_expect_tx(&sm.full[buf], stage_bytes);
            for (int s = 0; s < p.S; s++) {
                tma_load_3d(&sm.A[buf][s][0][0][0], &mapA, &sm.full[buf], 0, p0,
                            (s * p.norient + tile.orient) * p.nchunkA + ks * kSplitKStage);
                tma_load_3d(&sm.B[buf][s][0][0][0], &mapB, &sm.full[buf], 0, tile.e0, s * p.nchunkA + ks * kSplitKStage);
            }
        };
        auto drain = [&](int i) {
            if (pending[i] && ok) {
                ok = mbar_wait(&sm.mma_done[i], ph_mma[i]);
                ph_mma[i] ^= 1;
                pending[i] = false;
            }
        };
        issue(0);
        for (int ks = 0; ks < p.nkstage && ok; ks++) {
            const int buf = ks & 1;
            if (ks + 1 < p.nkstage) {
                drain(buf ^ 1);
                if (!ok)
                    break;
                issue(ks + 1);
            }
            ok = mbar_wait(&sm.full[buf], ph_full[buf]);
            ph_full[buf] ^= 1;
            if (!ok)
                break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int a = 1; a <= amax; a++) {
                for (int b = 1; b <= p.S && a + b <= p.L; b++) {
                    const int level = a + b;
                    const uint32_t dcol = tmem + (uint32_t)((level - 2) * kSplitN);
                    const int afirst = max(1, level - p.S);
                    for (int k = 0; k < kSplitKStage / 2; k++) {
                        const uint64_t ad = umma_desc(smem_u32(&sm.A[buf][a - 1][2 * k][0][0]), lboA, sbo);
                        const uint64_t bd = umma_desc(smem_u32(&sm.B[buf][b - 1][2 * k][0][0]), lboB, sbo);
                        const uint32_t acc = (ks == 0 && k == 0 && a == afirst) ? 0u : 1u;
                        umma_i8(dcol, ad, bd, idesc, acc);
                    }
                }
            }
            umma_commit(&sm.mma_done[buf]);
            pending[buf] = true;
        }
        drain(0);
        drain(1);
        if (!ok) {
            sm.failed = 1;
            atomicOr(p.error, 1u);
        }
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (!sm.failed) {
        // Epilogue: thread t owns TMEM lane (row) t = entry p0 + t.
        const int pe = p0 + tid;
        const int rex = p.rowexp[(int64_t)tile.orient * p.Ppad + min(pe, p.Ppad - 1)];
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
        for (int c0 = 0; c0 < kSplitN; c0 += 16) {
            double v[16];
#pragma unroll
            for (int i = 0; i < 16; i++) v[i] = 0.0;
            for (int level = p.L; level >= 2; level--) {
                uint32_t r[16];
                tmem_ld16(tmem + lane_base + (uint32_t)((level - 2) * kSplitN + c0), r);
                const double sc = ldexp(1.0, -7 * level);
#pragma unroll
                for (int i = 0; i < 16; i++) v[i] += (double)(int32_t)r[i] * sc;
            }
            if (pe < p.P) {
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const int ee = c0 + i;
                    if (ee < tile.ne)
                        p.out[(int64_t)(tile.e0 + ee) * p.P + pe] = ldexp(v[i], rex + sm.colexp[ee]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

}  // namespace slgpu
