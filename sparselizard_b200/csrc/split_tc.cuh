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
// |m c| <= 127^2 per q).  The epilogue recombines the levels.
//
// Level accumulators sit side by side in TMEM (level l at columns
// NE(l-2) .. NE(l-2)+NE-1 for an element tile of NE columns), and the column
// slices of one K step sit side by side in shared memory, so A slice a times
// the concatenation [c_1 | ... | c_k] (N = NE k <= 256) writes every pair
// (a, b) straight into level a+b's columns: for S = 7, 10 MMAs per K step
// (NE = 64) or 7 (NE = 32) instead of 28.
//
// Operands live in global memory already in the interleaved K-major layout
// that the UMMA "no swizzle" canonical form expects, blocked so that one K
// step of one tile is a single contiguous range (one bulk copy per operand):
//   A (rows of M):    [orient][ptile][kstep][slice][2][128][16 bytes]
//   B (columns of C): [unit][kstep][2][slice][NE][16 bytes]
// A core matrix (8 rows x 16 bytes) is 128 contiguous bytes; 8-row groups are
// SBO = 128 bytes apart, the two 16-byte K chunks of a step LBO bytes apart.
#pragma once

#include "engine_internal.h"

#include <cstdint>

namespace slgpu {

constexpr int kSplitM = 128;     // element-matrix entries per tile (TMEM lanes)
constexpr int kSplitKStep = 32;  // bytes of K per pipeline stage (one MMA K)
constexpr int kSplitMaxS = 7;    // slices per operand (levels 2..8)
constexpr int kSplitEpiWarps = 16;  // 4 per TMEM lane quarter, 16 columns each
constexpr int kSplitThreads = 64 + 32 * kSplitEpiWarps;
constexpr int kSplitABytes = 2 * kSplitM * 16;  // one slice of one K step of A

// Element-tile width NE (columns of one accumulator level) and what follows
// from it.  NE = 64: one accumulator (7 levels x 64 = 448 TMEM columns), the
// epilogue of a tile runs between its MMAs and the next tile's.  NE = 32: two
// accumulators (2 x 224 columns), the epilogue of one tile overlaps the MMAs
// of the next; A (the rows of M) is read twice as often per element.
template <int NE>
struct SplitShape {
    static constexpr int kUnits = 64 / NE;               // element tiles per 64-element tile
    static constexpr int kBufs = NE == 32 ? 2 : 1;       // TMEM accumulators
    static constexpr int kStages = NE == 32 ? 6 : 4;     // shared-memory pipeline depth
    static constexpr int kBBytes = 2 * NE * 16;          // one slice of one K step of B
    static constexpr int kGroup = 256 / NE;              // B slices per MMA (N <= 256)
};

// One group of a batched contraction launch.  Its work items are
// [w0, w0 + nwork) of the launch: item w0 + v is row tile v % ntp of element
// unit v / ntp.
struct SplitGroup {
    int P, Ppad, ntp, nk;   // entries, padded rows, row tiles, K steps
    int nrows, pad;         // rows of A computed (P, or the upper triangle)
    const int2* rowmap;     // [nrows]: the entry and its mirror; null: row r is entry r
    double* out2;           // null, or [nelem][P]: the transposed partner group's
                            // element matrices (entry rowmap[r].y from row r)
    const Tile* tiles;      // 64-element tiles; unit u = tile u / kUnits, part u % kUnits
    const int8_t* A;        // row slices
    const int8_t* B;        // column slices
    const int32_t* rowexp;  // [norient][Ppad]
    const int32_t* colexp;  // [ntiles][64]: exponent of each slot
    double* out;            // [nelem][P]
    int64_t w0, nwork;
};

// Groups of one launch (same S, L and NE), passed by value: every element
// group of a step runs in one persistent launch, whatever its entry count,
// Gauss points or element count.
constexpr int kSplitBatch = 24;
struct SplitParams {
    SplitGroup g[kSplitBatch];
    int ngroups;
    int64_t nwork;          // sum of the groups' work items
    unsigned int* error;    // set on a timed-out wait
    unsigned long long* next;  // work items handed out after each CTA's first; zero at launch
    int f32;                // out and out2 hold floats (FP32-level steps): same entry order
};

// Work items passed from a CTA's producer to its MMA and epilogue roles.
constexpr int kSplitItems = 8;

// Group of work item w, advanced from the group of the CTA's previous item
// (a CTA's items increase, so each role walks the groups once).
__device__ __forceinline__ int split_group_of(const SplitParams& p, int gi, int64_t w)
{
    while (gi + 1 < p.ngroups && w >= p.g[gi + 1].w0) gi++;
    return gi;
}

// Elements [e0, e0 + ne) and orientation of element unit u (ne <= 0: empty).
template <int NE>
__device__ __forceinline__ Tile split_unit(const Tile* tiles, int64_t u)
{
    Tile t = tiles[u / SplitShape<NE>::kUnits];
    const int part = (int)(u % SplitShape<NE>::kUnits) * NE;
    t.e0 += part;
    t.ne = min(t.ne - part, NE);
    return t;
}

// ---------------------------------------------------------------- slicing

// Row slices of M for one orientation: block per row p, threads over q.
// M[p][q] = T_t[o][i][g] * D_t[o][j][g] as in the FP64 contraction.
// Row r of A holds entry rowmap[r].x of M (entry r without a map); rows
// from nrows to Ppad are zero.
struct RowSliceParams {
    const double* tables;
    const int64_t* tab_off;
    const int32_t* term_tf;
    const int32_t* term_dof;
    const int2* rowmap;
    int nterms, ngp, ntf, ndof, norient, S, Qpad, Ppad, nrows;
    int8_t* slices;   // [orient][ptile][kstep][S][2][128][16]
    int32_t* rowexp;  // [norient][Ppad]
};

// M[pe][q] (pe < 0: zero).
__device__ __forceinline__ double m_entry(const RowSliceParams& p, int o, int pe, int q)
{
    const int Q = p.nterms * p.ngp;
    if (q >= Q || pe < 0)
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
    const int src = pe >= p.nrows ? -1 : p.rowmap != nullptr ? p.rowmap[pe].x : pe;
    __shared__ double red[256];
    double mx = 0;
    for (int q = threadIdx.x; q < p.Qpad; q += blockDim.x) mx = fmax(mx, fabs(m_entry(p, o, src, q)));
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
    const int ntp = p.Ppad / kSplitM, nk = p.Qpad / kSplitKStep;
    const int pt = pe / kSplitM, r = pe % kSplitM;
    for (int q = threadIdx.x; q < p.Qpad; q += blockDim.x) {
        int8_t sl[kSplitMaxS];
        split7(ldexp(m_entry(p, o, src, q), -ex), p.S, sl);
        const int ks = q / kSplitKStep, c = (q / 16) & 1;
        for (int s = 0; s < p.S; s++)
            p.slices[(((((int64_t)o * ntp + pt) * nk + ks) * p.S + s) * 2 + c) * (kSplitM * 16) + r * 16 + (q & 15)] = sl[s];
    }
}

// Column slices of C: thread per (64-element tile, slot); C[q][e] is read
// once, coalesced over the tile's consecutive elements, and 16-byte chunks
// are written coalesced over slots.  The exponent of each element (largest
// |C[q][e]| = f 2^ex, f in [0.5, 1)) comes from the coefficient kernel.
// Empty slots get zero slices.
struct ColSliceGroup {
    const double* C;  // [Q][nelem]
    const int32_t* elemexp;  // [nelem]; below -1100: the column is zero
    const Tile* tiles;
    int Q, Qpad;
    int64_t nelem, ntiles;
    int8_t* slices;   // [unit][kstep][2][S][NE][16]
    int32_t* colexp;  // [ntiles][64]
    int64_t t0;       // first tile of the group in the launch
};

struct ColSliceParams {
    ColSliceGroup g[kSplitBatch];
    int ngroups;
    int64_t ntiles;   // sum over the groups
};

template <int S, int NE>
__global__ void k_slice_cols(const __grid_constant__ ColSliceParams pb)
{
    const int64_t gt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t tg = gt / 64;
    const int slot = (int)(gt % 64);
    if (tg >= pb.ntiles)
        return;
    int gi = 0;
    while (gi + 1 < pb.ngroups && tg >= pb.g[gi + 1].t0) gi++;
    const ColSliceGroup& p = pb.g[gi];
    const int64_t t = tg - p.t0;
    const Tile tile = p.tiles[t];
    const bool valid = slot < tile.ne;
    const int64_t e = tile.e0 + slot;
    int ex = valid ? p.elemexp[e] : 0;
    if (ex < -1100)
        ex = 0;
    p.colexp[t * 64 + slot] = ex;
    const int nchunk = p.Qpad / 16;
    const int64_t unit = t * SplitShape<NE>::kUnits + slot / NE;
    uint4* out = reinterpret_cast<uint4*>(p.slices) + unit * (int64_t)nchunk * S * NE + slot % NE;
    const double* col = p.C + e;
    // |C| 2^(7S - ex) < 2^(7S): its integer part holds the S 7-bit slices
    // (the same digits repeated truncation of C 2^-ex by 128 produces).
    const bool fast = 7 * S - ex <= 1023;
    const double scale = fast ? __longlong_as_double((long long)(7 * S - ex + 1023) << 52) : 0.0;
    for (int c = 0; c < nchunk; c++) {
        double x[16];
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int q = c * 16 + k;
            x[k] = (valid && q < p.Q) ? col[(int64_t)q * p.nelem] : 0.0;
        }
        uint32_t w[S][4];
#pragma unroll
        for (int s = 0; s < S; s++)
#pragma unroll
            for (int k = 0; k < 4; k++) w[s][k] = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const double ax = fast ? fabs(x[k]) * scale : ldexp(fabs(x[k]), 7 * S - ex);
            const unsigned long long mag = __double2ull_rz(ax);
            const bool neg = x[k] < 0;
#pragma unroll
            for (int s = 0; s < S; s++) {
                const int d = (int)((mag >> (7 * (S - 1 - s))) & 127);
                w[s][k >> 2] |= (uint32_t)(uint8_t)(int8_t)(neg ? -d : d) << (8 * (k & 3));
            }
        }
        // chunk c of K step c/2 lands at [kstep][c&1][s][slot]: (c*S + s) * NE.
#pragma unroll
        for (int s = 0; s < S; s++) out[((int64_t)c * S + s) * NE] = make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
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

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait for the phase with the given parity.  Gives up (false) after
// 2^22 polls, or early once another role of the CTA has recorded a failure.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, const volatile int* failed)
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
        if ((it & 255) == 255 && *failed)
            return false;
    }
    return false;
}

// Contiguous global -> shared copy completing on an mbarrier (16-byte
// aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
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

// 16 consecutive 32-bit TMEM columns of this thread's lane (no wait).
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, int32_t* r)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
          "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 2^s as a double for a normal exponent, else ldexp (exact either way).
__device__ __forceinline__ double scale2(double x, int s)
{
    if (s >= -1022 && s <= 1023)
        return x * __longlong_as_double((long long)(s + 1023) << 52);
    return ldexp(x, s);
}

// Exact int64 -> double for |x| < 2^51 on the integer and FP64 pipes instead
// of the conversion unit (which the epilogue's two conversions per output
// saturate): x is added to the bit pattern of 1.5 * 2^52, whose mantissa ulp
// is 1, so the pattern encodes 1.5 * 2^52 + x exactly; subtracting 1.5 * 2^52
// is exact (both operands lie in [2^52, 2^53)).  The level sums meet the
// bound: level l holds at most l - 1 pair products of at most K * 127^2
// each, with K <= 16384, so |H| < 5.7e14 < 2^51 and |Lo| is smaller still.
__device__ __forceinline__ double i64_to_f64_exact(long long x)
{
    return __longlong_as_double(0x4338000000000000LL + x) - 0x1.8p52;
}

// ---------------------------------------------------------------- contraction

// Shared memory: pipeline stages, each one K step (32 bytes) of every A slice
// (128 rows) and every B slice (NE rows), plus barriers.
template <int NE>
struct SplitSmem {
    static constexpr int kSt = SplitShape<NE>::kStages;
    alignas(1024) int8_t A[kSt][kSplitMaxS * kSplitABytes];
    alignas(1024) int8_t B[kSt][kSplitMaxS * SplitShape<NE>::kBBytes];
    alignas(8) uint64_t full[kSt];
    uint64_t empty[kSt];
    uint64_t tmem_full[2], tmem_empty[2], drain;
    uint64_t item_full[kSplitItems], item_empty[kSplitItems];
    int64_t items[kSplitItems];
    uint32_t tmem;
    int failed;
};
template <int NE>
constexpr size_t split_smem_bytes() { return sizeof(SplitSmem<NE>) + 1024; }

// Persistent, warp-specialised kernel; one CTA per SM holds all 512 TMEM
// columns.  Work item w = (row tile w % ntp, element unit w / ntp).  Each
// CTA's first item is its index; later ones come from a global counter, so
// the items are taken in order and the CTAs working at the same time always
// hold neighbouring items: they share element units (B is read from L2 once
// per unit), and the 32-byte sectors that neighbouring row tiles' mirrored
// stores share are completed while they are still in L2.  (Handed out
// round-robin, the CTAs drift apart over a long launch.)  The producer skips
// empty units (past the end of a short tile) and passes each item to the MMA
// and epilogue roles through a ring of kSplitItems slots; -1 ends the CTA.
//   warp 0 (one thread): bulk copies of each K step into the stage ring;
//   warp 1 (one thread): MMAs; owns the TMEM allocation;
//   warps 2-17: epilogue; warp w reads TMEM lanes 32(w%4) .. 32(w%4)+31 and
//              16 of the NE columns.
// Barriers: full/empty per stage (copies -> MMA -> copies), tmem_full[b] (MMAs
// of a tile done -> epilogue) and tmem_empty[b] (epilogue has read
// accumulator b -> MMAs of the next tile using it).  Every wait is bounded: on
// timeout the CTA records the failure, the roles stop, outstanding copies and
// MMAs are waited for (bounded), the TMEM is freed and the CTA returns.
template <int S, int L, int NE>
__global__ void __launch_bounds__(kSplitThreads, 1) k_contract_split(const __grid_constant__ SplitParams p)
{
    static_assert(S <= kSplitMaxS && L - 1 <= S && L >= 6 && L <= 8, "level layout");
    using Sh = SplitShape<NE>;
    static_assert(Sh::kBufs == 1 ? (L - 1) * NE <= 512 : (L - 1) * NE <= 256, "accumulators fit the 512 TMEM columns");
    constexpr int kSt = Sh::kStages;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    SplitSmem<NE>& sm = *reinterpret_cast<SplitSmem<NE>*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr uint32_t kCols = 512;
    volatile int* failed = &sm.failed;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem)), "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < kSt; s++) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&sm.tmem_full[b], 1);
            mbar_init(&sm.tmem_empty[b], NE / 4);  // epilogue warps with columns
        }
        for (int k = 0; k < kSplitItems; k++) {
            mbar_init(&sm.item_full[k], 1);
            mbar_init(&sm.item_empty[k], 1 + NE / 4);  // MMA issuer and epilogue warps
        }
        mbar_init(&sm.drain, 1);
        sm.failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem;
    constexpr uint32_t kABytes = S * kSplitABytes, kBBytes = S * Sh::kBBytes;

    if (warp == 0 && lane == 0) {
        // ------------------------------------------------ producer
        int stage = 0;
        uint32_t phase = 0;
        uint32_t used = 0, last_parity = 0;  // per-stage bit sets
        bool ok = true;
        int gi = 0;
        int64_t w = blockIdx.x;
        for (uint32_t k = 0; ok; k++) {
            // The next non-empty work item, or -1 at the end.
            int64_t item = -1;
            while (w < p.nwork) {
                gi = split_group_of(p, gi, w);
                if (split_unit<NE>(p.g[gi].tiles, (w - p.g[gi].w0) / p.g[gi].ntp).ne > 0) {
                    item = w;
                    break;
                }
                w = (int64_t)atomicAdd(p.next, 1ull) + gridDim.x;
            }
            const int slot = (int)(k % kSplitItems);
            if (!mbar_wait(&sm.item_empty[slot], ((k / kSplitItems) & 1) ^ 1, failed)) {
                ok = false;
                break;
            }
            sm.items[slot] = item;
            mbar_arrive(&sm.item_full[slot]);
            if (item < 0)
                break;
            w = (int64_t)atomicAdd(p.next, 1ull) + gridDim.x;  // in flight during this item's copies
            const SplitGroup& G = p.g[gi];
            const int64_t v = item - G.w0;
            const int pt = (int)(v % G.ntp);
            const int64_t u = v / G.ntp;
            const Tile unit = split_unit<NE>(G.tiles, u);
            const int8_t* srcA = G.A + ((int64_t)unit.orient * G.ntp + pt) * G.nk * kABytes;
            const int8_t* srcB = G.B + u * G.nk * kBBytes;
            const int nk = G.nk;
            for (int ks = 0; ks < nk; ks++) {
                if (!mbar_wait(&sm.empty[stage], phase ^ 1, failed)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(&sm.full[stage], kABytes + kBBytes);
                bulk_load(sm.A[stage], srcA + (int64_t)ks * kABytes, kABytes, &sm.full[stage]);
                bulk_load(sm.B[stage], srcB + (int64_t)ks * kBBytes, kBBytes, &sm.full[stage]);
                used |= 1u << stage;
                last_parity = (last_parity & ~(1u << stage)) | (phase << stage);
                if (++stage == kSt) {
                    stage = 0;
                    phase ^= 1;
                }
            }
        }
        if (!ok) {
            *failed = 1;
            atomicOr(p.error, 1u);
        }
        // No copy may still be in flight when the CTA leaves.
        const int zero = 0;
        for (int s = 0; s < kSt; s++)
            if (used & (1u << s))
                if (!mbar_wait(&sm.full[s], (last_parity >> s) & 1, &zero))
                    atomicOr(p.error, 2u);
    } else if (warp == 1 && lane == 0) {
        // ------------------------------------------------ MMA issuer
        int stage = 0;
        uint32_t phase = 0;
        bool ok = true;
        int64_t i = 0;  // units processed by this CTA
        int gi = 0;
        for (uint32_t k = 0; ok; k++) {
            const int slot = (int)(k % kSplitItems);
            if (!mbar_wait(&sm.item_full[slot], (k / kSplitItems) & 1, failed)) {
                ok = false;
                break;
            }
            const int64_t w = sm.items[slot];
            mbar_arrive(&sm.item_empty[slot]);
            if (w < 0)
                break;
            gi = split_group_of(p, gi, w);
            const SplitGroup& G = p.g[gi];
            const int nk = G.nk;
            const int buf = (int)(i % Sh::kBufs);
            const int64_t use = i / Sh::kBufs;
            if (use > 0 && !mbar_wait(&sm.tmem_empty[buf], (uint32_t)((use - 1) & 1), failed)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t dbase = tmem + (uint32_t)(buf * 256);
            for (int ks = 0; ks < nk; ks++) {
                if (!mbar_wait(&sm.full[stage], phase, failed)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a_base = smem_u32(sm.A[stage]), b_base = smem_u32(sm.B[stage]);
#pragma unroll
                for (int a0 = 0; a0 < S; a0++) {
                    const int nbt = (S < L - 1 - a0) ? S : L - 1 - a0;  // b = 1 .. min(S, L - a)
                    const uint64_t ad = umma_desc(a_base + a0 * kSplitABytes, kSplitM * 16, 128);
#pragma unroll
                    for (int b0 = 0; b0 < nbt; b0 += Sh::kGroup) {
                        const int nb = (nbt - b0) < Sh::kGroup ? (nbt - b0) : Sh::kGroup;
                        const uint64_t bd = umma_desc(b_base + b0 * NE * 16, S * NE * 16, 128);
                        umma_i8(dbase + (uint32_t)(NE * (a0 + b0)), ad, bd, umma_idesc_i8(kSplitM, NE * nb),
                                (ks > 0 || a0 > 0) ? 1u : 0u);
                    }
                }
                umma_commit(&sm.empty[stage]);
                if (++stage == kSt) {
                    stage = 0;
                    phase ^= 1;
                }
            }
            if (!ok)
                break;
            umma_commit(&sm.tmem_full[buf]);
            i++;
        }
        if (!ok) {
            *failed = 1;
            atomicOr(p.error, 1u);
        }
        // Every MMA issued by this thread completes before the TMEM is freed.
        const int zero = 0;
        umma_commit(&sm.drain);
        if (!mbar_wait(&sm.drain, 0, &zero))
            atomicOr(p.error, 2u);
    } else if (warp >= 2) {
        // ------------------------------------------------ epilogue
        // Warp w reads TMEM lane quarter w % 4 and columns c0 .. c0+15 of
        // each level.  Only levels 2..5 (combined into H) and then 6..L are
        // held in registers before the accumulator is released; the rest of
        // the recombination and the stores overlap the next tile's MMAs.
        const int quarter = warp & 3;
        const int c0 = ((warp - 2) >> 2) * 16;
        const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
        int64_t i = 0;
        int gi = 0;
        for (uint32_t k = 0; c0 < NE; k++) {
            const int slot = (int)(k % kSplitItems);
            if (!mbar_wait(&sm.item_full[slot], (k / kSplitItems) & 1, failed)) {
                *failed = 1;
                atomicOr(p.error, 1u);
                break;
            }
            const int64_t w = sm.items[slot];
            __syncwarp();
            if (lane == 0)
                mbar_arrive(&sm.item_empty[slot]);
            if (w < 0)
                break;
            gi = split_group_of(p, gi, w);
            const SplitGroup& G = p.g[gi];
            const int64_t v = w - G.w0;
            const int pt = (int)(v % G.ntp);
            const int64_t u = v / G.ntp;
            const Tile unit = split_unit<NE>(G.tiles, u);
            const int buf = (int)(i % Sh::kBufs);
            if (!mbar_wait(&sm.tmem_full[buf], (uint32_t)((i / Sh::kBufs) & 1), failed)) {
                *failed = 1;
                atomicOr(p.error, 1u);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t col = lane_base + (uint32_t)(buf * 256 + c0);
            // V = 2^-35 (H + 2^-21 Lo): H = sum_{l<=5} r_l 2^(7(5-l)),
            // Lo = sum_{l>=6} r_l 2^(7(8-l)); both exact in int64.
            long long H[16];
            {
                int32_t r[4][16];
#pragma unroll
                for (int l = 0; l < 4; l++) tmem_ld16_nowait(col + (uint32_t)(l * NE), r[l]);
                tmem_ld_wait();
#pragma unroll
                for (int j = 0; j < 16; j++)
                    H[j] = (((long long)r[0][j] * 128 + r[1][j]) * 128 + r[2][j]) * 128 + r[3][j];
            }
            // Levels 6..L give Lo; the recombined value (exact up to the one
            // rounding of the fma) is formed before the stores' addresses are
            // live, so the store loop holds 16 doubles instead of the level
            // sums.
            double d[16];
            {
                int32_t t[L - 5][16];
#pragma unroll
                for (int l = 0; l < L - 5; l++) tmem_ld16_nowait(col + (uint32_t)((4 + l) * NE), t[l]);
                tmem_ld_wait();
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    long long lo = 0;
#pragma unroll
                    for (int l = 0; l < L - 5; l++) lo = lo * 128 + t[l][j];
                    lo <<= 7 * (8 - L);
                    d[j] = fma(i64_to_f64_exact(lo), 0x1p-21, i64_to_f64_exact(H[j]));
                }
            }
            // This warp's accumulators are in registers: release them.
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                mbar_arrive(&sm.tmem_empty[buf]);
            const int pe = pt * kSplitM + quarter * 32 + lane;
            if (pe < G.nrows) {
                const int rex = G.rowexp[(int64_t)unit.orient * G.Ppad + pe] - 35;
                const int32_t* ce = G.colexp + u * NE + c0;
                // Row pe is entry m.x and, for a symmetric group, also its
                // mirror m.y (the same entry on the diagonal); with a
                // transposed partner, entry (i, j) is also the partner's
                // entry (j, i).
                const int2 m = G.rowmap != nullptr ? G.rowmap[pe] : make_int2(pe, pe);
                const int P = G.P;
                const int64_t ebase = (int64_t)(unit.e0 + c0) * P;
                double* outp = G.out + ebase + m.x;
                double* outm = G.out2 != nullptr ? G.out2 + ebase + m.y : m.y != m.x ? G.out + ebase + m.y : nullptr;
                const int nj = min(16, unit.ne - c0);
#pragma unroll
                for (int j = 0; j < 16; j += 4) {
                    const int4 c4 = *reinterpret_cast<const int4*>(ce + j);
                    const int cx[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
                    for (int jj = 0; jj < 4; jj++) {
                        if (j + jj < nj) {
                            const double v = scale2(d[j + jj], rex + cx[jj]);
                            if (p.f32) {
                                // Entry k of a float matrix is float k of the same buffer.
                                const int64_t o = (int64_t)(j + jj) * P;
                                reinterpret_cast<float*>(G.out)[ebase + m.x + o] = (float)v;
                                if (outm != nullptr)
                                    reinterpret_cast<float*>(G.out2 != nullptr ? G.out2 : G.out)[ebase + m.y + o] = (float)v;
                            } else {
                                outp[(int64_t)(j + jj) * P] = v;
                                if (outm != nullptr)
                                    outm[(int64_t)(j + jj) * P] = v;
                            }
                        }
                    }
                }
            }
            i++;
        }
    }
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

}  // namespace slgpu
