// CSR values by persistent warps that stream their rows' incidences through
// a ring of shared-memory entries filled by asynchronous copies.
//
// The value phase of rawmat::process (duplicate summation in insertion order,
// src/formulation/rawmat.cpp:67-125 and 221-299) is a gather of element-matrix
// rows: every incidence of a CSR row is a contiguous run of `width` element
// values (element-major buffer) plus the run of their 16-bit row slots.  The
// one-row-per-warp kernel (k_row_values) issues those gathers a few at a time
// and waits on each batch, so for short rows of long incidences it is bound
// by DRAM latency.  Here a warp owns chunks of consecutive rows (chunk c,
// c + W, c + 2W, ... for warp c of W) and keeps R incidences of its stream in
// flight: entry k % R of the ring receives incidence k's values and slots
// (16-byte aligned supersets of the two runs, copied 16 bytes per lane with
// cp.async, one commit group per incidence) while incidences k+1..k+R-1 are
// still arriving.  The additions are the same as k_row_values', in the same
// order (incidences in order; lane j adds column j; serial incidences by lane
// 0 in column order), so the results are bit-identical.
#pragma once

#include "engine_internal.h"

#include <cstdint>

namespace slgpu {

struct RowStreamParams {
    RowParams r;
    int vw, sw;           // ring entry capacity: doubles of values, int16 of slots
    int lpad;             // row buffer doubles per warp (>= longest row, even)
    int rows_per_chunk;   // <= 31 (a chunk's row bounds are held one per lane)
    int64_t nchunks;
    int64_t nwarps;       // warps in the grid (the chunk stride)
};

struct RowStreamMeta {
    double mult;
    int32_t info;  // width | serial << 16 | value shift << 17 | slot shift << 18
    int32_t pad;
};

constexpr int kStreamWarps = 8;

__host__ __device__ constexpr size_t row_stream_warp_bytes(int ring, int vw, int sw, int lpad)
{
    return (size_t)ring * 16 + (size_t)ring * vw * 8 + (size_t)ring * sw * 2 + (size_t)lpad * 8;
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(reinterpret_cast<uint64_t>(src))
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int R>
__global__ void __launch_bounds__(kStreamWarps * 32) k_row_stream(RowStreamParams sp)
{
    extern __shared__ __align__(16) unsigned char stream_smem[];
    const RowParams& p = sp.r;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t gw = (int64_t)blockIdx.x * kStreamWarps + wib;
    if (gw >= sp.nwarps)
        return;
    unsigned char* base = stream_smem + (size_t)wib * row_stream_warp_bytes(R, sp.vw, sp.sw, sp.lpad);
    RowStreamMeta* meta = reinterpret_cast<RowStreamMeta*>(base);
    double* rv = reinterpret_cast<double*>(base + (size_t)R * 16);
    int16_t* rs = reinterpret_cast<int16_t*>(base + (size_t)R * 16 + (size_t)R * sp.vw * 8);
    double* buf = reinterpret_cast<double*>(base + (size_t)R * 16 + (size_t)R * sp.vw * 8 + (size_t)R * sp.sw * 2);

    // ---- producer state: next incidence to fetch (pk) within chunk pc
    int64_t pc = gw;
    uint32_t pk = 0, pk_end = 0;
    auto chunk_incidences = [&](int64_t c, uint32_t& a, uint32_t& b) {
        const int64_t r0 = c * sp.rows_per_chunk;
        const int64_t r1 = min(r0 + sp.rows_per_chunk, p.nrows);
        a = p.inc_ptr[r0];
        b = p.inc_ptr[r1];
    };
    bool pdone = pc >= sp.nchunks;
    if (!pdone)
        chunk_incidences(pc, pk, pk_end);
    // Decoded headers of incidences hb .. hb+31 (lane l holds hb + l).
    uint32_t hb = 0;
    bool hvalid = false;
    long long h_voff = 0, h_coo = 0;
    double h_mult = 0.0;
    int h_info = 0;
    uint32_t issued = 0, consumed = 0;

    // Warp-collective: fetches the next incidence of the stream into entry
    // issued % R (every lane commits one group, possibly empty).  Returns
    // false at the end of the stream.
    auto issue_next = [&]() -> bool {
        while (!pdone && pk == pk_end) {
            pc += sp.nwarps;
            hvalid = false;
            if (pc >= sp.nchunks) {
                pdone = true;
                break;
            }
            chunk_incidences(pc, pk, pk_end);
        }
        if (pdone)
            return false;
        if (!hvalid || pk >= hb + 32) {
            hb = pk;
            hvalid = true;
            const uint32_t k = hb + lane;
            if (k < pk_end) {
                const unsigned long long pkd = p.inc[k];
                const RowSeg sg = p.segs[(pkd >> 40) & ((1ull << 23) - 1)];
                h_coo = (long long)(pkd & ((1ull << 40) - 1));
                h_voff = sg.val_base + (h_coo - sg.coo_base);
                h_mult = sg.mult;
                h_info = sg.width | ((pkd >> 63) != 0 ? (1 << 16) : 0);
            }
        }
        const int src = (int)(pk - hb);
        const long long vo = __shfl_sync(0xffffffffu, h_voff, src);
        const long long co = __shfl_sync(0xffffffffu, h_coo, src);
        const double m = __shfl_sync(0xffffffffu, h_mult, src);
        const int inf = __shfl_sync(0xffffffffu, h_info, src);
        const uint32_t e = issued % (uint32_t)R;
        const int width = inf & 0xffff;
        const uintptr_t v0 = reinterpret_cast<uintptr_t>(p.vals + vo);
        const uintptr_t va = v0 & ~uintptr_t(15), vb = (v0 + (uintptr_t)width * 8 + 15) & ~uintptr_t(15);
        const uintptr_t s0 = reinterpret_cast<uintptr_t>(p.slotmap + co);
        const uintptr_t sa = s0 & ~uintptr_t(15), sb = (s0 + (uintptr_t)width * 2 + 15) & ~uintptr_t(15);
        const int nv = (int)((vb - va) >> 4), ns = (int)((sb - sa) >> 4);
        unsigned char* dv = reinterpret_cast<unsigned char*>(rv + (size_t)e * sp.vw);
        unsigned char* ds = reinterpret_cast<unsigned char*>(rs + (size_t)e * sp.sw);
        for (int i = lane; i < nv + ns; i += 32) {
            if (i < nv)
                cp_async16(dv + 16 * i, reinterpret_cast<const void*>(va + 16 * (uintptr_t)i));
            else
                cp_async16(ds + 16 * (i - nv), reinterpret_cast<const void*>(sa + 16 * (uintptr_t)(i - nv)));
        }
        cp_async_commit();
        if (lane == 0) {
            meta[e].mult = m;
            meta[e].info = inf | (int)(((v0 - va) >> 3) << 17) | (int)(((s0 - sa) >> 1) << 18);
        }
        pk++;
        issued++;
        return true;
    };

    for (int i = 0; i < R; i++)
        if (!issue_next())
            break;

    for (int64_t cc = gw; cc < sp.nchunks; cc += sp.nwarps) {
        const int64_t r0 = cc * sp.rows_per_chunk;
        const int nr = (int)min((int64_t)sp.rows_per_chunk, p.nrows - r0);
        // Row bounds of the chunk, one row per lane (lane nr: the end).
        uint32_t a_lo = 0, d_lo = 0, i_lo = 0;
        if (lane <= nr) {
            a_lo = p.Arows[r0 + lane];
            d_lo = p.Drows ? p.Drows[r0 + lane] : 0u;
            i_lo = p.inc_ptr[r0 + lane];
        }
        for (int rr = 0; rr < nr; rr++) {
            const uint32_t a0 = __shfl_sync(0xffffffffu, a_lo, rr), a1 = __shfl_sync(0xffffffffu, a_lo, rr + 1);
            const uint32_t d0 = __shfl_sync(0xffffffffu, d_lo, rr), d1 = __shfl_sync(0xffffffffu, d_lo, rr + 1);
            const uint32_t k0 = __shfl_sync(0xffffffffu, i_lo, rr), k1 = __shfl_sync(0xffffffffu, i_lo, rr + 1);
            const int la = (int)(a1 - a0), L = la + (int)(d1 - d0);
            for (int s = lane; s < L; s += 32) buf[s] = 0.0;
            __syncwarp();
            for (uint32_t k = k0; k < k1; k++) {
                const uint32_t e = consumed % (uint32_t)R;
                // The oldest of the groups in flight is incidence `consumed`.
                if (issued - consumed >= (uint32_t)R)
                    cp_async_wait<R - 1>();
                else
                    cp_async_wait<0>();
                __syncwarp();
                const double m = meta[e].mult;
                const int inf = meta[e].info;
                const int width = inf & 0xffff;
                const double* v = rv + (size_t)e * sp.vw + ((inf >> 17) & 1);
                const int16_t* sl = rs + (size_t)e * sp.sw + ((inf >> 18) & 7);
                if (inf & (1 << 16)) {
                    if (lane == 0)
                        for (int j = 0; j < width; j++) {
                            const int s = sl[j];
                            if (s >= 0)
                                buf[s] = fma(v[j], m, buf[s]);
                        }
                } else {
                    for (int j = lane; j < width; j += 32) {
                        const int s = sl[j];
                        if (s >= 0)
                            buf[s] = fma(v[j], m, buf[s]);
                    }
                }
                __syncwarp();
                consumed++;
                issue_next();
            }
            const int64_t r = r0 + rr;
            if (p.dense != nullptr) {
                if (lane == 0)
                    p.dense[r] = L > 0 ? -buf[0] : 0.0;
            } else {
                for (int s = lane; s < L; s += 32) {
                    if (s < la)
                        p.Avals[a0 + s] = buf[s];
                    else
                        p.Dvals[d0 + (s - la)] = buf[s];
                }
            }
            __syncwarp();
        }
    }
}

}  // namespace slgpu
