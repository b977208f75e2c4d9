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
    int lpad;             // row buffer doubles per warp (>= longest row, even)
    int rows_per_chunk;   // <= 31 (a chunk's row bounds are held one per lane)
    int64_t nchunks;
    int64_t nwarps;       // warps in the grid (the chunk stride)
};

// Decoded incidence: where its values and slots start (16-byte units from
// the value buffer and the slot map) and how to copy and add them.
struct RowStreamDesc {
    double mult;
    uint32_t va16, sa16;  // first 16-byte unit of the values / slots superset
    uint32_t info;        // width | serial << 7 | value shift << 8 | slot shift << 9 | nv << 12 | ns << 18
    uint32_t pad;
    uint64_t pad2;
};
constexpr int kStreamDescs = 64;  // per warp: decoded incidences (>= ring + 32, a power of two)
constexpr int kStreamWarps = 4;

// Ring shapes by incidence width: R entries, 2^VSH bytes of values and 2^SSH
// bytes of slots per entry (at least 8 width + 16 and 2 width + 30: the
// 16-byte aligned supersets).  Narrow (width <= 30): one copy and one
// addition per lane and incidence.  Wide (width <= 62): loops over the lanes.
struct StreamNarrow {
    static constexpr int R = 16, VSH = 8, SSH = 7, WMAX = 30;
    static constexpr bool kNarrow = true;
};
struct StreamWide {
    static constexpr int R = 8, VSH = 9, SSH = 8, WMAX = 62;
    static constexpr bool kNarrow = false;
};

__host__ __device__ constexpr size_t row_stream_warp_bytes(int ring, int vsh, int ssh, int lpad)
{
    return (size_t)kStreamDescs * sizeof(RowStreamDesc) + ((size_t)ring << vsh) + ((size_t)ring << ssh) + (size_t)lpad * 8;
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

template <class Shape>
__global__ void __launch_bounds__(kStreamWarps * 32) k_row_stream(RowStreamParams sp)
{
    constexpr int R = Shape::R, VSH = Shape::VSH, SSH = Shape::SSH;
    static_assert(kStreamDescs >= R + 32 && (kStreamDescs & (kStreamDescs - 1)) == 0, "descriptor ring");
    static_assert((R & (R - 1)) == 0, "ring size a power of two");
    extern __shared__ __align__(16) unsigned char stream_smem[];
    const RowParams& p = sp.r;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t gw = (int64_t)blockIdx.x * kStreamWarps + wib;
    if (gw >= sp.nwarps)
        return;
    unsigned char* base = stream_smem + (size_t)wib * row_stream_warp_bytes(R, VSH, SSH, sp.lpad);
    RowStreamDesc* desc = reinterpret_cast<RowStreamDesc*>(base);
    unsigned char* rv = base + (size_t)kStreamDescs * sizeof(RowStreamDesc);
    unsigned char* rs = rv + ((size_t)R << VSH);
    double* buf = reinterpret_cast<double*>(rs + ((size_t)R << SSH));
    const unsigned char* vals16 = reinterpret_cast<const unsigned char*>(p.vals);
    const unsigned char* slots16 = reinterpret_cast<const unsigned char*>(p.slotmap);
    // The row buffer is kept zero between rows (the write-back clears it).
    for (int s = lane; s < sp.lpad; s += 32) buf[s] = 0.0;

    // ---- producer: decodes incidences 32 at a time (pk), issues copies
    int64_t pc = gw;
    uint32_t pk = 0, pk_end = 0;
    auto chunk_incidences = [&](int64_t c) {
        const int64_t r0 = c * sp.rows_per_chunk;
        const int64_t r1 = min(r0 + sp.rows_per_chunk, p.nrows);
        pk = p.inc_ptr[r0];
        pk_end = p.inc_ptr[r1];
    };
    bool pdone = pc >= sp.nchunks;
    if (!pdone)
        chunk_incidences(pc);
    uint32_t decoded = 0, issued = 0, consumed = 0;  // stream sequence numbers

    auto decode = [&]() -> bool {
        while (!pdone && pk == pk_end) {
            pc += sp.nwarps;
            if (pc >= sp.nchunks)
                pdone = true;
            else
                chunk_incidences(pc);
        }
        if (pdone)
            return false;
        const uint32_t n = min(32u, pk_end - pk);
        if ((uint32_t)lane < n) {
            const unsigned long long pkd = p.inc[pk + lane];
            const RowSeg sg = p.segs[(pkd >> 40) & ((1ull << 23) - 1)];
            const long long co = (long long)(pkd & ((1ull << 40) - 1));
            const long long vo = sg.val_base + (co - sg.coo_base);
            const int width = sg.width;
            const uint64_t vbyte = (uint64_t)vo * 8, sbyte = (uint64_t)co * 2;
            const uint32_t nv = (uint32_t)(((vbyte + (uint64_t)width * 8 + 15) >> 4) - (vbyte >> 4));
            const uint32_t ns = (uint32_t)(((sbyte + (uint64_t)width * 2 + 15) >> 4) - (sbyte >> 4));
            RowStreamDesc d;
            d.mult = sg.mult;
            d.va16 = (uint32_t)(vbyte >> 4);
            d.sa16 = (uint32_t)(sbyte >> 4);
            d.info = (uint32_t)width | ((pkd >> 63) != 0 ? (1u << 7) : 0u) | (uint32_t)((vbyte >> 3) & 1) << 8 |
                     (uint32_t)((sbyte >> 1) & 7) << 9 | nv << 12 | ns << 18;
            d.pad = 0;
            d.pad2 = 0;
            desc[(decoded + lane) & (kStreamDescs - 1)] = d;
        }
        decoded += n;
        pk += n;
        __syncwarp();
        return true;
    };

    // Warp-collective: copies incidence `issued` into ring entry issued % R
    // (every lane commits one group, possibly empty).
    auto issue = [&]() -> bool {
        if (issued == decoded && !decode())
            return false;
        const RowStreamDesc& d = desc[issued & (kStreamDescs - 1)];
        const uint32_t info = d.info;
        const int nv = (int)((info >> 12) & 63), ns = (int)((info >> 18) & 63);
        unsigned char* dv = rv + ((issued & (R - 1)) << VSH);
        unsigned char* ds = rs + ((issued & (R - 1)) << SSH);
        if (Shape::kNarrow) {  // nv + ns <= 24
            if (lane < nv)
                cp_async16(dv + 16 * lane, vals16 + 16 * ((uint64_t)d.va16 + lane));
            else if (lane < nv + ns)
                cp_async16(ds + 16 * (lane - nv), slots16 + 16 * ((uint64_t)d.sa16 + (lane - nv)));
        } else {
            for (int i = lane; i < nv + ns; i += 32) {
                if (i < nv)
                    cp_async16(dv + 16 * i, vals16 + 16 * ((uint64_t)d.va16 + i));
                else
                    cp_async16(ds + 16 * (i - nv), slots16 + 16 * ((uint64_t)d.sa16 + (i - nv)));
            }
        }
        cp_async_commit();
        issued++;
        return true;
    };

    for (int i = 0; i < R; i++)
        if (!issue())
            break;
    // Entry of the first incidence in place for every lane.
    if (issued - consumed >= (uint32_t)R)
        cp_async_wait<R - 1>();
    else
        cp_async_wait<0>();
    __syncwarp();

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
            for (uint32_t k = k0; k < k1; k++) {
                // Incidence `consumed` is in ring entry consumed % R (waited for
                // before the barrier that ended the previous step).
                const RowStreamDesc& d = desc[consumed & (kStreamDescs - 1)];
                const uint32_t info = d.info;
                const double m = d.mult;
                const int width = (int)(info & 127);
                const double* v = reinterpret_cast<const double*>(rv + ((consumed & (R - 1)) << VSH)) + ((info >> 8) & 1);
                const int16_t* sl = reinterpret_cast<const int16_t*>(rs + ((consumed & (R - 1)) << SSH)) + ((info >> 9) & 7);
                if (info & (1u << 7)) {
                    if (lane == 0)
                        for (int j = 0; j < width; j++) {
                            const int s = sl[j];
                            if (s >= 0)
                                buf[s] = fma(v[j], m, buf[s]);
                        }
                } else if (Shape::kNarrow) {
                    if (lane < width) {
                        const int s = sl[lane];
                        if (s >= 0)
                            buf[s] = fma(v[lane], m, buf[s]);
                    }
                } else {
                    for (int j = lane; j < width; j += 32) {
                        const int s = sl[j];
                        if (s >= 0)
                            buf[s] = fma(v[j], m, buf[s]);
                    }
                }
                consumed++;
                // The next incidence's group (the oldest still pending) done.
                if (issued - consumed >= (uint32_t)(R - 1))
                    cp_async_wait<R - 2>();
                else
                    cp_async_wait<0>();
                __syncwarp();  // additions ordered, next entry visible, this entry free
                issue();
            }
            const int64_t r = r0 + rr;
            if (p.dense != nullptr) {
                if (lane == 0)
                    p.dense[r] = L > 0 ? -buf[0] : 0.0;
                __syncwarp();
                for (int s = lane; s < L; s += 32) buf[s] = 0.0;
            } else {
                for (int s = lane; s < L; s += 32) {
                    const double x = buf[s];
                    buf[s] = 0.0;
                    if (s < la)
                        p.Avals[a0 + s] = x;
                    else
                        p.Dvals[d0 + (s - la)] = x;
                }
            }
            __syncwarp();
        }
    }
}

}  // namespace slgpu
