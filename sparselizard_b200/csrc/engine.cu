// slgpu assembly engine: C ABI implementation, coefficient-program compiler,
// geometry/coefficient kernel, FP64 contraction kernel and the COO -> CSR
// builder.  Written for sm_100a (B200); one context per device.
//
// Data flow of slgpu_matrix_process (one call = one sparselizard rawmat::process):
//   1. geometry+coefficients  (per group, thread per (element, Gauss point)):
//        J, detJ, invJ from the curved nodes and Lagrange derivative tables,
//        then the group's coefficient program; writes
//        C[(term, gp)][elem] = coef * scale * w_gp * |detJ|
//   2. contraction (per group, 64x64 output tiles of (tf*ndof+dof) x elements):
//        V[p][e] = sum_{term, gp} T_term[i][gp] * D_term[j][gp] * C[(term,gp)][e]
//      which is contribution.cpp's M = tf (.) dof, K = M * coef^T (:187, :210)
//      without materialising M.
//   3. pattern (cached): COO keys (row, col) of every (group, destination, p, e)
//      and raw fragment, stable radix sort, run detection, A/D split with local
//      renumbering -> CSR structure plus a sorted-position -> COO map.
//   4. values: one thread per CSR entry sums its COO contributions in sorted
//      order (stable sort => insertion order within a (row, col)), so the
//      result is deterministic; no floating-point atomics.
#include "engine_internal.h"
#include "engine_kernels.cuh"
#include "split_tc.cuh"
#include "row_stream.cuh"
#include "contract_f64.cuh"

#include <cudaTypedefs.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <condition_variable>
#include <sys/mman.h>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <stdexcept>

namespace slgpu {

static const char* kNoDevice = "record-only context: nothing is executed";


[[noreturn]] static void fail(int code, const std::string& msg) { throw SlgpuException(code, msg); }

static void cuda_check(cudaError_t err, const char* what)
{
    if (err != cudaSuccess)
        fail(SLGPU_E_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
}

DevBuf& DevBuf::operator=(DevBuf&& o) noexcept
{
    if (this != &o) {
        release();
        ctx_ = o.ctx_;
        s_ = o.s_;
        p_ = o.p_;
        n_ = o.n_;
        arena_ = o.arena_;
        o.ctx_ = nullptr;
        o.p_ = nullptr;
        o.n_ = 0;
        o.arena_ = false;
    }
    return *this;
}

void DevBuf::alloc(Ctx* ctx, size_t bytes)
{
    release();
    if (bytes == 0)
        bytes = 16;
    bytes = (bytes + 255) & ~size_t(255);
    Exec& x = *ctx->x;
    if (x.arena_on) {
        if (x.arena_off + bytes <= x.arena.bytes()) {
            p_ = x.arena.as<char>() + x.arena_off;
            x.arena_off += bytes;
            ctx_ = ctx;
            s_ = x.stream;
            n_ = bytes;
            arena_ = true;
            return;
        }
        x.arena_miss += bytes;
    }
    if ((size_t)ctx->in_use + bytes > ctx->budget)
        fail(SLGPU_E_BUDGET, "device allocation of " + std::to_string(bytes) + " bytes exceeds the HBM budget (" +
                                 std::to_string(ctx->in_use) + " of " + std::to_string(ctx->budget) + " in use)");
    cudaError_t err = cudaMallocAsync(&p_, bytes, ctx->x->stream);
    if (err != cudaSuccess) {
        p_ = nullptr;
        fail(SLGPU_E_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(err));
    }
    ctx_ = ctx;
    s_ = ctx->x->stream;
    n_ = bytes;
    ctx->in_use += (int64_t)bytes;
}

void DevBuf::release()
{
    if (p_ != nullptr && ctx_ != nullptr && !arena_) {
        cudaFreeAsync(p_, s_);
        ctx_->in_use -= (int64_t)n_;
    }
    p_ = nullptr;
    n_ = 0;
    ctx_ = nullptr;
    arena_ = false;
}

// Host -> device copy of a large pageable array on the context's stream:
// 4 MB chunks through a ring of page-locked blocks.  Up to 8 worker threads
// (created per call), worker w taking chunks w, w + 8, ... into its two
// blocks: it waits for the block's previous copy, copies the chunk in, queues
// the copy to the device and records the block's event.  The source has been
// read when this returns; the device copies complete in stream order.  (A
// pageable cudaMemcpyAsync is staged by the driver on the calling thread.)
static void h2d_pageable(Ctx* ctx, void* dst, const void* src, size_t n)
{
    constexpr size_t kChunk = size_t(4) << 20;
    std::lock_guard<std::mutex> lk(ctx->ul_mu);
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nw = std::max(1, std::min(std::min(hw, 8), Ctx::kUlStages / 2));
    for (int b = 0; b < 2 * nw; b++) {
        if (ctx->ul_stage[b] == nullptr)
            cuda_check(cudaHostAlloc(reinterpret_cast<void**>(&ctx->ul_stage[b]), kChunk, cudaHostAllocDefault), "cudaHostAlloc");
        if (ctx->ul_ev[b] == nullptr)
            cuda_check(cudaEventCreateWithFlags(&ctx->ul_ev[b], cudaEventDisableTiming), "cudaEventCreate");
    }
    const size_t nch = (n + kChunk - 1) / kChunk;
    std::mutex emu;
    std::string err;
    std::vector<std::thread> workers;
    for (int w = 0; w < nw; w++)
        workers.emplace_back([&, w] {
            int use = 0;
            for (size_t i = (size_t)w; i < nch; i += (size_t)nw, use ^= 1) {
                const int b = 2 * w + use;
                const size_t off = i * kChunk, len = std::min(kChunk, n - off);
                cudaError_t e = cudaEventSynchronize(ctx->ul_ev[b]);
                if (e == cudaSuccess) {
                    std::memcpy(ctx->ul_stage[b], static_cast<const char*>(src) + off, len);
                    e = cudaMemcpyAsync(static_cast<char*>(dst) + off, ctx->ul_stage[b], len, cudaMemcpyHostToDevice, ctx->x->stream);
                }
                if (e == cudaSuccess)
                    e = cudaEventRecord(ctx->ul_ev[b], ctx->x->stream);
                if (e != cudaSuccess) {
                    std::lock_guard<std::mutex> g(emu);
                    err = std::string("H2D chunk: ") + cudaGetErrorString(e);
                    return;
                }
            }
        });
    for (auto& t : workers) t.join();
    if (!err.empty())
        fail(SLGPU_E_CUDA, err);
}

template <class T>
static void upload(Ctx* ctx, DevBuf& buf, const T* src, size_t count)
{
    buf.alloc(ctx, count * sizeof(T));
    const size_t bytes = count * sizeof(T);
    ctx->bytes_h2d += (int64_t)bytes;
    if (count == 0)
        return;
    if (bytes >= (size_t(8) << 20) && !ctx->x->capturing) {
        cudaPointerAttributes a{};
        const bool pinned = cudaPointerGetAttributes(&a, src) == cudaSuccess && a.type == cudaMemoryTypeHost;
        cudaGetLastError();
        if (!pinned) {
            h2d_pageable(ctx, buf.as<void>(), src, bytes);
            return;
        }
    }
    cuda_check(cudaMemcpyAsync(buf.as<void>(), src, bytes, cudaMemcpyHostToDevice, ctx->x->stream), "cudaMemcpyAsync H2D");
}

template <class T>
static void upload(Ctx* ctx, DevBuf& buf, const std::vector<T>& v)
{
    upload(ctx, buf, v.data(), v.size());
}

static unsigned grid_for(int64_t n, int block) { return (unsigned)std::max<int64_t>(1, (n + block - 1) / block); }

// ------------------------------------------------------------ program compiler
// Turns the node DAG into straight-line code over kMaxSlots registers: each
// node gets a free slot, operand slots are freed after their last use, and a
// STORE is emitted right after a node that is some term's coefficient.
static std::vector<Instr> compile_program(const slgpu_group& g, int nterms)
{
    const int n = g.nnodes;
    std::vector<int> last_use(n, -1);
    std::vector<char> needed(n, 0);
    for (int t = 0; t < nterms; t++) {
        int c = g.terms[t].coef_node;
        if (c < 0 || c >= n)
            fail(SLGPU_E_ARG, "term coefficient node out of range");
        needed[c] = 1;
    }
    auto is_binary = [](int op) { return op == SLGPU_OP_ADD || op == SLGPU_OP_MUL || op == SLGPU_OP_POW; };
    auto is_unary = [](int op) { return op == SLGPU_OP_INV || op == SLGPU_OP_NEG; };
    for (int k = n - 1; k >= 0; k--) {
        if (!needed[k])
            continue;
        const slgpu_node& nd = g.nodes[k];
        if (is_binary(nd.op) || is_unary(nd.op)) {
            int ops[2] = {nd.a, is_binary(nd.op) ? nd.b : -1};
            for (int o : ops) {
                if (o < 0)
                    continue;
                if (o >= k)
                    fail(SLGPU_E_ARG, "coefficient program operand must precede its node");
                needed[o] = 1;
                last_use[o] = std::max(last_use[o], k);
            }
        }
    }
    std::vector<Instr> prog;
    std::vector<int> slot_of(n, -1);
    std::vector<int> free_slots;
    for (int s = kMaxSlots - 1; s >= 0; s--) free_slots.push_back(s);
    for (int k = 0; k < n; k++) {
        if (!needed[k])
            continue;
        const slgpu_node& nd = g.nodes[k];
        Instr in{nd.op, -1, nd.a, nd.b};
        switch (nd.op) {
        case SLGPU_OP_CONST:
            if (nd.a < 0 || nd.a >= g.nconsts) fail(SLGPU_E_ARG, "constant index out of range");
            break;
        case SLGPU_OP_JAC:
        case SLGPU_OP_INVJAC:
            if (nd.a < 0 || nd.a >= g.problemdim || nd.b < 0 || nd.b >= g.problemdim)
                fail(SLGPU_E_ARG, "Jacobian entry out of range");
            break;
        case SLGPU_OP_DETJAC:
            break;
        case SLGPU_OP_ELEM:
            if (nd.a < 0 || nd.a >= g.nelemdata) fail(SLGPU_E_ARG, "element data index out of range");
            break;
        case SLGPU_OP_FIELD:
            if (nd.a < 0 || nd.a >= g.nfielddata || nd.b < 0 || nd.b >= g.ntables)
                fail(SLGPU_E_ARG, "field data / table index out of range");
            if (g.tables[nd.b].rows != g.fieldrows[nd.a])
                fail(SLGPU_E_ARG, "field coefficient rows do not match its table");
            break;
        case SLGPU_OP_COORD:
            if (nd.a < 0 || nd.a > 2) fail(SLGPU_E_ARG, "coordinate index out of range");
            break;
        case SLGPU_OP_ADD:
        case SLGPU_OP_MUL:
        case SLGPU_OP_POW:
            in.a = slot_of[nd.a];
            in.b = slot_of[nd.b];
            break;
        case SLGPU_OP_INV:
        case SLGPU_OP_NEG:
            in.a = slot_of[nd.a];
            break;
        default:
            fail(SLGPU_E_UNSUPPORTED, "unknown coefficient program op " + std::to_string(nd.op));
        }
        // Free operand slots whose last use is this node (before taking the
        // destination so that an operand slot can be reused in place).
        if (is_binary(nd.op) || is_unary(nd.op)) {
            int ops[2] = {nd.a, is_binary(nd.op) ? nd.b : -1};
            for (int i = 0; i < 2; i++) {
                int o = ops[i];
                if (o < 0 || last_use[o] != k || slot_of[o] < 0)
                    continue;
                if (i == 1 && ops[0] == o)
                    continue;
                free_slots.push_back(slot_of[o]);
                slot_of[o] = -2;
            }
        }
        if (free_slots.empty())
            fail(SLGPU_E_UNSUPPORTED, "coefficient program needs more than " + std::to_string(kMaxSlots) + " live values");
        in.dst = free_slots.back();
        free_slots.pop_back();
        slot_of[k] = in.dst;
        prog.push_back(in);
        for (int t = 0; t < nterms; t++)
            if (g.terms[t].coef_node == k)
                prog.push_back(Instr{INSTR_STORE, -1, in.dst, t});
        if (last_use[k] < 0) {  // only stored
            free_slots.push_back(in.dst);
            slot_of[k] = -2;
        }
    }
    return prog;
}

// ------------------------------------------------------------ hashing
// Hashes of several device arrays (data[i], n[i] entries, salt[i]) into
// out[2 i], out[2 i + 1], with one read-back.
static void hash_device_many(Ctx* ctx, const std::vector<const int32_t*>& data, const std::vector<int64_t>& n,
                             const std::vector<uint64_t>& salt, uint64_t* out)
{
    const size_t m = data.size();
    if (m == 0)
        return;
    if (ctx->hash_acc.bytes() < 2 * m * sizeof(unsigned long long))
        ctx->hash_acc.alloc(ctx, 2 * m * sizeof(unsigned long long));
    unsigned long long* acc = ctx->hash_acc.as<unsigned long long>();
    cuda_check(cudaMemsetAsync(acc, 0, 2 * m * sizeof(unsigned long long), ctx->x->stream), "memset");
    for (size_t i = 0; i < m; i++)
        if (n[i] > 0) {
            unsigned blocks = (unsigned)std::min<int64_t>(148 * 8, grid_for(n[i], 256));
            k_hash_i32<<<blocks, 256, 0, ctx->x->stream>>>(data[i], n[i], salt[i], acc + 2 * i);
            cuda_check(cudaGetLastError(), "k_hash_i32");
        }
    std::vector<unsigned long long> h(2 * m);
    cuda_check(cudaMemcpyAsync(h.data(), acc, 2 * m * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->x->stream), "D2H hash");
    cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync hash");
    for (size_t i = 0; i < 2 * m; i++) out[i] = h[i];
}

static void hash_device(Ctx* ctx, const int32_t* data, int64_t n, uint64_t salt, uint64_t out[2])
{
    if (ctx->hash_acc.empty())
        ctx->hash_acc.alloc(ctx, 2 * sizeof(unsigned long long));
    cuda_check(cudaMemsetAsync(ctx->hash_acc.as<void>(), 0, 2 * sizeof(unsigned long long), ctx->x->stream), "memset");
    if (n > 0) {
        unsigned blocks = (unsigned)std::min<int64_t>(148 * 8, grid_for(n, 256));
        k_hash_i32<<<blocks, 256, 0, ctx->x->stream>>>(data, n, salt, ctx->hash_acc.as<unsigned long long>());
        cuda_check(cudaGetLastError(), "k_hash_i32");
    }
    unsigned long long h[2];
    cuda_check(cudaMemcpyAsync(h, ctx->hash_acc.as<void>(), sizeof(h), cudaMemcpyDeviceToHost, ctx->x->stream), "D2H hash");
    cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync hash");
    out[0] = h[0];
    out[1] = h[1];
}

static inline uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// ------------------------------------------------------------ group upload
struct GroupDev::Record {
    std::vector<int32_t> elems, orient, fieldrows;
    std::vector<double> weights, lagrange, consts;
    std::vector<std::vector<double>> tables, elemdata, fielddata;
    std::vector<slgpu_table> tabdesc;
    std::vector<slgpu_node> nodes;
    std::vector<const double*> elemdata_ptr, fielddata_ptr;
    std::vector<slgpu_term> terms;
    std::vector<std::vector<int32_t>> tfaddr, dofaddr;
    std::vector<slgpu_dest> dests;
    slgpu_group desc{};
};

// `with_dests`: the group is assembled, so it needs at least one valid
// destination (the allocation-free element-matrix call has none).
static void validate_group(const slgpu_group& g, bool with_dests = true)
{
    if (g.nelem < 0 || g.ngp <= 0 || g.ntf <= 0 || g.ndof <= 0 || g.nterms <= 0 || (with_dests && g.ndests <= 0) || g.norient <= 0)
        fail(SLGPU_E_ARG, "group sizes must be positive");
    if (g.elemdim < 0 || g.elemdim > g.problemdim)
        fail(SLGPU_E_ARG, "element dimension must be in [0, mesh dimension] (element dim " + std::to_string(g.elemdim) +
                              ", mesh dim " + std::to_string(g.problemdim) + ")");
    if (g.problemdim < 1 || g.problemdim > 3)
        fail(SLGPU_E_ARG, "problem dimension must be 1..3");
    if (g.ncurvednodes <= 0 || g.ncurvednodes > 64)
        fail(SLGPU_E_UNSUPPORTED, "curved node count out of range");
    for (int t = 0; t < g.nterms; t++) {
        const slgpu_term& tm = g.terms[t];
        if (tm.tf_table < 0 || tm.tf_table >= g.ntables || g.tables[tm.tf_table].rows != g.ntf)
            fail(SLGPU_E_ARG, "term tf table invalid or its rows differ from ntf");
        bool rhs_term = tm.dof_table < 0;
        if (rhs_term != (g.ndof == 1 && g.terms[0].dof_table < 0))
            fail(SLGPU_E_ARG, "a group mixes right-hand-side and matrix terms");
        if (!rhs_term && (tm.dof_table >= g.ntables || g.tables[tm.dof_table].rows != g.ndof))
            fail(SLGPU_E_ARG, "term dof table invalid or its rows differ from ndof");
    }
    for (int d = 0; with_dests && d < g.ndests; d++) {
        if (g.dests[d].tfaddr == nullptr)
            fail(SLGPU_E_ARG, "destination without test-function addresses");
        if (g.terms[0].dof_table >= 0 && g.dests[d].dofaddr == nullptr)
            fail(SLGPU_E_ARG, "matrix destination without dof addresses");
    }
    if ((int64_t)g.ntf * g.ndof * std::max<int64_t>(g.nelem, 1) >= (int64_t(1) << 40))
        fail(SLGPU_E_UNSUPPORTED, "group too large");
}

// Mirror term of each term when the group's element matrices are symmetric
// (empty otherwise).  The condition: ntf == ndof, and every term t has a
// partner u (t itself allowed) whose test-function table holds the values of
// t's dof table and whose dof table holds those of t's test-function table,
// with a coefficient node that computes the same expression: the same
// operations on the same inputs, the operands of + in either order and the
// factors of a chain of products in any order.  Entry (j, i) of term u is
// then the product of entry (i, j) of term t with u's coefficient.
//
// `exact`: every coefficient also equals its mirror's bit for bit (IEEE
// addition and multiplication commute exactly, so this holds when only the
// two operands of single operations are swapped); the split contraction's
// exact integer sums then give M[i][j] == M[j][i] with or without the
// mirroring.  Otherwise a reordered product of n factors differs from its
// mirror by at most about n units in the last place, far below the split
// tiers' error bounds.  The scales are checked where the contraction is
// launched (they can change).
struct Mirror {
    std::vector<int32_t> term;
    bool exact = false;
};

static Mirror mirror_terms(const slgpu_group& g)
{
    if (g.ntf != g.ndof || g.terms[0].dof_table < 0)
        return {};
    // Tables with equal values share a class.
    std::vector<int> tcls(g.ntables);
    for (int k = 0; k < g.ntables; k++) {
        tcls[k] = k;
        const size_t n = (size_t)g.norient * g.tables[k].rows * g.ngp;
        for (int k2 = 0; k2 < k; k2++)
            if (tcls[k2] == k2 && g.tables[k2].rows == g.tables[k].rows &&
                std::memcmp(g.tables[k2].vals, g.tables[k].vals, n * sizeof(double)) == 0) {
                tcls[k] = k2;
                break;
            }
    }
    // Two classes per node by hash-consing over the program order: `ecls`
    // (same value bit for bit: + and * with operands in either order) and
    // `rcls` (same value up to the order of factors: a chain of products is
    // keyed by the sorted classes of its factors).
    std::map<std::vector<int64_t>, int> eids, rids;
    std::vector<int> ecls(g.nnodes), rcls(g.nnodes);
    std::vector<std::vector<int64_t>> factors(g.nnodes);
    for (int k = 0; k < g.nnodes; k++) {
        const slgpu_node& nd = g.nodes[k];
        const bool ref_a = nd.op == SLGPU_OP_ADD || nd.op == SLGPU_OP_MUL || nd.op == SLGPU_OP_POW || nd.op == SLGPU_OP_INV ||
                           nd.op == SLGPU_OP_NEG;
        const bool ref_b = nd.op == SLGPU_OP_ADD || nd.op == SLGPU_OP_MUL || nd.op == SLGPU_OP_POW;
        if ((ref_a && (nd.a < 0 || nd.a >= k)) || (ref_b && (nd.b < 0 || nd.b >= k)))
            return {};
        std::vector<int64_t> ek{nd.op, nd.a, ref_b ? nd.b : (int64_t)nd.b, nd.c}, rk;
        switch (nd.op) {
        case SLGPU_OP_CONST:
            if (nd.a < 0 || nd.a >= g.nconsts)
                return {};
            std::memcpy(&ek[1], &g.consts[nd.a], 8);
            ek[2] = 0;
            break;
        case SLGPU_OP_FIELD:
            if (nd.b < 0 || nd.b >= g.ntables)
                return {};
            ek[2] = tcls[nd.b];
            break;
        default:
            break;
        }
        rk = ek;
        if (ref_a) {
            ek[1] = ecls[nd.a];
            rk[1] = rcls[nd.a];
        }
        if (ref_b) {
            ek[2] = ecls[nd.b];
            rk[2] = rcls[nd.b];
        }
        if (nd.op == SLGPU_OP_ADD || nd.op == SLGPU_OP_MUL) {
            if (ek[1] > ek[2])
                std::swap(ek[1], ek[2]);
            if (rk[1] > rk[2])
                std::swap(rk[1], rk[2]);
        }
        if (nd.op == SLGPU_OP_MUL) {
            std::vector<int64_t>& f = factors[k];
            for (int x : {nd.a, nd.b}) {
                if (g.nodes[x].op == SLGPU_OP_MUL)
                    f.insert(f.end(), factors[x].begin(), factors[x].end());
                else
                    f.push_back(rcls[x]);
            }
            std::sort(f.begin(), f.end());
            rk.assign(1, SLGPU_OP_MUL);
            rk.insert(rk.end(), f.begin(), f.end());
        }
        ecls[k] = eids.emplace(ek, (int)eids.size()).first->second;
        rcls[k] = rids.emplace(rk, (int)rids.size()).first->second;
    }
    Mirror m;
    m.term.assign(g.nterms, -1);
    m.exact = true;
    for (int t = 0; t < g.nterms; t++) {
        if (m.term[t] >= 0)
            continue;
        const slgpu_term& a = g.terms[t];
        if (a.coef_node < 0 || a.coef_node >= g.nnodes)
            return {};
        for (int u = t; u < g.nterms; u++) {
            const slgpu_term& b = g.terms[u];
            if (m.term[u] < 0 && b.coef_node >= 0 && b.coef_node < g.nnodes && tcls[b.tf_table] == tcls[a.dof_table] &&
                tcls[b.dof_table] == tcls[a.tf_table] && rcls[b.coef_node] == rcls[a.coef_node]) {
                m.term[t] = u;
                m.term[u] = t;
                m.exact = m.exact && ecls[b.coef_node] == ecls[a.coef_node];
                break;
            }
        }
        if (m.term[t] < 0)
            return {};
    }
    return m;
}

// 128-bit content keys (two independent 64-bit mixes).
static GroupDev::Key key_mix(GroupDev::Key k, uint64_t v)
{
    return {mix64(k.a ^ v), mix64(k.b + (v ^ 0xD6E8FEB86659FD93ull) * 0x9E3779B97F4A7C15ull)};
}

// Key of an array: four interleaved chains (entry i goes to chain i % 4, so
// their multiplies overlap), combined at the end with the length.
static GroupDev::Key key_of(const double* v, size_t n, uint64_t tag)
{
    GroupDev::Key c[4];
    for (int j = 0; j < 4; j++) c[j] = GroupDev::Key{tag + (uint64_t)j, ~tag - (uint64_t)j};
    size_t i = 0;
    for (; i + 4 <= n; i += 4) {
        uint64_t w[4];
        std::memcpy(w, &v[i], 32);
        c[0] = key_mix(c[0], w[0]);
        c[1] = key_mix(c[1], w[1]);
        c[2] = key_mix(c[2], w[2]);
        c[3] = key_mix(c[3], w[3]);
    }
    for (; i < n; i++) {
        uint64_t w;
        std::memcpy(&w, &v[i], 8);
        c[i % 4] = key_mix(c[i % 4], w);
    }
    GroupDev::Key k = key_mix(GroupDev::Key{tag, ~tag}, n);
    for (int j = 0; j < 4; j++) k = key_mix(key_mix(k, c[j].a), c[j].b);
    return k;
}

// Per-term content keys (tables by value, coefficient nodes by expression with
// + operands and product factors in any order) and data array keys.
static void content_keys(const slgpu_group& g, GroupDev& gd)
{
    gd.term_keys.clear();
    gd.data_keys.clear();
    for (int k = 0; k < g.nelemdata; k++) gd.data_keys.push_back(key_of(g.elemdata[k], (size_t)g.nelem, 1));
    for (int k = 0; k < g.nfielddata; k++)
        gd.data_keys.push_back(key_of(g.fielddata[k], (size_t)g.fieldrows[k] * g.nelem, 2));
    if (g.terms[0].dof_table < 0)
        return;
    std::vector<GroupDev::Key> tk(g.ntables);
    for (int k = 0; k < g.ntables; k++)
        tk[k] = key_mix(key_of(g.tables[k].vals, (size_t)g.norient * g.tables[k].rows * g.ngp, 3), (uint64_t)g.tables[k].rows);
    std::vector<GroupDev::Key> nk(g.nnodes);
    std::vector<std::vector<GroupDev::Key>> factors(g.nnodes);
    auto less = [](const GroupDev::Key& x, const GroupDev::Key& y) { return x.a != y.a ? x.a < y.a : x.b < y.b; };
    for (int k = 0; k < g.nnodes; k++) {
        const slgpu_node& nd = g.nodes[k];
        // Operands precede their node (checked by the program compiler for
        // the nodes it uses); others key as zero.
        auto at = [&](int x) { return x >= 0 && x < k ? nk[x] : GroupDev::Key{}; };
        GroupDev::Key h{(uint64_t)nd.op * 0x100000001B3ull, (uint64_t)nd.op};
        switch (nd.op) {
        case SLGPU_OP_CONST: {
            uint64_t w = 0;
            if (nd.a >= 0 && nd.a < g.nconsts)
                std::memcpy(&w, &g.consts[nd.a], 8);
            h = key_mix(h, w);
            break;
        }
        case SLGPU_OP_FIELD:
            h = key_mix(key_mix(h, (uint64_t)nd.a), nd.b >= 0 && nd.b < g.ntables ? tk[nd.b].a : 0);
            h = key_mix(h, nd.b >= 0 && nd.b < g.ntables ? tk[nd.b].b : 0);
            break;
        case SLGPU_OP_ADD: {
            GroupDev::Key x = at(nd.a), y = at(nd.b);
            if (less(y, x))
                std::swap(x, y);
            h = key_mix(key_mix(key_mix(key_mix(h, x.a), x.b), y.a), y.b);
            break;
        }
        case SLGPU_OP_MUL: {
            std::vector<GroupDev::Key>& f = factors[k];
            for (int x : {nd.a, nd.b}) {
                if (x >= 0 && x < k && g.nodes[x].op == SLGPU_OP_MUL)
                    f.insert(f.end(), factors[x].begin(), factors[x].end());
                else
                    f.push_back(at(x));
            }
            std::sort(f.begin(), f.end(), less);
            for (const GroupDev::Key& x : f) h = key_mix(key_mix(h, x.a), x.b);
            break;
        }
        case SLGPU_OP_POW:
            h = key_mix(key_mix(key_mix(key_mix(h, at(nd.a).a), at(nd.a).b), at(nd.b).a), at(nd.b).b);
            break;
        case SLGPU_OP_INV:
        case SLGPU_OP_NEG:
            h = key_mix(key_mix(h, at(nd.a).a), at(nd.a).b);
            break;
        default:
            h = key_mix(key_mix(key_mix(h, (uint64_t)(uint32_t)nd.a), (uint64_t)(uint32_t)nd.b), (uint64_t)(uint32_t)nd.c);
            break;
        }
        nk[k] = h;
    }
    for (int t = 0; t < g.nterms; t++) gd.term_keys.push_back({tk[g.terms[t].tf_table], tk[g.terms[t].dof_table], nk[g.terms[t].coef_node]});
}

static std::shared_ptr<GroupDev> make_group(Ctx* ctx, const slgpu_group& g,
                                            std::map<std::pair<const void*, int64_t>, Matrix::SharedAddresses>* shared = nullptr)
{
    validate_group(g);
    auto gd = std::make_shared<GroupDev>();
    gd->serial = ctx->next_serial++;
    gd->mesh = g.mesh;
    gd->elemtype = g.elemtype;
    gd->elemdim = g.elemdim;
    gd->problemdim = g.problemdim;
    gd->nelem = g.nelem;
    gd->norient = g.norient;
    gd->ngp = g.ngp;
    gd->ncn = g.ncurvednodes;
    gd->ntf = g.ntf;
    gd->ndof = g.ndof;
    gd->nterms = g.nterms;
    gd->ndests = g.ndests;
    gd->rhs = g.terms[0].dof_table < 0;
    gd->prog = compile_program(g, g.nterms);
    gd->nodes.assign(g.nodes, g.nodes + g.nnodes);
    for (int t = 0; t < g.nterms; t++) gd->term_node.push_back(g.terms[t].coef_node);
    {
        Mirror m = mirror_terms(g);
        gd->mirror = std::move(m.term);
        gd->mirror_exact = m.exact;
    }
    content_keys(g, *gd);
    gd->hconsts.assign(g.consts, g.consts + g.nconsts);
    {
        // Geometry key: groups with the same key share elements, orientations,
        // Gauss points and Lagrange tables, so one kernel evaluates them all.
        uint64_t h = mix64((uint64_t)g.mesh ^ (uint64_t)g.elemtype << 8 ^ (uint64_t)g.ngp << 16 ^ (uint64_t)g.ncurvednodes << 32 ^
                           (uint64_t)g.problemdim << 48);
        h = mix64(h ^ (uint64_t)g.nelem ^ (uint64_t)(uint32_t)g.mesh << 40 ^ (uint64_t)(uint32_t)g.elemtype << 56);
        // Elements and orientations in four interleaved chains (e % 4).
        auto word = [&](int64_t e) { return (uint64_t)(uint32_t)g.elems[e] << 8 | (uint64_t)(uint32_t)g.orient[e] << 40; };
        uint64_t c0 = h, c1 = h + 1, c2 = h + 2, c3 = h + 3;
        int64_t e = 0;
        for (; e + 4 <= g.nelem; e += 4) {
            c0 = mix64(c0 ^ word(e));
            c1 = mix64(c1 ^ word(e + 1));
            c2 = mix64(c2 ^ word(e + 2));
            c3 = mix64(c3 ^ word(e + 3));
        }
        for (; e < g.nelem; e++) c0 = mix64(c0 ^ word(e) ^ (uint64_t)e);
        h = mix64(mix64(mix64(mix64(h ^ c0) ^ c1) ^ c2) ^ c3);
        const size_t nl = (size_t)(1 + g.elemdim) * g.ncurvednodes * g.ngp;
        for (size_t k = 0; k < nl; k++) {
            uint64_t w;
            std::memcpy(&w, &g.lagrange[k], 8);
            h = mix64(h ^ w);
        }
        for (int k = 0; k < g.ngp; k++) {
            uint64_t w;
            std::memcpy(&w, &g.weights[k], 8);
            h = mix64(h ^ w);
        }
        gd->geom_hash = h;
    }
    int64_t off = 0;
    for (int k = 0; k < g.ntables; k++) {
        gd->tab_off.push_back(off);
        gd->tab_rows.push_back(g.tables[k].rows);
        off += (int64_t)g.norient * g.tables[k].rows * g.ngp;
    }
    const int64_t tables_total = off;
    for (int k = 0; k < g.nelemdata; k++) gd->elemdata_off.push_back((int64_t)k * g.nelem);
    off = 0;
    for (int k = 0; k < g.nfielddata; k++) {
        gd->field_off.push_back(off);
        gd->field_rows.push_back(g.fieldrows[k]);
        off += (int64_t)g.fieldrows[k] * g.nelem;
    }
    const int64_t field_total = off;
    for (int t = 0; t < g.nterms; t++) {
        gd->term_scale.push_back(g.terms[t].scale);
        gd->term_tf.push_back(g.terms[t].tf_table);
        gd->term_dof.push_back(g.terms[t].dof_table);
    }
    for (int d = 0; d < g.ndests; d++) gd->dest_mult.push_back(g.dests[d].multiplier);
    // Orientation-uniform tiles of at most kTileE elements.
    for (int64_t e = 0; e < g.nelem;) {
        int o = g.orient[e];
        if (o < 0 || o >= g.norient)
            fail(SLGPU_E_ARG, "orientation index out of range");
        int64_t e1 = e;
        while (e1 < g.nelem && g.orient[e1] == o && e1 - e < kTileE) e1++;
        gd->tiles.push_back(Tile{(int32_t)e, (int32_t)(e1 - e), o, 0});
        e = e1;
    }
    if (g.nelem >= (int64_t(1) << 31))
        fail(SLGPU_E_UNSUPPORTED, "more than 2^31 elements in a group");

    if (ctx->record_only) {
        auto r = std::make_shared<GroupDev::Record>();
        r->elems.assign(g.elems, g.elems + g.nelem);
        r->orient.assign(g.orient, g.orient + g.nelem);
        r->weights.assign(g.weights, g.weights + g.ngp);
        r->lagrange.assign(g.lagrange, g.lagrange + (size_t)(1 + g.elemdim) * g.ncurvednodes * g.ngp);
        r->consts.assign(g.consts, g.consts + g.nconsts);
        for (int k = 0; k < g.ntables; k++)
            r->tables.emplace_back(g.tables[k].vals, g.tables[k].vals + (size_t)g.norient * g.tables[k].rows * g.ngp);
        for (int k = 0; k < g.ntables; k++) r->tabdesc.push_back(slgpu_table{g.tables[k].rows, r->tables[k].data()});
        r->nodes.assign(g.nodes, g.nodes + g.nnodes);
        for (int k = 0; k < g.nelemdata; k++) r->elemdata.emplace_back(g.elemdata[k], g.elemdata[k] + g.nelem);
        for (int k = 0; k < g.nfielddata; k++)
            r->fielddata.emplace_back(g.fielddata[k], g.fielddata[k] + (size_t)g.fieldrows[k] * g.nelem);
        for (auto& v : r->elemdata) r->elemdata_ptr.push_back(v.data());
        for (auto& v : r->fielddata) r->fielddata_ptr.push_back(v.data());
        r->fieldrows.assign(g.fieldrows, g.fieldrows + g.nfielddata);
        r->terms.assign(g.terms, g.terms + g.nterms);
        for (int d = 0; d < g.ndests; d++) {
            r->tfaddr.emplace_back(g.dests[d].tfaddr, g.dests[d].tfaddr + (size_t)g.ntf * g.nelem);
            if (!gd->rhs)
                r->dofaddr.emplace_back(g.dests[d].dofaddr, g.dests[d].dofaddr + (size_t)g.ndof * g.nelem);
            else
                r->dofaddr.emplace_back();
        }
        for (int d = 0; d < g.ndests; d++)
            r->dests.push_back(slgpu_dest{r->tfaddr[d].data(), gd->rhs ? nullptr : r->dofaddr[d].data(), g.dests[d].multiplier});
        r->desc = g;
        r->desc.elems = r->elems.data();
        r->desc.orient = r->orient.data();
        r->desc.weights = r->weights.data();
        r->desc.lagrange = r->lagrange.data();
        r->desc.tables = r->tabdesc.data();
        r->desc.nodes = r->nodes.data();
        r->desc.consts = r->consts.data();
        r->desc.elemdata = r->elemdata_ptr.data();
        r->desc.fielddata = r->fielddata_ptr.data();
        r->desc.fieldrows = r->fieldrows.data();
        r->desc.terms = r->terms.data();
        r->desc.dests = r->dests.data();
        gd->rec = r;
        return gd;
    }

    auto mit = ctx->meshes.find(g.mesh);
    if (mit == ctx->meshes.end() || mit->second.types.count(g.elemtype) == 0)
        fail(SLGPU_E_STATE, "mesh geometry for this element type was not uploaded");
    const MeshDev::Type& mt = mit->second.types.at(g.elemtype);
    if (mt.ncn != g.ncurvednodes)
        fail(SLGPU_E_ARG, "curved node count differs from the uploaded mesh");
    for (int64_t e = 0; e < g.nelem; e++)
        if (g.elems[e] < 0 || g.elems[e] >= mt.nelem)
            fail(SLGPU_E_ARG, "element number out of range of the uploaded mesh");

    upload(ctx, gd->elems, g.elems, (size_t)g.nelem);
    upload(ctx, gd->orient, g.orient, (size_t)g.nelem);
    upload(ctx, gd->weights, g.weights, (size_t)g.ngp);
    upload(ctx, gd->lagrange, g.lagrange, (size_t)(1 + g.elemdim) * g.ncurvednodes * g.ngp);
    gd->tables.alloc(ctx, (size_t)tables_total * sizeof(double));
    ctx->bytes_h2d += (int64_t)tables_total * 8 + (int64_t)g.nelemdata * g.nelem * 8 + field_total * 8;
    for (int k = 0; k < g.ntables; k++)
        cuda_check(cudaMemcpyAsync(gd->tables.as<double>() + gd->tab_off[k], g.tables[k].vals,
                                   (size_t)g.norient * g.tables[k].rows * g.ngp * sizeof(double), cudaMemcpyHostToDevice,
                                   ctx->x->stream),
                   "upload tables");
    upload(ctx, gd->consts, g.consts, (size_t)g.nconsts);
    upload(ctx, gd->prog_d, gd->prog);
    gd->elemdata.alloc(ctx, (size_t)g.nelemdata * g.nelem * sizeof(double));
    for (int k = 0; k < g.nelemdata; k++)
        cuda_check(cudaMemcpyAsync(gd->elemdata.as<double>() + gd->elemdata_off[k], g.elemdata[k],
                                   (size_t)g.nelem * sizeof(double), cudaMemcpyHostToDevice, ctx->x->stream),
                   "upload elemdata");
    gd->fielddata.alloc(ctx, (size_t)field_total * sizeof(double));
    for (int k = 0; k < g.nfielddata; k++)
        cuda_check(cudaMemcpyAsync(gd->fielddata.as<double>() + gd->field_off[k], g.fielddata[k],
                                   (size_t)g.fieldrows[k] * g.nelem * sizeof(double), cudaMemcpyHostToDevice, ctx->x->stream),
                   "upload fielddata");
    upload(ctx, gd->field_off_d, gd->field_off);
    upload(ctx, gd->field_rows_d, gd->field_rows);
    upload(ctx, gd->tab_off_d, gd->tab_off);
    upload(ctx, gd->tab_rows_d, gd->tab_rows);
    upload(ctx, gd->term_scale_d, gd->term_scale);
    upload(ctx, gd->term_tf_d, gd->term_tf);
    upload(ctx, gd->term_dof_d, gd->term_dof);
    upload(ctx, gd->tiles_d, gd->tiles);
    // Address arrays: uploaded and hashed by content, or, where the caller
    // allows it, taken from an earlier group of the same matrix given the same
    // host array.  The destination's place (salt) is mixed in on the host.
    gd->tfaddr.resize(g.ndests);
    gd->dofaddr.resize(g.ndests);
    struct Part {
        std::shared_ptr<DevBuf>* dst;
        const int32_t* host;
        int64_t n;
        uint64_t salt;
        uint64_t hash[2];
    };
    std::vector<Part> parts;
    for (int d = 0; d < g.ndests; d++) {
        parts.push_back(Part{&gd->tfaddr[d], g.dests[d].tfaddr, (int64_t)g.ntf * g.nelem, (uint64_t)(2 * d + 1), {0, 0}});
        if (!gd->rhs)
            parts.push_back(Part{&gd->dofaddr[d], g.dests[d].dofaddr, (int64_t)g.ndof * g.nelem, (uint64_t)(2 * d + 2), {0, 0}});
    }
    std::vector<const int32_t*> hdata;
    std::vector<int64_t> hn;
    std::vector<size_t> hpart;
    for (size_t i = 0; i < parts.size(); i++) {
        Part& pt = parts[i];
        if (shared != nullptr) {
            auto it = shared->find({pt.host, pt.n});
            if (it != shared->end()) {
                *pt.dst = it->second.buf;
                pt.hash[0] = it->second.hash[0];
                pt.hash[1] = it->second.hash[1];
                continue;
            }
        }
        *pt.dst = std::make_shared<DevBuf>();
        upload(ctx, **pt.dst, pt.host, (size_t)pt.n);
        hdata.push_back((*pt.dst)->as<int32_t>());
        hn.push_back(pt.n);
        hpart.push_back(i);
    }
    std::vector<uint64_t> hh(2 * hdata.size());
    hash_device_many(ctx, hdata, hn, std::vector<uint64_t>(hdata.size(), 0), hh.data());
    for (size_t k = 0; k < hpart.size(); k++) {
        Part& pt = parts[hpart[k]];
        pt.hash[0] = hh[2 * k];
        pt.hash[1] = hh[2 * k + 1];
        if (shared != nullptr)
            (*shared)[{pt.host, pt.n}] = Matrix::SharedAddresses{*pt.dst, {pt.hash[0], pt.hash[1]}};
    }
    uint64_t h0 = 0, h1 = 0;
    for (const Part& pt : parts) {
        h0 = mix64(h0 ^ mix64(pt.hash[0] ^ pt.salt * 0x9E3779B97F4A7C15ull));
        h1 = mix64(h1 ^ mix64(pt.hash[1] + pt.salt));
    }
    gd->addr_hash[0] = mix64(h0 ^ (uint64_t)g.ntf << 40 ^ (uint64_t)g.ndof << 20 ^ (uint64_t)g.nelem);
    gd->addr_hash[1] = mix64(h1 ^ (uint64_t)g.ndests << 32 ^ (uint64_t)gd->rhs);
    return gd;
}

// ------------------------------------------------------------ launches
static CoefParams coef_params(Ctx* ctx, const GroupDev& g, double* C)
{
    const MeshDev& m = ctx->meshes.at(g.mesh);
    const MeshDev::Type& t = m.types.at(g.elemtype);
    CoefParams p{};
    p.xyz = m.xyz.as<double>();
    p.conn = t.conn.as<int32_t>();
    p.ncn = g.ncn;
    p.elems = g.elems.as<int32_t>();
    p.orient = g.orient.as<int32_t>();
    p.nelem = g.nelem;
    p.ngp = g.ngp;
    p.weights = g.weights.as<double>();
    p.lagrange = g.lagrange.as<double>();
    p.dim = g.problemdim;
    p.edim = g.elemdim;
    p.prog = g.prog_d.as<Instr>();
    p.nprog = (int)g.prog.size();
    p.consts = g.consts.as<double>();
    p.tables = g.tables.as<double>();
    p.tab_off = g.tab_off_d.as<int64_t>();
    p.tab_rows = g.tab_rows_d.as<int32_t>();
    p.elemdata = g.elemdata.as<double>();
    p.fielddata = g.fielddata.as<double>();
    p.field_off = g.field_off_d.as<int64_t>();
    p.term_scale = g.term_scale_d.as<double>();
    p.nterms = g.nterms;
    p.C = C;
    return p;
}

// Segments of the COO space: (group, destination) blocks then raw fragments.
std::vector<Segment> build_segments(const Matrix& M, std::vector<int64_t>* group_val_base, int64_t* total_vals, bool f32)
{
    std::vector<Segment> segs;
    int64_t coo = 0, vb = 0;
    group_val_base->clear();
    for (auto& g : M.groups) {
        const int64_t P = (int64_t)g->ntf * g->ndof;
        group_val_base->push_back(vb);
        for (int d = 0; d < g->ndests; d++) {
            segs.push_back(Segment{coo, P * g->nelem, vb, g->dest_mult[d]});
            coo += P * g->nelem;
        }
        // Float values take half as many doubles of the buffer.
        vb += f32 ? (P * g->nelem + 1) / 2 : P * g->nelem;
    }
    for (auto& f : M.frags) {
        const int64_t n = (int64_t)f->nr * f->nc;
        segs.push_back(Segment{coo, n, vb, 1.0});
        coo += n;
        vb += n;
    }
    *total_vals = vb;
    return segs;
}

void stage_reset(Exec& x) { x.stage_used = 0; }

void stage_free(Exec& x)
{
    if (x.stage != nullptr)
        cudaFreeHost(x.stage);
    for (char* p : x.stage_old) cudaFreeHost(p);
    x.stage = nullptr;
    x.stage_old.clear();
    x.stage_bytes = x.stage_used = 0;
}

void upload_staged(Ctx* ctx, DevBuf& buf, const void* src, size_t bytes)
{
    buf.alloc(ctx, bytes);
    upload_staged_into(ctx, buf.as<void>(), src, bytes);
}

void upload_staged_into(Ctx* ctx, void* dst, const void* src, size_t bytes)
{
    Exec& x = *ctx->x;
    if (bytes == 0)
        return;
    const size_t need = (bytes + 255) & ~size_t(255);
    if (x.stage_used + need > x.stage_bytes) {
        // Grow; the old block may still be read by queued copies of this
        // call, so it is kept until the state is freed.
        if (x.stage != nullptr)
            x.stage_old.push_back(x.stage);
        x.stage = nullptr;
        const size_t nb = std::max<size_t>(need, std::max<size_t>(2 * x.stage_bytes, 1 << 16));
        cuda_check(cudaHostAlloc(reinterpret_cast<void**>(&x.stage), nb, cudaHostAllocDefault), "cudaHostAlloc staging");
        x.stage_bytes = nb;
        x.stage_used = 0;
    }
    char* p = x.stage + x.stage_used;
    x.stage_used += need;
    std::memcpy(p, src, bytes);
    cuda_check(cudaMemcpyAsync(dst, p, bytes, cudaMemcpyHostToDevice, x.stream), "cudaMemcpyAsync H2D staged");
}

namespace {
struct HostTrace {
    bool on = false;
    std::mutex mu;
    struct Acc {
        double total = 0, max = 0;
        int64_t n = 0;
    };
    std::map<std::string, Acc> acc;
    HostTrace()
    {
        const char* v = std::getenv("SLGPU_HOST_TRACE");
        on = v != nullptr && std::strcmp(v, "1") == 0;
    }
    ~HostTrace()
    {
        if (!on || acc.empty())
            return;
        std::fprintf(stderr, "slgpu host trace (label: calls, mean us, max us, total ms)\n");
        for (auto& [k, v] : acc)
            std::fprintf(stderr, "  %-30s %9lld %10.2f %10.2f %10.2f\n", k.c_str(), (long long)v.n, v.total * 1e6 / std::max<int64_t>(v.n, 1),
                         v.max * 1e6, v.total * 1e3);
    }
};
HostTrace g_htrace;
double host_seconds() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }
}  // namespace

void htrace_begin(Ctx* ctx)
{
    if (g_htrace.on)
        ctx->x->trace_t = host_seconds();
}

void htrace_mark(Ctx* ctx, const char* label)
{
    if (!g_htrace.on)
        return;
    const double t = host_seconds();
    {
        std::lock_guard<std::mutex> lk(g_htrace.mu);
        auto& a = g_htrace.acc[label];
        a.total += t - ctx->x->trace_t;
        a.max = std::max(a.max, t - ctx->x->trace_t);
        a.n++;
    }
    ctx->x->trace_t = t;
}

// Kernel-family timers: kstat_start/kstat_stop bracket launches with an
// event pair; kstat_collect sums them once the stream has been synchronised.
int kstat_start(Ctx* ctx, const char* family, double work)
{
    if (!ctx->timers)
        return -1;
    const size_t i = ctx->x->kev_tag.size();
    while (ctx->x->kev.size() < 2 * (i + 1)) {
        cudaEvent_t e;
        cuda_check(cudaEventCreate(&e), "cudaEventCreate");
        ctx->x->kev.push_back(e);
    }
    record_event(ctx, ctx->x->kev[2 * i]);
    ctx->x->kev_tag.emplace_back(family, work);
    return (int)i;
}

void kstat_stop(Ctx* ctx, int i)
{
    if (i >= 0)
        record_event(ctx, ctx->x->kev[2 * i + 1]);
}

// Phase boundary events (within a process()), recorded only with timers on.
static void phase_event(Ctx* ctx, cudaEvent_t e)
{
    if (ctx->timers)
        record_event(ctx, e);
}

void record_event(Ctx* ctx, cudaEvent_t e)
{
    const cudaError_t err = ctx->x->capturing ? cudaEventRecordWithFlags(e, ctx->x->stream, cudaEventRecordExternal)
                                              : cudaEventRecord(e, ctx->x->stream);
    cuda_check(err, "cudaEventRecord");
}

void kstat_collect(Ctx* ctx)
{
    ctx->x->kstats.clear();
    for (size_t i = 0; i < ctx->x->kev_tag.size(); i++) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->x->kev[2 * i], ctx->x->kev[2 * i + 1]);
        KernelStat& k = ctx->x->kstats[ctx->x->kev_tag[i].first];
        k.ms += ms;
        k.work += ctx->x->kev_tag[i].second;
        k.launches++;
    }
    ctx->x->kev_tag.clear();
}

static void ev_record(Ctx* ctx, int i) { record_event(ctx, ctx->x->ev[i]); }

static float ev_ms(Ctx* ctx, int a, int b)
{
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->x->ev[a], ctx->x->ev[b]);
    return ms;
}

static int bits_for(int64_t n)
{
    int b = 1;
    while ((int64_t(1) << b) <= n) b++;
    return b;
}

// Builds (or fetches) the pattern for matrix M with the given constraints
// (all-zero constraints for a right-hand side, which has one column).
static std::shared_ptr<Pattern> get_pattern(Ctx* ctx, Matrix& M, const std::vector<Segment>& segs, const uint8_t* dconstr,
                                            bool rhs, uint64_t key0, uint64_t key1, bool* reused)
{
    for (auto& p : ctx->patterns) {
        if (p->key[0] == key0 && p->key[1] == key1 && p->ndofs == M.ndofs) {
            p->last_use = ++ctx->use_clock;
            *reused = true;
            return p;
        }
    }
    *reused = false;
    auto P = std::make_shared<Pattern>();
    P->key[0] = key0;
    P->key[1] = key1;
    P->serial = ++ctx->pattern_serial;
    P->ndofs = M.ndofs;
    const int64_t ncoo = segs.empty() ? 0 : segs.back().coo_base + segs.back().count;
    P->ncoo = ncoo;
    if (ncoo >= (int64_t)0xFFFFFFFFll)
        fail(SLGPU_E_UNSUPPORTED, "more than 2^32-1 COO entries in one matrix");
    const int rowbits = bits_for(M.ndofs);
    const int colbits = rhs ? 0 : bits_for(M.ndofs);
    if (rowbits + colbits > 64)
        fail(SLGPU_E_UNSUPPORTED, "too many DOFs for 64-bit keys");
    const uint64_t invalid = (rowbits + colbits == 64) ? ~0ull : ((1ull << (rowbits + colbits)) - 1);
    size_t temp = 0;
    DevBuf tmp;

    // ---- COO keys in COO order, stable radix sort on the used bits.
    DevBuf keys, keys_alt, idx, idx_alt, counter;
    keys.alloc(ctx, std::max<int64_t>(ncoo, 1) * 8);
    keys_alt.alloc(ctx, std::max<int64_t>(ncoo, 1) * 8);
    idx.alloc(ctx, std::max<int64_t>(ncoo, 1) * 4);
    idx_alt.alloc(ctx, std::max<int64_t>(ncoo, 1) * 4);
    counter.alloc(ctx, 16);
    cuda_check(cudaMemsetAsync(counter.as<void>(), 0, 16, ctx->x->stream), "memset");
    int si = 0;
    for (auto& g : M.groups) {
        for (int d = 0; d < g->ndests; d++, si++) {
            KeyParams kp{};
            kp.tfaddr = g->tfaddr[d]->as<int32_t>();
            kp.dofaddr = rhs ? nullptr : g->dofaddr[d]->as<int32_t>();
            kp.ndof = g->ndof;
            kp.ntf = g->ntf;
            kp.nelem = g->nelem;
            kp.count = segs[si].count;
            kp.coo_base = segs[si].coo_base;
            kp.ndofs = M.ndofs;
            kp.colbits = colbits;
            kp.constrained = dconstr;
            kp.invalid = invalid;
            kp.keys = keys.as<unsigned long long>();
            kp.idx = idx.as<uint32_t>();
            kp.nvalid = counter.as<unsigned long long>();
            if (kp.count > 0) {
                k_group_keys<<<grid_for(kp.count, 256), 256, 0, ctx->x->stream>>>(kp);
                cuda_check(cudaGetLastError(), "k_group_keys");
            }
        }
    }
    for (auto& f : M.frags) {
        FragKeyParams fp{};
        fp.rows = f->rows.as<int32_t>();
        fp.cols = f->cols.as<int32_t>();
        fp.ntr = f->ntr;
        fp.ndr = f->ndr;
        fp.nr = f->nr;
        fp.nc = f->nc;
        fp.coo_base = segs[si].coo_base;
        fp.colbits = colbits;
        fp.constrained = dconstr;
        fp.invalid = invalid;
        fp.keys = keys.as<unsigned long long>();
        fp.idx = idx.as<uint32_t>();
        fp.nvalid = counter.as<unsigned long long>();
        fp.ndofs = M.ndofs;
        k_frag_keys<<<grid_for((int64_t)f->nr * f->nc, 256), 256, 0, ctx->x->stream>>>(fp);
        cuda_check(cudaGetLastError(), "k_frag_keys");
        si++;
    }
    cub::DoubleBuffer<unsigned long long> dk(keys.as<unsigned long long>(), keys_alt.as<unsigned long long>());
    cub::DoubleBuffer<uint32_t> dv(idx.as<uint32_t>(), idx_alt.as<uint32_t>());
    cuda_check(cub::DeviceRadixSort::SortPairs(nullptr, temp, dk, dv, (int64_t)ncoo, 0, rowbits + colbits, ctx->x->stream),
               "SortPairs size");
    tmp.alloc(ctx, temp);
    cuda_check(cub::DeviceRadixSort::SortPairs(tmp.as<void>(), temp, dk, dv, (int64_t)ncoo, 0, rowbits + colbits, ctx->x->stream),
               "SortPairs");
    tmp.release();
    unsigned long long counts_h[2] = {0, 0};
    cuda_check(cudaMemcpyAsync(counts_h, counter.as<void>(), 16, cudaMemcpyDeviceToHost, ctx->x->stream), "D2H nvalid");
    cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync nvalid");
    if (counts_h[1] != 0)
        fail(SLGPU_E_ARG, std::to_string(counts_h[1]) + " COO addresses are >= the DOF count");
    const int64_t nvalid = (int64_t)counts_h[0];
    P->nvalid = nvalid;
    const unsigned long long* sk = dk.Current();
    const uint32_t* perm = dv.Current();

    // ---- runs (one per CSR entry).
    DevBuf head, runidx;
    head.alloc(ctx, std::max<int64_t>(nvalid, 1) * 4);
    runidx.alloc(ctx, std::max<int64_t>(nvalid, 1) * 4);
    if (nvalid > 0) {
        k_run_heads<<<grid_for(nvalid, 256), 256, 0, ctx->x->stream>>>(sk, nvalid, head.as<uint32_t>());
        cuda_check(cudaGetLastError(), "k_run_heads");
        temp = 0;
        cuda_check(cub::DeviceScan::ExclusiveSum(nullptr, temp, head.as<uint32_t>(), runidx.as<uint32_t>(), (int64_t)nvalid, ctx->x->stream),
                   "scan size");
        tmp.alloc(ctx, temp);
        cuda_check(cub::DeviceScan::ExclusiveSum(tmp.as<void>(), temp, head.as<uint32_t>(), runidx.as<uint32_t>(), (int64_t)nvalid,
                                                 ctx->x->stream),
                   "scan");
        tmp.release();
    }
    uint32_t last[2] = {0, 0};
    if (nvalid > 0) {
        cuda_check(cudaMemcpyAsync(&last[0], runidx.as<uint32_t>() + nvalid - 1, 4, cudaMemcpyDeviceToHost, ctx->x->stream), "D2H");
        cuda_check(cudaMemcpyAsync(&last[1], head.as<uint32_t>() + nvalid - 1, 4, cudaMemcpyDeviceToHost, ctx->x->stream), "D2H");
        cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync");
    }
    const int64_t nruns = nvalid > 0 ? (int64_t)last[0] + last[1] : 0;
    DevBuf run_start;
    run_start.alloc(ctx, (nruns + 1) * 4);
    if (nvalid > 0) {
        k_run_starts<<<grid_for(nvalid, 256), 256, 0, ctx->x->stream>>>(head.as<uint32_t>(), runidx.as<uint32_t>(), nvalid,
                                                                     run_start.as<uint32_t>());
        cuda_check(cudaGetLastError(), "k_run_starts");
    }

    // ---- local renumbering of constrained / unconstrained DOFs.
    DevBuf renum;
    renum.alloc(ctx, std::max<int64_t>(M.ndofs, 1) * 4);
    int64_t nA = 0, nD = 0;
    {
        DevBuf flagsA, scanA, flagsD, scanD;
        flagsA.alloc(ctx, (M.ndofs + 1) * 4);
        flagsD.alloc(ctx, (M.ndofs + 1) * 4);
        scanA.alloc(ctx, (M.ndofs + 1) * 4);
        scanD.alloc(ctx, (M.ndofs + 1) * 4);
        k_constraint_flags<<<grid_for(M.ndofs + 1, 256), 256, 0, ctx->x->stream>>>(dconstr, M.ndofs, flagsA.as<uint32_t>(),
                                                                                 flagsD.as<uint32_t>());
        cuda_check(cudaGetLastError(), "k_constraint_flags");
        temp = 0;
        cuda_check(cub::DeviceScan::ExclusiveSum(nullptr, temp, flagsA.as<uint32_t>(), scanA.as<uint32_t>(), (int64_t)M.ndofs + 1,
                                                 ctx->x->stream),
                   "scan size");
        tmp.alloc(ctx, temp);
        cuda_check(cub::DeviceScan::ExclusiveSum(tmp.as<void>(), temp, flagsA.as<uint32_t>(), scanA.as<uint32_t>(), (int64_t)M.ndofs + 1,
                                                 ctx->x->stream),
                   "scan");
        cuda_check(cub::DeviceScan::ExclusiveSum(tmp.as<void>(), temp, flagsD.as<uint32_t>(), scanD.as<uint32_t>(), (int64_t)M.ndofs + 1,
                                                 ctx->x->stream),
                   "scan");
        tmp.release();
        uint32_t tot[2];
        cuda_check(cudaMemcpyAsync(&tot[0], scanA.as<uint32_t>() + M.ndofs, 4, cudaMemcpyDeviceToHost, ctx->x->stream), "D2H");
        cuda_check(cudaMemcpyAsync(&tot[1], scanD.as<uint32_t>() + M.ndofs, 4, cudaMemcpyDeviceToHost, ctx->x->stream), "D2H");
        k_renumber<<<grid_for(M.ndofs, 256), 256, 0, ctx->x->stream>>>(dconstr, M.ndofs, scanA.as<uint32_t>(), scanD.as<uint32_t>(),
                                                                     renum.as<int32_t>());
        cuda_check(cudaGetLastError(), "k_renumber");
        cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync");
        nA = tot[0];
        nD = tot[1];
        P->ainds.alloc(ctx, std::max<int64_t>(nA, 1) * 4);
        P->dinds.alloc(ctx, std::max<int64_t>(nD, 1) * 4);
        if (M.ndofs > 0) {
            k_dof_split<<<grid_for(M.ndofs, 256), 256, 0, ctx->x->stream>>>(dconstr, M.ndofs, scanA.as<uint32_t>(), scanD.as<uint32_t>(),
                                                                          P->ainds.as<int32_t>(), P->dinds.as<int32_t>());
            cuda_check(cudaGetLastError(), "k_dof_split");
        }
    }
    P->nA = nA;
    P->nD = nD;

    // ---- A / D classification, CSR structure, slot of every run.
    DevBuf run_target;
    run_target.alloc(ctx, std::max<int64_t>(nruns, 1) * 4);
    {
        DevBuf isA, slotA, slotD, isD, rowcA, rowcD;
        isA.alloc(ctx, (nruns + 1) * 4);
        isD.alloc(ctx, (nruns + 1) * 4);
        slotA.alloc(ctx, (nruns + 1) * 4);
        slotD.alloc(ctx, (nruns + 1) * 4);
        rowcA.alloc(ctx, (nA + 1) * 4);
        rowcD.alloc(ctx, (nA + 1) * 4);
        cuda_check(cudaMemsetAsync(rowcA.as<void>(), 0, (nA + 1) * 4, ctx->x->stream), "memset");
        cuda_check(cudaMemsetAsync(rowcD.as<void>(), 0, (nA + 1) * 4, ctx->x->stream), "memset");
        k_classify_runs<<<grid_for(nruns + 1, 256), 256, 0, ctx->x->stream>>>(sk, run_start.as<uint32_t>(), nruns, colbits, dconstr,
                                                                            renum.as<int32_t>(), isA.as<uint32_t>(), isD.as<uint32_t>(),
                                                                            rowcA.as<uint32_t>(), rowcD.as<uint32_t>());
        cuda_check(cudaGetLastError(), "k_classify_runs");
        temp = 0;
        cuda_check(cub::DeviceScan::ExclusiveSum(nullptr, temp, isA.as<uint32_t>(), slotA.as<uint32_t>(), (int64_t)nruns + 1, ctx->x->stream),
                   "scan size");
        size_t temp2 = 0;
        cuda_check(cub::DeviceScan::ExclusiveSum(nullptr, temp2, rowcA.as<uint32_t>(), rowcA.as<uint32_t>(), (int64_t)nA + 1, ctx->x->stream),
                   "scan size");
        temp = std::max(temp, temp2);
        tmp.alloc(ctx, temp);
        cuda_check(cub::DeviceScan::ExclusiveSum(tmp.as<void>(), temp, isA.as<uint32_t>(), slotA.as<uint32_t>(), (int64_t)nruns + 1,
                                                 ctx->x->stream),
                   "scan");
        cuda_check(cub::DeviceScan::ExclusiveSum(tmp.as<void>(), temp, isD.as<uint32_t>(), slotD.as<uint32_t>(), (int64_t)nruns + 1,
                                                 ctx->x->stream),
                   "scan");
        P->Arows.alloc(ctx, (nA + 1) * 4);
        P->Drows.alloc(ctx, (nA + 1) * 4);
        cuda_check(cub::DeviceScan::ExclusiveSum(tmp.as<void>(), temp, rowcA.as<uint32_t>(), P->Arows.as<uint32_t>(), (int64_t)nA + 1,
                                                 ctx->x->stream),
                   "scan");
        cuda_check(cub::DeviceScan::ExclusiveSum(tmp.as<void>(), temp, rowcD.as<uint32_t>(), P->Drows.as<uint32_t>(), (int64_t)nA + 1,
                                                 ctx->x->stream),
                   "scan");
        tmp.release();
        uint32_t tot[2];
        cuda_check(cudaMemcpyAsync(&tot[0], slotA.as<uint32_t>() + nruns, 4, cudaMemcpyDeviceToHost, ctx->x->stream), "D2H");
        cuda_check(cudaMemcpyAsync(&tot[1], slotD.as<uint32_t>() + nruns, 4, cudaMemcpyDeviceToHost, ctx->x->stream), "D2H");
        cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync");
        P->nnzA = tot[0];
        P->nnzD = tot[1];
        if (P->nnzA >= (int64_t(1) << 31) || P->nnzD >= (int64_t(1) << 31))
            fail(SLGPU_E_UNSUPPORTED, "more than 2^31-1 nonzeros in a CSR block (32-bit PETSc row pointers)");
        P->Acols.alloc(ctx, std::max<int64_t>(P->nnzA, 1) * 4);
        P->Dcols.alloc(ctx, std::max<int64_t>(P->nnzD, 1) * 4);
        if (nruns > 0) {
            k_fill_runs<<<grid_for(nruns, 256), 256, 0, ctx->x->stream>>>(sk, run_start.as<uint32_t>(), nruns, colbits, isA.as<uint32_t>(),
                                                                        slotA.as<uint32_t>(), slotD.as<uint32_t>(), renum.as<int32_t>(),
                                                                        run_target.as<int32_t>(), P->Acols.as<int32_t>(),
                                                                        P->Dcols.as<int32_t>());
            cuda_check(cudaGetLastError(), "k_fill_runs");
        }
    }
    run_start.release();

    // ---- slot map: position of each kept COO entry inside its row segment.
    P->slotmap.alloc(ctx, std::max<int64_t>(ncoo, 1) * 2);
    cuda_check(cudaMemsetAsync(P->slotmap.as<void>(), 0xFF, std::max<int64_t>(ncoo, 1) * 2, ctx->x->stream), "memset slotmap");
    cuda_check(cudaMemsetAsync(counter.as<void>(), 0, 16, ctx->x->stream), "memset");
    std::vector<CooSeg> csegs;
    {
        size_t s = 0;
        for (auto& g : M.groups)
            for (int d = 0; d < g->ndests; d++, s++) csegs.push_back(CooSeg{segs[s].coo_base, (int64_t)std::max(1, g->ndof)});
        for (size_t f = 0; f < M.frags.size(); f++, s++) csegs.push_back(CooSeg{segs[s].coo_base, 1});
    }
    DevBuf dcsegs, dup;
    upload(ctx, dcsegs, csegs);
    dup.alloc(ctx, std::max<int64_t>(ncoo, 1));
    cuda_check(cudaMemsetAsync(dup.as<void>(), 0, std::max<int64_t>(ncoo, 1), ctx->x->stream), "memset dup");
    if (nvalid > 0) {
        k_slotmap<<<grid_for(nvalid, 256), 256, 0, ctx->x->stream>>>(sk, perm, head.as<uint32_t>(), runidx.as<uint32_t>(), nvalid, colbits,
                                                                  run_target.as<int32_t>(), renum.as<int32_t>(), P->Arows.as<uint32_t>(),
                                                                  P->Drows.as<uint32_t>(), P->slotmap.as<int16_t>(),
                                                                  counter.as<unsigned long long>(), dcsegs.as<CooSeg>(), (int)csegs.size(),
                                                                  dup.as<uint8_t>());
        cuda_check(cudaGetLastError(), "k_slotmap");
    }
    head.release();
    runidx.release();
    run_target.release();
    keys.release();
    keys_alt.release();
    idx.release();
    idx_alt.release();

    // ---- incidences: element-matrix rows (or fragment entries) grouped by row.
    std::vector<IncSeg> isegs;
    int64_t ninc_total = 0;
    si = 0;
    for (auto& g : M.groups) {
        for (int d = 0; d < g->ndests; d++, si++) {
            IncSeg s{};
            s.inc_base = ninc_total;
            s.count = g->nelem * (int64_t)g->ntf;
            s.coo_base = segs[si].coo_base;
            s.val_base = segs[si].val_base;
            s.mult = segs[si].mult;
            s.width = g->ndof;
            s.ntf = g->ntf;
            s.kind = 0;
            s.nelem = g->nelem;
            s.rows = g->tfaddr[d]->as<int32_t>();
            isegs.push_back(s);
            ninc_total += s.count;
        }
    }
    for (auto& f : M.frags) {
        IncSeg s{};
        s.inc_base = ninc_total;
        s.count = (int64_t)f->nr * f->nc;
        s.coo_base = segs[si].coo_base;
        s.val_base = segs[si].val_base;
        s.mult = 1.0;
        s.width = 1;
        s.kind = 1;
        s.ntr = f->ntr;
        s.ndr = f->ndr;
        s.nr = f->nr;
        s.nc = f->nc;
        s.rows = f->rows.as<int32_t>();
        s.cols = f->cols.as<int32_t>();
        isegs.push_back(s);
        ninc_total += s.count;
        si++;
    }
    if (ninc_total >= (int64_t)0xFFFFFFFFll)
        fail(SLGPU_E_UNSUPPORTED, "more than 2^32-1 element-matrix rows in one matrix");
    DevBuf disegs;
    upload(ctx, disegs, isegs);
    DevBuf ikeys, ikeys_alt, iids, iids_alt;
    ikeys.alloc(ctx, std::max<int64_t>(ninc_total, 1) * 4);
    ikeys_alt.alloc(ctx, std::max<int64_t>(ninc_total, 1) * 4);
    iids.alloc(ctx, std::max<int64_t>(ninc_total, 1) * 4);
    iids_alt.alloc(ctx, std::max<int64_t>(ninc_total, 1) * 4);
    for (size_t s = 0; s < isegs.size(); s++) {
        if (isegs[s].count == 0)
            continue;
        k_inc_keys<<<grid_for(isegs[s].count, 256), 256, 0, ctx->x->stream>>>(disegs.as<IncSeg>(), (int)s, dconstr, M.ndofs,
                                                                          ikeys.as<uint32_t>(), iids.as<uint32_t>(),
                                                                          counter.as<unsigned long long>() + 1);
        cuda_check(cudaGetLastError(), "k_inc_keys");
    }
    cub::DoubleBuffer<uint32_t> ik(ikeys.as<uint32_t>(), ikeys_alt.as<uint32_t>());
    cub::DoubleBuffer<uint32_t> iv(iids.as<uint32_t>(), iids_alt.as<uint32_t>());
    temp = 0;
    cuda_check(cub::DeviceRadixSort::SortPairs(nullptr, temp, ik, iv, (int64_t)ninc_total, 0, 32, ctx->x->stream), "SortPairs size");
    tmp.alloc(ctx, temp);
    cuda_check(cub::DeviceRadixSort::SortPairs(tmp.as<void>(), temp, ik, iv, (int64_t)ninc_total, 0, 32, ctx->x->stream), "SortPairs");
    tmp.release();
    cuda_check(cudaMemcpyAsync(counts_h, counter.as<void>(), 16, cudaMemcpyDeviceToHost, ctx->x->stream), "D2H");
    cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync");
    if (counts_h[0] != 0)
        fail(SLGPU_E_UNSUPPORTED, "a CSR row is longer than 32767 entries");
    const int64_t ninc = (int64_t)counts_h[1];
    P->ninc = ninc;
    P->inc.alloc(ctx, std::max<int64_t>(ninc, 1) * 8);
    DevBuf rowcount;
    rowcount.alloc(ctx, (nA + 1) * 4);
    cuda_check(cudaMemsetAsync(rowcount.as<void>(), 0, (nA + 1) * 4, ctx->x->stream), "memset");
    if (isegs.size() >= (size_t(1) << 23))
        fail(SLGPU_E_UNSUPPORTED, "too many element groups and fragments in one matrix");
    if (ninc > 0) {
        k_inc_finalize<<<grid_for(ninc, 256), 256, 0, ctx->x->stream>>>(ik.Current(), iv.Current(), ninc, disegs.as<IncSeg>(),
                                                                     (int)isegs.size(), renum.as<int32_t>(), dup.as<uint8_t>(),
                                                                     P->inc.as<unsigned long long>(), rowcount.as<uint32_t>());
        cuda_check(cudaGetLastError(), "k_inc_finalize");
    }
    dup.release();
    P->inc_ptr.alloc(ctx, (nA + 1) * 4);
    temp = 0;
    cuda_check(cub::DeviceScan::ExclusiveSum(nullptr, temp, rowcount.as<uint32_t>(), P->inc_ptr.as<uint32_t>(), (int64_t)nA + 1, ctx->x->stream),
               "scan size");
    tmp.alloc(ctx, temp);
    cuda_check(cub::DeviceScan::ExclusiveSum(tmp.as<void>(), temp, rowcount.as<uint32_t>(), P->inc_ptr.as<uint32_t>(), (int64_t)nA + 1,
                                             ctx->x->stream),
               "scan");
    tmp.release();
    // Longest row.
    cuda_check(cudaMemsetAsync(counter.as<void>(), 0, 16, ctx->x->stream), "memset");
    if (nA > 0) {
        k_max_rowlen<<<grid_for(nA, 256), 256, 0, ctx->x->stream>>>(P->Arows.as<uint32_t>(), P->Drows.as<uint32_t>(), nA,
                                                                   counter.as<unsigned long long>());
        cuda_check(cudaGetLastError(), "k_max_rowlen");
    }
    cuda_check(cudaMemcpyAsync(counts_h, counter.as<void>(), 16, cudaMemcpyDeviceToHost, ctx->x->stream), "D2H");
    cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync");
    P->lmax = (int)counts_h[0];

    P->last_use = ++ctx->use_clock;
    ctx->patterns.push_back(P);
    // Keep at most 8 resident patterns (least recently used evicted).
    while (ctx->patterns.size() > 8) {
        auto it = std::min_element(ctx->patterns.begin(), ctx->patterns.end(),
                                   [](const std::shared_ptr<Pattern>& a, const std::shared_ptr<Pattern>& b) { return a->last_use < b->last_use; });
        ctx->patterns.erase(it);
    }
    return P;
}

// ------------------------------------------------------------ split precision (host side)

// Tier 0: 7 slices, levels <= 8 (28 INT8 products; about 1e-12 relative per
// element matrix, well inside 1e-10); tier 1: 5 slices, levels <= 6 (15
// products; about 1e-8, inside the FP32-level 1e-6).
// Whether the split contraction of a group computes only the upper triangle
// of its element matrices: the group has mirror terms with equal scales
// (SLGPU_SPLIT_SYMMETRY=0 turns this off).
static bool mirror_forms_enabled()
{
    static const bool enabled = [] {
        const char* v = std::getenv("SLGPU_SPLIT_SYMMETRY");
        return v == nullptr || std::strcmp(v, "0") != 0;
    }();
    return enabled;
}

static bool symmetric_form(const GroupDev& g)
{
    if (!mirror_forms_enabled() || g.mirror.empty())
        return false;
    for (int t = 0; t < g.nterms; t++)
        if (std::memcmp(&g.term_scale[t], &g.term_scale[g.mirror[t]], sizeof(double)) != 0)
            return false;
    return true;
}

bool group_symmetric(const GroupDev& g) { return symmetric_form(g); }

// Rows of A for the mirrored forms (the upper triangle of a symmetric group,
// or every entry of a group with a transposed partner), each with the entry
// it is and the entry its value also goes to: (j, i) of the same matrix, or
// (j, i) of the partner's.  They come in blocks of 4 rows i by 8 columns j
// (row-major inside a block), so that a warp's 32 stores of one element
// cover 4 runs of 8 entries and their mirrors 8 runs of 4, rather than one
// run of 32 and 32 scattered entries.
static std::vector<int2> mirrored_rows(int ntf, int ndof, bool upper)
{
    std::vector<int2> map;
    for (int bi = 0; bi < ntf; bi += 4)
        for (int bj = 0; bj < ndof; bj += 8)
            for (int i = bi; i < std::min(bi + 4, ntf); i++)
                for (int j = bj; j < std::min(bj + 8, ndof); j++)
                    if (!upper || j >= i)
                        map.push_back(make_int2(i * ndof + j, j * ntf + i));
    return map;
}

// Row slices of a group for a tier (0 split, 1 FP32 level) and form (0 every
// entry, 1 upper triangle of a symmetric group, 2 every entry with its
// transposed partner's): slot tier + 2 form.
static GroupDev::Split& build_split(Ctx* ctx, GroupDev& g, int slot)
{
    std::unique_ptr<GroupDev::Split>& sp = g.split[slot];
    if (sp)
        return *sp;
    const int tier = slot & 1, form = slot >> 1;
    sp.reset(new GroupDev::Split());
    sp->S = tier == 0 ? 7 : 5;
    sp->L = tier == 0 ? 8 : 6;
    const int Q = g.nterms * g.ngp, P = g.ntf * g.ndof;
    sp->Qpad = std::max(kSplitKStep, (Q + kSplitKStep - 1) / kSplitKStep * kSplitKStep);
    sp->nrows = form == 1 ? g.ntf * (g.ntf + 1) / 2 : P;
    sp->Ppad = (sp->nrows + kSplitM - 1) / kSplitM * kSplitM;
    if (form != 0)
        upload(ctx, sp->rowmap, mirrored_rows(g.ntf, g.ndof, form == 1));
    sp->slices.alloc(ctx, (size_t)sp->S * g.norient * sp->Qpad * sp->Ppad);
    sp->rowexp.alloc(ctx, (size_t)g.norient * sp->Ppad * 4);
    RowSliceParams rp{};
    rp.rowmap = sp->rowmap.empty() ? nullptr : sp->rowmap.as<int2>();
    rp.nrows = sp->nrows;
    rp.tables = g.tables.as<double>();
    rp.tab_off = g.tab_off_d.as<int64_t>();
    rp.term_tf = g.term_tf_d.as<int32_t>();
    rp.term_dof = g.term_dof_d.as<int32_t>();
    rp.nterms = g.nterms;
    rp.ngp = g.ngp;
    rp.ntf = g.ntf;
    rp.ndof = g.ndof;
    rp.norient = g.norient;
    rp.S = sp->S;
    rp.Qpad = sp->Qpad;
    rp.Ppad = sp->Ppad;
    rp.slices = sp->slices.as<int8_t>();
    rp.rowexp = sp->rowexp.as<int32_t>();
    if (g.norient > 65535)
        fail(SLGPU_E_UNSUPPORTED, "too many orientation variants");
    k_slice_rows<<<dim3((unsigned)sp->Ppad, (unsigned)g.norient), 256, 0, ctx->x->stream>>>(rp);
    cuda_check(cudaGetLastError(), "k_slice_rows");
    ctx->launches++;
    return *sp;
}

// The row slices are resident with the group, so they are built in the main
// execution state's stream order; a request stream waits for them.
static GroupDev::Split& ensure_split(Ctx* ctx, GroupDev& g, int tier, bool paired)
{
    const int slot = tier + 2 * (paired ? 2 : symmetric_form(g) ? 1 : 0);
    if (g.split[slot])
        return *g.split[slot];
    Exec* cur = ctx->x;
    ctx->x = &ctx->main;
    try {
        build_split(ctx, g, slot);
    } catch (...) {
        ctx->x = cur;
        throw;
    }
    ctx->x = cur;
    if (cur != &ctx->main) {
        cudaEvent_t e;
        cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
        cuda_check(cudaEventRecord(e, ctx->main.stream), "cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(cur->stream, e, 0), "cudaStreamWaitEvent");
        cudaEventDestroy(e);
    }
    return *g.split[slot];
}

// Whether a group's contraction can take the split path: level sums stay
// below 2^31 (at most 7 * Qpad * 127^2) and the integer recombination stays
// exact in FP64.
static bool split_supported(const GroupDev& g)
{
    const int64_t Q = (int64_t)g.nterms * g.ngp;
    return Q > 0 && Q <= 16384;
}

template <int S, int L, int NE>
static void launch_split(Ctx* ctx, const SplitParams& p)
{
    static bool attr = false;
    constexpr size_t smem = split_smem_bytes<NE>();
    if (!attr) {
        cuda_check(cudaFuncSetAttribute(k_contract_split<S, L, NE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                   "smem attribute");
        attr = true;
    }
    const int64_t grid = std::min<int64_t>(p.nwork, std::max(ctx->nsm, 1));
    cuda_check(cudaMemsetAsync(p.next, 0, sizeof(unsigned long long), ctx->x->stream), "memset");
    k_contract_split<S, L, NE><<<(unsigned)grid, kSplitThreads, smem, ctx->x->stream>>>(p);
}

// Element-tile width of the split kernel forced by SLGPU_SPLIT_TILE=32 or 64;
// 0: picked per group shape by timing (tile_choice).
static int split_tile_forced()
{
    static const int ne = [] {
        const char* v = std::getenv("SLGPU_SPLIT_TILE");
        if (v == nullptr)
            return 0;
        return std::strcmp(v, "32") == 0 ? 32 : std::strcmp(v, "64") == 0 ? 64 : 0;
    }();
    return ne;
}

// One split-precision contraction of a launch: group, tier, form and where
// its coefficients, exponents and element matrices (and, for a transposed
// pair, the partner's) are.
struct SplitJob {
    GroupDev* g;
    int tier;
    bool paired;
    const double* C;
    const int32_t* elemexp;
    double* out;
    double* out2;
    bool f32;  // out and out2 hold floats
};

static std::array<int, 5> split_shape_key(const GroupDev& g, int tier) { return {0, tier, g.ntf, g.ndof, g.ngp}; }

// Column-slice bytes of one group in the scratch (256-byte aligned blocks).
static size_t split_col_bytes(const GroupDev& g, const GroupDev::Split& sp)
{
    return ((size_t)sp.S * sp.Qpad * g.tiles.size() * 64 + 255) & ~size_t(255);
}
static size_t split_exp_bytes(const GroupDev& g) { return (g.tiles.size() * 64 * 4 + 255) & ~size_t(255); }

template <int S, int NE>
static void launch_slices(Ctx* ctx, const ColSliceParams& cs)
{
    k_slice_cols<S, NE><<<grid_for(cs.ntiles * 64, 128), 128, 0, ctx->x->stream>>>(cs);
}

// Column slicing and the tcgen05 contraction of a set of jobs of one tier
// with element-tile width NE: one slicing launch and one persistent
// contraction launch per kSplitBatch jobs.  Every job's column slices and
// exponents get their own block of the execution state's scratch.
static void run_split_jobs(Ctx* ctx, const std::vector<SplitJob>& jobs, int NE)
{
    if (jobs.empty())
        return;
    const int tier = jobs[0].tier;
    size_t colb = 0, expb = 0;
    for (const SplitJob& j : jobs) {
        const GroupDev::Split& sp = ensure_split(ctx, *j.g, tier, j.paired);
        colb += split_col_bytes(*j.g, sp);
        expb += split_exp_bytes(*j.g);
    }
    {
        ArenaPause keep(*ctx->x);  // per-state scratch, kept between requests
        if (ctx->x->split_cols.bytes() < colb)
            ctx->x->split_cols.alloc(ctx, colb);
        if (ctx->x->split_colexp.bytes() < expb)
            ctx->x->split_colexp.alloc(ctx, expb);
    }
    int8_t* cols = ctx->x->split_cols.as<int8_t>();
    int32_t* cexp = ctx->x->split_colexp.as<int32_t>();
    for (size_t b0 = 0; b0 < jobs.size(); b0 += kSplitBatch) {
        const size_t b1 = std::min(jobs.size(), b0 + kSplitBatch);
        ColSliceParams cs{};
        SplitParams sp{};
        double slice_bytes = 0, ops = 0;
        int S = 0;
        for (size_t k = b0; k < b1; k++) {
            const SplitJob& j = jobs[k];
            const GroupDev& g = *j.g;
            const GroupDev::Split& s = *g.split[tier + 2 * (j.paired ? 2 : symmetric_form(g) ? 1 : 0)];
            S = s.S;
            const int64_t ntiles = (int64_t)g.tiles.size();
            const int Q = g.nterms * g.ngp;
            ColSliceGroup& c = cs.g[cs.ngroups++];
            c.C = j.C;
            c.elemexp = j.elemexp;
            c.tiles = g.tiles_d.as<Tile>();
            c.Q = Q;
            c.Qpad = s.Qpad;
            c.nelem = g.nelem;
            c.ntiles = ntiles;
            c.slices = cols;
            c.colexp = cexp;
            c.t0 = cs.ntiles;
            cs.ntiles += ntiles;
            SplitGroup& G = sp.g[sp.ngroups++];
            G.P = g.ntf * g.ndof;
            G.Ppad = s.Ppad;
            G.ntp = s.Ppad / kSplitM;
            G.nk = s.Qpad / kSplitKStep;
            G.nrows = s.nrows;
            G.rowmap = s.rowmap.empty() ? nullptr : s.rowmap.as<int2>();
            G.out2 = j.out2;
            G.tiles = g.tiles_d.as<Tile>();
            G.A = s.slices.as<int8_t>();
            G.B = cols;
            G.rowexp = s.rowexp.as<int32_t>();
            G.colexp = cexp;
            G.out = j.out;
            G.w0 = sp.nwork;
            G.nwork = (int64_t)G.ntp * ntiles * (64 / NE);
            sp.nwork += G.nwork;
            const size_t cb = split_col_bytes(g, s);
            slice_bytes += 8.0 * Q * g.nelem + 4.0 * g.nelem + (double)cb + 4.0 * ntiles * 64;
            // Algorithmic INT8 operations: 2 per product, pairs (a, b) with a + b <= L.
            int pairs = 0;
            for (int a = 1; a <= s.S; a++)
                for (int bb = 1; bb <= s.S; bb++) pairs += (a + bb <= s.L);
            ops += 2.0 * pairs * s.nrows * Q * g.nelem;
            cols += cb;
            cexp += split_exp_bytes(g) / 4;
        }
        sp.error = ctx->x->split_error.as<unsigned int>();
        sp.f32 = jobs[b0].f32 ? 1 : 0;
        sp.next = reinterpret_cast<unsigned long long*>(ctx->x->split_error.as<char>() + 16);
        const int kt = kstat_start(ctx, "slice_cols", slice_bytes);
        if (S == 7 && NE == 64)
            launch_slices<7, 64>(ctx, cs);
        else if (S == 7)
            launch_slices<7, 32>(ctx, cs);
        else if (S == 5 && NE == 64)
            launch_slices<5, 64>(ctx, cs);
        else if (S == 5)
            launch_slices<5, 32>(ctx, cs);
        else
            fail(SLGPU_E_UNSUPPORTED, "unsupported slice count");
        kstat_stop(ctx, kt);
        cuda_check(cudaGetLastError(), "k_slice_cols");
        ctx->launches++;
        const int kc = kstat_start(ctx, S == 7 ? "contract_split" : "contract_split_fp32", ops);
        if (S == 7 && NE == 64)
            launch_split<7, 8, 64>(ctx, sp);
        else if (S == 7)
            launch_split<7, 8, 32>(ctx, sp);
        else if (NE == 64)
            launch_split<5, 6, 64>(ctx, sp);
        else
            launch_split<5, 6, 32>(ctx, sp);
        kstat_stop(ctx, kc);
        cuda_check(cudaGetLastError(), "k_contract_split");
        ctx->launches++;
    }
}

// Times the candidates on the jobs' own data and returns the fastest.  The
// first candidate is the default: it runs once untimed first (clocks ramp up
// on a GPU that was idle), then every candidate runs three times in turn and
// its best run counts; another candidate replaces the default only when its
// best run is at least 3 % faster.  The candidates give identical results.
template <class Run>
static int pick_by_timing(Ctx* ctx, const std::vector<int>& cand, Run run)
{
    constexpr int kRounds = 3;
    const size_t nc = cand.size();
    std::vector<cudaEvent_t> ev(kRounds * nc + 1);
    for (auto& e : ev) cuda_check(cudaEventCreate(&e), "cudaEventCreate");
    run(cand[0]);
    cuda_check(cudaEventRecord(ev[0], ctx->x->stream), "cudaEventRecord");
    for (size_t r = 0; r < kRounds; r++)
        for (size_t c = 0; c < nc; c++) {
            run(cand[c]);
            cuda_check(cudaEventRecord(ev[1 + r * nc + c], ctx->x->stream), "cudaEventRecord");
        }
    cuda_check(cudaEventSynchronize(ev[kRounds * nc]), "sync");
    std::vector<float> best(nc, 0.0f);
    for (size_t c = 0; c < nc; c++)
        for (size_t r = 0; r < kRounds; r++) {
            float t = 0;
            cudaEventElapsedTime(&t, ev[r * nc + c], ev[r * nc + c + 1]);
            best[c] = r == 0 ? t : std::min(best[c], t);
        }
    for (auto& e : ev) cudaEventDestroy(e);
    size_t pick = 0;
    for (size_t c = 1; c < nc; c++)
        if (best[c] < 0.97f * best[pick])
            pick = c;
    return cand[pick];
}

// Element-tile width for a group shape: forced, tuned, or (while graph
// capture or a request stream prevents timing) 64.
static int split_ne_of(Ctx* ctx, const GroupDev& g, int tier)
{
    if (split_tile_forced() != 0)
        return split_tile_forced();
    auto it = ctx->tile_choice.find(split_shape_key(g, tier));
    return it == ctx->tile_choice.end() ? 64 : it->second;
}

// All split jobs of one process: shapes without a tuned width are timed
// first (their jobs at each width), then one launch pair per width.
static void contract_split_all(Ctx* ctx, const std::vector<SplitJob>& jobs)
{
    if (jobs.empty())
        return;
    if (split_tile_forced() == 0 && !ctx->x->capturing && ctx->x == &ctx->main) {
        std::map<std::array<int, 5>, std::vector<SplitJob>> untuned;
        for (const SplitJob& j : jobs)
            if (!ctx->tile_choice.count(split_shape_key(*j.g, j.tier)))
                untuned[split_shape_key(*j.g, j.tier)].push_back(j);
        for (auto& kv : untuned)
            ctx->tile_choice[kv.first] = pick_by_timing(ctx, {64, 32}, [&](int ne) { run_split_jobs(ctx, kv.second, ne); });
    }
    std::vector<SplitJob> by[2];
    for (const SplitJob& j : jobs) by[split_ne_of(ctx, *j.g, j.tier) == 32 ? 1 : 0].push_back(j);
    run_split_jobs(ctx, by[0], 64);
    run_split_jobs(ctx, by[1], 32);
}

// Whether a group's contraction runs in split precision: element matrices
// with at least 64 entries (order >= 2 in practice); right-hand sides and
// small matrices stay in FP64.
static bool uses_split(const GroupDev& g, int precision)
{
    return precision != SLGPU_PREC_FP64 && !g.rhs && (int64_t)g.ntf * g.ndof >= 64 && split_supported(g);
}

// Shared memory of k_contract_small for a group (M of every orientation and
// the block's staged outputs), and whether its FP64 contraction uses it:
// element matrices of at most 32 entries whose tables fit.
static size_t small_kernel_smem(const GroupDev& g)
{
    const int64_t P = (int64_t)g.ntf * g.ndof;
    return ((size_t)g.norient * g.nterms * g.ngp * P + (size_t)kSmallE * (P + 1)) * 8;
}
static bool uses_small_kernel(const GroupDev& g) { return (int64_t)g.ntf * g.ndof <= kSmallP && small_kernel_smem(g) <= kSmallSmem; }

// Whether an FP64 contraction of a group may use the mirrored forms (upper
// triangle of a symmetric group, transposed pairs): matrix groups with at
// least 64 entries, as for split precision.
static bool fp64_mirrored(const GroupDev& g) { return !g.rhs && (int64_t)g.ntf * g.ndof >= 64; }

// Groups whose contraction may take a mirrored form at this precision.
static bool mirror_eligible(const GroupDev& g, int precision)
{
    return precision == SLGPU_PREC_FP64 ? fp64_mirrored(g) : uses_split(g, precision);
}

// Resident M^T of a group for the FP64 tensor-core kernel, built on first use
// in the main execution state's stream order (a request stream waits for it).
static GroupDev::Fp64Mt& ensure_fmt(Ctx* ctx, GroupDev& g, int form)
{
    std::unique_ptr<GroupDev::Fp64Mt>& f = g.fmt[form];
    if (f)
        return *f;
    Exec* cur = ctx->x;
    ctx->x = &ctx->main;
    try {
        f.reset(new GroupDev::Fp64Mt());
        const int Q = g.nterms * g.ngp, P = g.ntf * g.ndof;
        f->nrows = form == 1 ? g.ntf * (g.ntf + 1) / 2 : P;
        f->Qpad = (Q + kMmaBQ - 1) / kMmaBQ * kMmaBQ;
        f->rpad = (f->nrows + kMmaBPMax - 1) / kMmaBPMax * kMmaBPMax;
        if (form != 0)
            upload(ctx, f->rowmap, mirrored_rows(g.ntf, g.ndof, form == 1));
        f->Mt.alloc(ctx, (size_t)g.norient * f->Qpad * f->rpad * sizeof(double));
        BuildMtParams bp{};
        bp.tables = g.tables.as<double>();
        bp.tab_off = g.tab_off_d.as<int64_t>();
        bp.term_tf = g.term_tf_d.as<int32_t>();
        bp.term_dof = g.term_dof_d.as<int32_t>();
        bp.rowmap = f->rowmap.empty() ? nullptr : f->rowmap.as<int2>();
        bp.nterms = g.nterms;
        bp.ngp = g.ngp;
        bp.ntf = g.ntf;
        bp.ndof = g.ndof;
        bp.norient = g.norient;
        bp.nrows = f->nrows;
        bp.Qpad = f->Qpad;
        bp.rpad = f->rpad;
        bp.Mt = f->Mt.as<double>();
        const int64_t n = (int64_t)g.norient * f->Qpad * f->rpad;
        k_build_mt<<<(unsigned)std::min<int64_t>((n + 255) / 256, 65536), 256, 0, ctx->x->stream>>>(bp);
        cuda_check(cudaGetLastError(), "k_build_mt");
        ctx->launches++;
    } catch (...) {
        f.reset();
        ctx->x = cur;
        throw;
    }
    ctx->x = cur;
    if (cur != &ctx->main) {
        cudaEvent_t e;
        cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
        cuda_check(cudaEventRecord(e, ctx->main.stream), "cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(cur->stream, e, 0), "cudaStreamWaitEvent");
        cudaEventDestroy(e);
    }
    return *f;
}

template <int BP>
static void launch_f64mma(Ctx* ctx, const GroupDev& g, MmaParams mp)
{
    static std::once_flag attr;
    std::call_once(attr, [] {
        cudaFuncSetAttribute(k_contract_f64mma<BP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MmaShape<BP>::Smem);
    });
    mp.nrt = mp.rpad / BP;
    const int64_t nblocks = (int64_t)g.tiles.size() * mp.nrt;
    if (nblocks > INT32_MAX)
        fail(SLGPU_E_UNSUPPORTED, "group too large for one FP64 contraction launch");
    k_contract_f64mma<BP><<<(unsigned)nblocks, 256, MmaShape<BP>::Smem, ctx->x->stream>>>(mp);
    cuda_check(cudaGetLastError(), "k_contract_f64mma");
    ctx->launches++;
}

// FP64 contraction of one group on the FP64 tensor cores: every entry, the
// upper triangle of a symmetric group (mirrored into the lower), or every
// entry with the transposed partner's element matrices written into out2.
// Rows per block (128 or 64) are picked per group shape by timing on first
// use (SLGPU_F64_TILE=128 or 64 forces one).
static void contract_fp64_mma(Ctx* ctx, GroupDev& g, const double* C, double* out, double* out2)
{
    const int form = out2 != nullptr ? 2 : (fp64_mirrored(g) && symmetric_form(g)) ? 1 : 0;
    GroupDev::Fp64Mt& f = ensure_fmt(ctx, g, form);
    MmaParams mp{};
    mp.Mt = f.Mt.as<double>();
    mp.C = C;
    mp.tiles = g.tiles_d.as<Tile>();
    mp.rowmap = f.rowmap.empty() ? nullptr : f.rowmap.as<int2>();
    mp.Q = g.nterms * g.ngp;
    mp.Qpad = f.Qpad;
    mp.rpad = f.rpad;
    mp.nrows = f.nrows;
    mp.P = g.ntf * g.ndof;
    mp.mirror = form;
    mp.nelem = g.nelem;
    mp.out = out;
    mp.out2 = out2;
    static const int forced = [] {
        const char* v = std::getenv("SLGPU_F64_TILE");
        return v == nullptr ? 0 : std::strcmp(v, "64") == 0 ? 64 : std::strcmp(v, "128") == 0 ? 128 : 0;
    }();
    auto run = [&](int bp) {
        if (bp == 64)
            launch_f64mma<64>(ctx, g, mp);
        else
            launch_f64mma<128>(ctx, g, mp);
    };
    const std::array<int, 5> key{1, 0, g.ntf, g.ndof, g.ngp};
    int bp = forced;
    if (bp == 0) {
        auto it = ctx->tile_choice.find(key);
        if (it != ctx->tile_choice.end())
            bp = it->second;
        else if (!ctx->x->capturing && ctx->x == &ctx->main)
            bp = ctx->tile_choice[key] = pick_by_timing(ctx, {128, 64}, run);
        else
            bp = 128;
    }
    const int kt = kstat_start(ctx, "contract_fp64", 2.0 * f.nrows * mp.Q * g.nelem);
    run(bp);
    kstat_stop(ctx, kt);
}

// Transposed pairs among a matrix's split-precision groups: group j is the
// partner of group i when its element matrices are the transposes of i's:
// same elements, orientations and geometry, ntf and ndof swapped, the same
// element and field data, and a one-to-one map of terms u = pi(t) with u's
// test-function table holding the values of t's dof table, u's dof table
// those of t's test-function table, the same coefficient expression (factors
// in any order) and the same scale.  The contraction of the lower-numbered
// group then also writes the other's element matrices, transposed, and the
// other's contraction is skipped.  Groups whose data are replaced for one
// assembly (`ov`) and groups contracted as symmetric are not paired.
// Returns the partner of each group (-1: none).
static std::vector<int> cross_pairs(const Matrix& M, int precision, const std::vector<GroupData>* ov)
{
    const size_t n = M.groups.size();
    std::vector<int> pair(n, -1);
    static const bool enabled = [] {
        const char* v = std::getenv("SLGPU_SPLIT_PAIRS");
        return v == nullptr || std::strcmp(v, "0") != 0;
    }();
    if (!enabled || !mirror_forms_enabled())
        return pair;
    auto eligible = [&](size_t i) {
        const GroupDev& g = *M.groups[i];
        if (g.nelem == 0 || !mirror_eligible(g, precision) || symmetric_form(g) || g.term_keys.empty())
            return false;
        return ov == nullptr || ((*ov)[i].elemdata == nullptr && (*ov)[i].fielddata == nullptr && (*ov)[i].term_scale == nullptr);
    };
    std::vector<char> used;
    for (size_t i = 0; i < n; i++) {
        if (pair[i] >= 0 || !eligible(i))
            continue;
        const GroupDev& a = *M.groups[i];
        for (size_t j = i + 1; j < n; j++) {
            if (pair[j] >= 0 || !eligible(j))
                continue;
            const GroupDev& b = *M.groups[j];
            if (b.mesh != a.mesh || b.elemtype != a.elemtype || b.geom_hash != a.geom_hash || b.nelem != a.nelem ||
                b.ngp != a.ngp || b.norient != a.norient || b.ntf != a.ndof || b.ndof != a.ntf || b.nterms != a.nterms ||
                !(b.data_keys == a.data_keys))
                continue;
            used.assign(b.nterms, 0);
            bool ok = true;
            for (int t = 0; t < a.nterms && ok; t++) {
                const GroupDev::TermKey& ka = a.term_keys[t];
                int found = -1;
                for (int u = 0; u < b.nterms && found < 0; u++) {
                    const GroupDev::TermKey& kb = b.term_keys[u];
                    if (!used[u] && kb.tf == ka.dof && kb.dof == ka.tf && kb.coef == ka.coef &&
                        std::memcmp(&b.term_scale[u], &a.term_scale[t], sizeof(double)) == 0)
                        found = u;
                }
                if (found < 0)
                    ok = false;
                else
                    used[found] = 1;
            }
            if (ok) {
                pair[i] = (int)j;
                pair[j] = (int)i;
                break;
            }
        }
    }
    return pair;
}

// Host mirror of the runtime-compiled kernel's parameter structs (coef_jit.cu).
struct JitGeom {
    const double* xyz;
    const int32_t* conn;
    const int32_t* elems;
    const int32_t* orient;
    long long nelem;
    const double* weights;
    const double* lagrange;
};
struct JitGroup {
    const double* tables;
    const double* elemdata;
    const double* fielddata;
    const double* term_scale;
    double* C;
    int32_t* elemexp;  // nullptr, or per element: atomicMax of frexp exponents of |C|
};

// Geometry + coefficients of every group into C (offsets coff).  Consecutive
// groups with the same geometry key run as one runtime-compiled kernel; the
// interpreter kernel is used when SLGPU_COEF_INTERPRETER=1 or when a kernel
// cannot be compiled.
// Groups per runtime-compiled coefficient kernel: their descriptors (48 bytes
// each) are one by-value kernel parameter.
constexpr int kJitBatch = 64;

static void launch_coefficients(Ctx* ctx, const Matrix& M, double* C, const std::vector<int64_t>& coff, int32_t* elemexp,
                                const std::vector<int64_t>& eoff, const std::vector<GroupData>* ov, const std::vector<int>& pair)
{
    // The second group of a transposed pair needs no coefficients.
    auto skip = [&](size_t j) { return pair[j] >= 0 && pair[j] < (int)j; };
    static const bool interp_only = [] {
        const char* v = std::getenv("SLGPU_COEF_INTERPRETER");
        return v != nullptr && std::strcmp(v, "1") == 0;
    }();
    const size_t ng = M.groups.size();
    size_t k = 0;
    while (k < ng) {
        const GroupDev& g0 = *M.groups[k];
        size_t k1 = k + 1;
        while (k1 < ng && k1 - k < kJitBatch && M.groups[k1]->geom_hash == g0.geom_hash) k1++;
        if (g0.nelem == 0) {
            k = k1;
            continue;
        }
        bool done = false;
        // The runtime-compiled kernel covers elements of the mesh dimension;
        // lower-dimensional ones (boundary projections) use the interpreter.
        if (!interp_only && !ctx->jit_broken && g0.elemdim == g0.problemdim) {
            try {
                std::vector<const GroupDev*> batch;
                for (size_t j = k; j < k1; j++) batch.push_back(M.groups[j].get());
                // The kernel of a batch is remembered by its first group (the
                // source depends only on the batch's groups).
                std::vector<uint64_t> ids;
                for (const GroupDev* b : batch) ids.push_back(b->serial);
                cudaKernel_t kern = nullptr;
                if (g0.jit_members == ids)
                    kern = g0.jit_kernel;
                else {
                    kern = jit_coef_kernel(ctx, jit_coef_source(batch));
                    g0.jit_members = ids;
                    g0.jit_kernel = kern;
                }
                std::vector<JitGroup> jg;
                for (size_t j = k; j < k1; j++) {
                    GroupDev& G = *M.groups[j];
                    const double* ed = ov != nullptr && (*ov)[j].elemdata != nullptr ? (*ov)[j].elemdata : G.elemdata.as<double>();
                    const double* fd = ov != nullptr && (*ov)[j].fielddata != nullptr ? (*ov)[j].fielddata : G.fielddata.as<double>();
                    const double* ts = ov != nullptr && (*ov)[j].term_scale != nullptr ? (*ov)[j].term_scale : G.term_scale_d.as<double>();
                    jg.push_back(JitGroup{G.tables.as<double>(), ed, fd, ts, skip(j) ? nullptr : C + coff[j],
                                          eoff[j] >= 0 && !skip(j) ? elemexp + eoff[j] : nullptr});
                }
                const MeshDev& m = ctx->meshes.at(g0.mesh);
                JitGeom geom{m.xyz.as<double>(), m.types.at(g0.elemtype).conn.as<int32_t>(), g0.elems.as<int32_t>(), g0.orient.as<int32_t>(),
                             (long long)g0.nelem, g0.weights.as<double>(), g0.lagrange.as<double>()};
                void* args[] = {&geom, jg.data()};  // the group array is one by-value parameter
                const int64_t n = g0.nelem * (int64_t)g0.ngp;
                double cbytes = 0;
                for (size_t j = k; j < k1; j++)
                    if (!skip(j))
                        cbytes += 8.0 * M.groups[j]->nterms * M.groups[j]->ngp * M.groups[j]->nelem;
                const int kt = kstat_start(ctx, "coefficients", cbytes);
                cuda_check(cudaLaunchKernel((const void*)kern, dim3(grid_for(n, 128)), dim3(128), args, 0, ctx->x->stream),
                           "coefficient kernel launch");
                kstat_stop(ctx, kt);
                ctx->launches++;
                done = true;
            } catch (const SlgpuException&) {
                throw;
            } catch (const std::exception& e) {
                ctx->jit_broken = true;
                ctx->jit_error = e.what();
            }
        }
        if (!done) {
            for (size_t j = k; j < k1; j++) {
                if (skip(j))
                    continue;
                GroupDev& G = *M.groups[j];
                CoefParams cp = coef_params(ctx, G, C + coff[j]);
                cp.elemexp = eoff[j] >= 0 ? elemexp + eoff[j] : nullptr;
                if (ov != nullptr && (*ov)[j].elemdata != nullptr)
                    cp.elemdata = (*ov)[j].elemdata;
                if (ov != nullptr && (*ov)[j].fielddata != nullptr)
                    cp.fielddata = (*ov)[j].fielddata;
                if (ov != nullptr && (*ov)[j].term_scale != nullptr)
                    cp.term_scale = (*ov)[j].term_scale;
                const int64_t n = G.nelem * (int64_t)G.ngp;
                const int kt = kstat_start(ctx, "coefficients", 8.0 * G.nterms * G.ngp * G.nelem);
                k_geometry_coef<<<grid_for(n, 128), 128, 0, ctx->x->stream>>>(cp);
                kstat_stop(ctx, kt);
                cuda_check(cudaGetLastError(), "k_geometry_coef");
                ctx->launches++;
            }
        }
        k = k1;
    }
}

// Steps 1 and 2 on the current execution state's stream: coefficients of
// every group (with per-group data overrides, if given), contraction of each
// group into `vals` at the group's value base, fragment values after them.
bool float_values(const Matrix& M, int precision)
{
    if (precision != SLGPU_PREC_FP32 || !M.frags.empty() || M.groups.empty())
        return false;
    for (auto& g : M.groups)
        if (g->nelem > 0 && !uses_split(*g, precision))
            return false;
    return true;
}

void launch_contractions(Ctx* ctx, const Matrix& M, int precision, const std::vector<int64_t>& gvb, double* vals,
                         const std::vector<GroupData>* ov, bool f32)
{
    // Coefficients of every group coexist ([term][gp][element] per group) so
    // that groups sharing geometry are evaluated by one kernel.
    std::vector<int64_t> coff(M.groups.size());
    int64_t ctot = 0;
    for (size_t k = 0; k < M.groups.size(); k++) {
        coff[k] = ctot;
        ctot += (int64_t)M.groups[k]->nterms * M.groups[k]->ngp * M.groups[k]->nelem;
    }
    DevBuf C;
    C.alloc(ctx, std::max<int64_t>(ctot, 1) * 8);
    if (precision != SLGPU_PREC_FP64) {
        if (ctx->x->split_error.empty()) {
            ArenaPause keep(*ctx->x);
            ctx->x->split_error.alloc(ctx, 32);
        }
        cuda_check(cudaMemsetAsync(ctx->x->split_error.as<void>(), 0, 16, ctx->x->stream), "memset");
    }
    while (ctx->x->evpool.size() < 3) {
        cudaEvent_t e;
        cuda_check(cudaEventCreate(&e), "cudaEventCreate");
        ctx->x->evpool.push_back(e);
    }
    // Split-precision groups: per-element exponents of the coefficients,
    // gathered by the coefficient kernels (atomicMax from a very negative start).
    std::vector<int64_t> eoff(M.groups.size(), -1);
    int64_t etot = 0;
    for (size_t k = 0; k < M.groups.size(); k++)
        if (uses_split(*M.groups[k], precision)) {
            eoff[k] = etot;
            etot += M.groups[k]->nelem;
        }
    DevBuf E;
    if (etot > 0) {
        E.alloc(ctx, (size_t)etot * 4);
        cuda_check(cudaMemsetAsync(E.as<void>(), 0x80, (size_t)etot * 4, ctx->x->stream), "memset");
    }
    const std::vector<int> pair = cross_pairs(M, precision, ov);
    phase_event(ctx, ctx->x->evpool[0]);
    launch_coefficients(ctx, M, C.as<double>(), coff, E.as<int32_t>(), eoff, ov, pair);
    phase_event(ctx, ctx->x->evpool[1]);
    size_t gi = 0;
    std::vector<SplitJob> split_jobs;  // every split-precision group of the step, contracted together
    for (auto& g : M.groups) {
        if (g->nelem > 0) {
            double* Cg = C.as<double>() + coff[gi];
            // Split precision for the larger element matrices (order >= 2);
            // right-hand sides and small matrices stay in FP64.  The second
            // group of a transposed pair is written by the first's contraction.
            if (uses_split(*g, precision)) {
                if (pair[gi] < 0 || pair[gi] > (int)gi)
                    split_jobs.push_back(SplitJob{g.get(), precision == SLGPU_PREC_SPLIT ? 0 : 1, pair[gi] > (int)gi, Cg,
                                                  E.as<int32_t>() + eoff[gi], vals + gvb[gi],
                                                  pair[gi] > (int)gi ? vals + gvb[pair[gi]] : nullptr, f32});
                gi++;
                continue;
            }
            // The second group of a transposed pair is written by the first's contraction.
            if (pair[gi] >= 0 && pair[gi] < (int)gi) {
                gi++;
                continue;
            }
            if (f32)
                fail(SLGPU_E_STATE, "float element values need every group contracted by the split kernels");
            const int64_t P = (int64_t)g->ntf * g->ndof;
            const size_t small_smem = small_kernel_smem(*g);
            if (uses_small_kernel(*g)) {
                ContractParams kp{};
                kp.tables = g->tables.as<double>();
                kp.tab_off = g->tab_off_d.as<int64_t>();
                kp.term_tf = g->term_tf_d.as<int32_t>();
                kp.term_dof = g->term_dof_d.as<int32_t>();
                kp.nterms = g->nterms;
                kp.ngp = g->ngp;
                kp.ntf = g->ntf;
                kp.ndof = g->ndof;
                kp.nelem = g->nelem;
                kp.C = Cg;
                kp.tiles = g->tiles_d.as<Tile>();
                kp.out = vals + gvb[gi];
                static std::once_flag attr;
                std::call_once(attr, [] { cudaFuncSetAttribute(k_contract_small, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmallSmem); });
                const int kt = kstat_start(ctx, "contract_fp64", 2.0 * P * g->nterms * g->ngp * g->nelem);
                k_contract_small<<<(unsigned)((g->nelem + kSmallE - 1) / kSmallE), kSmallE, small_smem, ctx->x->stream>>>(
                    kp, g->orient.as<int32_t>(), g->norient);
                kstat_stop(ctx, kt);
                cuda_check(cudaGetLastError(), "k_contract_small");
                ctx->launches++;
            } else {
                contract_fp64_mma(ctx, *g, Cg, vals + gvb[gi], pair[gi] > (int)gi ? vals + gvb[pair[gi]] : nullptr);
            }
        }
        gi++;
    }
    contract_split_all(ctx, split_jobs);
    phase_event(ctx, ctx->x->evpool[2]);
    C.release();
    {
        int64_t vb = 0;
        for (auto& g : M.groups) vb += (int64_t)g->ntf * g->ndof * g->nelem;
        for (auto& f : M.frags) {
            int64_t n = (int64_t)f->nr * f->nc;
            if (n > 0)
                cuda_check(cudaMemcpyAsync(vals + vb, f->vals.as<double>(), n * 8, cudaMemcpyDeviceToDevice, ctx->x->stream),
                           "D2D fragment values");
            vb += n;
        }
    }
}

// CSR value kernel: -1 = chosen per pattern by timing the candidates
// (default), 0 = streaming warps (SLGPU_ROW_KERNEL=stream), 1 = warp per row
// (SLGPU_ROW_KERNEL=warp), 2 = thread per row, rows of at most 32 entries
// (SLGPU_ROW_KERNEL=thread).
static int row_kernel_forced()
{
    static const int k = [] {
        const char* v = std::getenv("SLGPU_ROW_KERNEL");
        if (v != nullptr && std::strcmp(v, "warp") == 0)
            return 1;
        if (v != nullptr && std::strcmp(v, "stream") == 0)
            return 0;
        if (v != nullptr && std::strcmp(v, "thread") == 0)
            return 2;
        return -1;
    }();
    return k;
}

std::vector<RowSeg> row_segments(const Matrix& M, const std::vector<Segment>& segs, bool f32)
{
    std::vector<RowSeg> rsegs(segs.size());
    size_t s = 0;
    for (auto& g : M.groups)
        for (int d = 0; d < g->ndests; d++, s++) rsegs[s] = RowSeg{segs[s].coo_base, segs[s].val_base, segs[s].mult, g->ndof, f32 ? 1 : 0};
    for (size_t f = 0; f < M.frags.size(); f++, s++) rsegs[s] = RowSeg{segs[s].coo_base, segs[s].val_base, 1.0, 1, 0};
    return rsegs;
}

namespace {
// Launch shape of the streaming value kernel for a pattern and segment widths.
struct StreamLaunch {
    RowStreamParams sp{};
    size_t smem = 0;
    bool ok = false;
    unsigned grid = 0;
    void (*kern)(RowStreamParams) = nullptr;
};

StreamLaunch stream_launch(Ctx* ctx, const RowParams& rp, const std::vector<RowSeg>& rsegs)
{
    StreamLaunch L;
    int wmax = 1;
    for (const RowSeg& sg : rsegs) wmax = std::max(wmax, (int)sg.width);
    RowStreamParams& sp = L.sp;
    const bool narrow = wmax <= StreamNarrow::WMAX;
    const int ring = narrow ? StreamNarrow::R : StreamWide::R;
    sp.r = rp;
    sp.lpad = (rp.lmax + 1) & ~1;
    sp.rows_per_chunk = 31;  // its 32 row bounds fit one per lane
    sp.nchunks = (rp.nrows + sp.rows_per_chunk - 1) / sp.rows_per_chunk;
    L.smem = (narrow ? row_stream_warp_bytes(StreamNarrow::R, StreamNarrow::VSH, StreamNarrow::SSH, sp.lpad)
                     : row_stream_warp_bytes(StreamWide::R, StreamWide::VSH, StreamWide::SSH, sp.lpad)) *
             kStreamWarps;
    if (wmax > StreamWide::WMAX || L.smem > 227 * 1024)
        return L;
    L.kern = narrow ? k_row_stream<StreamNarrow> : k_row_stream<StreamWide>;
    // Occupancy by ring depth and shared memory size; the kernels' shared
    // memory limit only ever grows (launches on other streams may use a
    // larger one).
    static std::mutex occ_mu;
    static std::map<std::pair<int, size_t>, int> blocks_per_sm;
    static size_t attr_max = 48 * 1024;
    int nblk = 1;
    {
        std::lock_guard<std::mutex> lk(occ_mu);
        if (L.smem > attr_max) {
            for (auto k : {k_row_stream<StreamNarrow>, k_row_stream<StreamWide>})
                cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem), "smem attribute");
            attr_max = L.smem;
        }
        const auto key = std::make_pair(ring, L.smem);
        auto bi = blocks_per_sm.find(key);
        if (bi == blocks_per_sm.end()) {
            int nb = 0;
            cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, L.kern, kStreamWarps * 32, L.smem), "occupancy");
            bi = blocks_per_sm.emplace(key, std::max(nb, 1)).first;
        }
        nblk = bi->second;
    }
    sp.nwarps = std::min<int64_t>(sp.nchunks, (int64_t)std::max(ctx->nsm, 1) * nblk * kStreamWarps);
    L.grid = (unsigned)((sp.nwarps + kStreamWarps - 1) / kStreamWarps);
    L.ok = sp.nwarps > 0;
    return L;
}

void launch_stream_rows(Ctx* ctx, const StreamLaunch& L)
{
    L.kern<<<L.grid, kStreamWarps * 32, L.smem, ctx->x->stream>>>(L.sp);
    cuda_check(cudaGetLastError(), "k_row_stream");
    ctx->launches++;
}

void launch_thread_rows(Ctx* ctx, const RowParams& rp, bool f32)
{
    const size_t smem = (size_t)rp.lmax * kThreadRows * 8;
    if (f32)
        k_row_thread<float><<<grid_for(rp.nrows, kThreadRows), kThreadRows, smem, ctx->x->stream>>>(rp);
    else
        k_row_thread<double><<<grid_for(rp.nrows, kThreadRows), kThreadRows, smem, ctx->x->stream>>>(rp);
    cuda_check(cudaGetLastError(), "k_row_thread");
    ctx->launches++;
}

void launch_warp_rows(Ctx* ctx, RowParams rp, bool f32)
{
    // Consecutive rows per warp: up to kRowsPerWarp (the row buffer stays
    // clean between them), fewer when the rows are too few to fill the
    // device with about 48 warps per multiprocessor.
    const int64_t target = (int64_t)std::max(ctx->nsm, 1) * 48;
    rp.rows_per_warp = (int)std::min<int64_t>(kRowsPerWarp, std::max<int64_t>(1, rp.nrows / target));
    const size_t per_warp = (size_t)rp.lmax * 8;
    int wpb = (int)std::max<size_t>(1, std::min<size_t>(8, (48 * 1024) / per_warp));
    size_t smem = per_warp * wpb;
    if (smem > 48 * 1024) {
        if (smem > 227 * 1024)
            fail(SLGPU_E_UNSUPPORTED, "a CSR row is too long for the shared-memory row buffer");
        cuda_check(cudaFuncSetAttribute(k_row_values<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attribute");
        cuda_check(cudaFuncSetAttribute(k_row_values<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attribute");
        cuda_check(cudaFuncSetAttribute(k_row_values<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attribute");
        cuda_check(cudaFuncSetAttribute(k_row_values<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attribute");
    }
    const unsigned grid = grid_for((rp.nrows + rp.rows_per_warp - 1) / rp.rows_per_warp, wpb);
    const bool U = rp.uniform_width > 0;
    if (f32 && U)
        k_row_values<float, true><<<grid, 32 * wpb, smem, ctx->x->stream>>>(rp);
    else if (f32)
        k_row_values<float, false><<<grid, 32 * wpb, smem, ctx->x->stream>>>(rp);
    else if (U)
        k_row_values<double, true><<<grid, 32 * wpb, smem, ctx->x->stream>>>(rp);
    else
        k_row_values<double, false><<<grid, 32 * wpb, smem, ctx->x->stream>>>(rp);
    cuda_check(cudaGetLastError(), "k_row_values");
    ctx->launches++;
}
}  // namespace

// Step 4 on the current execution state's stream: A/D values (or the dense
// right-hand side) from the element values through the resident pattern.
// `dsegs` is the device copy of `rsegs`.  The two value kernels add in the
// same order (bit-identical results); the first process() of a pattern on
// the context's own stream times both on its data and keeps the faster one
// for the pattern.
void launch_row_values(Ctx* ctx, const Matrix& M, Pattern& P, const std::vector<RowSeg>& rsegs, const RowSeg* dsegs, bool rhs,
                       const double* vals, double* Avals, double* Dvals)
{
    if (P.nA <= 0)
        return;
    RowParams rp{};
    rp.inc_ptr = P.inc_ptr.as<uint32_t>();
    rp.inc = P.inc.as<unsigned long long>();
    rp.segs = dsegs;
    rp.slotmap = P.slotmap.as<int16_t>();
    rp.vals = vals;
    rp.Arows = P.Arows.as<uint32_t>();
    rp.Drows = P.Drows.as<uint32_t>();
    rp.nrows = P.nA;
    rp.lmax = std::max(1, P.lmax);
    rp.Avals = Avals;
    rp.Dvals = rhs ? nullptr : Dvals;
    rp.dense = rhs ? Avals : nullptr;
    // Element values stored as floats (every segment alike, float_values()).
    const bool f32 = !rsegs.empty() && rsegs[0].f32 != 0;
    // Segments of one width (<= 32) with multiplier 1: the warp kernel takes
    // both from the launch instead of from each incidence.
    rp.uniform_width = 0;
    if (!rsegs.empty() && rsegs[0].width >= 1 && rsegs[0].width <= 32) {
        bool uni = true;
        for (const RowSeg& sg : rsegs)
            uni = uni && sg.width == rsegs[0].width && sg.mult == 1.0;
        if (uni)
            rp.uniform_width = rsegs[0].width;
    }
    // Bytes: kept element values and their slots, incidences, row
    // pointers read; A and D values written.
    const double rbytes = (f32 ? 6.0 : 10.0) * P.nvalid + 8.0 * P.ninc + 4.0 * (P.nA + 1) + 8.0 * (rhs ? M.ndofs : P.nnzA + P.nnzD);
    const StreamLaunch sl = stream_launch(ctx, rp, rsegs);
    const bool thread_ok = rp.lmax <= kThreadRowMax;
    // Candidates: warp per row always, streaming warps (double values) and
    // thread per row where their shapes allow.
    std::vector<int> cand{1};
    if (sl.ok && !f32)
        cand.push_back(0);
    if (thread_ok)
        cand.push_back(2);
    auto launch = [&](int c) {
        if (c == 0)
            launch_stream_rows(ctx, sl);
        else if (c == 2)
            launch_thread_rows(ctx, rp, f32);
        else
            launch_warp_rows(ctx, rp, f32);
    };
    int choice = row_kernel_forced();
    if (choice < 0)
        choice = P.row_kernel;
    // A kernel this call cannot use (the streaming warps with float values):
    // warp per row.
    if (choice >= 0 && std::find(cand.begin(), cand.end(), choice) == cand.end())
        choice = 1;
    if (choice < 0 && !ctx->x->capturing && ctx->x == &ctx->main) {
        // Every candidate timed on this call's data (their outputs are
        // identical), warp per row being the default.
        const int kt = kstat_start(ctx, "row_values", (1.0 + 3.0 * cand.size()) * rbytes);
        P.row_kernel = pick_by_timing(ctx, cand, launch);
        kstat_stop(ctx, kt);
        return;
    }
    if (choice < 0)
        choice = 1;
    const int kt = kstat_start(ctx, "row_values", rbytes);
    launch(choice);
    kstat_stop(ctx, kt);
}

// Everything the value path creates lazily (split-precision row slices,
// column-slice buffers, the error flag), made ahead of time on the current
// execution state so that the value path itself allocates none of it.
void prepare_value_path(Ctx* ctx, const Matrix& M, int precision)
{
    if (precision == SLGPU_PREC_FP64) {
        // The FP64 tensor-core operands of every tiled group, in the forms a
        // step can use (the plain or symmetric form; the paired form for the
        // first group of a transposed pair).
        const std::vector<int> pair = cross_pairs(M, precision, nullptr);
        for (size_t gi = 0; gi < M.groups.size(); gi++) {
            GroupDev* g = M.groups[gi].get();
            if (g->nelem == 0 || uses_small_kernel(*g))
                continue;
            ensure_fmt(ctx, *g, (fp64_mirrored(*g) && symmetric_form(*g)) ? 1 : 0);
            if (pair[gi] > (int)gi)
                ensure_fmt(ctx, *g, 2);
        }
        return;
    }
    const int tier = precision == SLGPU_PREC_SPLIT ? 0 : 1;
    size_t colbytes = 0, expbytes = 0;
    // Both the unpaired form (assemblies with replaced data) and, for the
    // first group of a transposed pair, the paired one.
    const std::vector<int> pair = cross_pairs(M, precision, nullptr);
    for (size_t gi = 0; gi < M.groups.size(); gi++) {
        GroupDev* g = M.groups[gi].get();
        if (g->nelem > 0 && uses_split(*g, precision)) {
            const GroupDev::Split& sp = ensure_split(ctx, *g, tier, false);
            if (pair[gi] > (int)gi)
                ensure_split(ctx, *g, tier, true);
            // The groups of a step are sliced and contracted together.
            colbytes += split_col_bytes(*g, sp);
            expbytes += split_exp_bytes(*g);
        }
    }
    Exec& x = *ctx->x;
    if (x.split_cols.bytes() < colbytes)
        x.split_cols.alloc(ctx, colbytes);
    if (x.split_colexp.bytes() < expbytes)
        x.split_colexp.alloc(ctx, expbytes);
    if (x.split_error.empty())
        x.split_error.alloc(ctx, 32);
}

ValueGraph::~ValueGraph()
{
    if (exec != nullptr)
        cudaGraphExecDestroy(exec);
    if (graph != nullptr)
        cudaGraphDestroy(graph);
    for (char* p : stage) cudaFreeHost(p);
}

// What the value path's launches take from host state: device pointers,
// kernel handles and sizes.  Contents that can change in place (per-element
// data, field data, term scales, the destination multipliers of the resident
// segment array, node coordinates) are read by the kernels at run time and
// are not part of it.  A group's own buffers and sizes are fixed at creation,
// so its serial number stands for them.
static std::vector<uint64_t> value_signature(Ctx* ctx, const Matrix& M, int precision, bool rhs, const Pattern& P,
                                             const std::vector<Segment>& segs)
{
    std::vector<uint64_t> s;
    auto u = [&](uint64_t v) { s.push_back(v); };
    auto p = [&](const void* q) { s.push_back((uint64_t)(uintptr_t)q); };
    const Exec& x = *ctx->x;
    u((uint64_t)precision);
    u(rhs ? 1 : 0);
    p(&P);
    u((uint64_t)P.row_kernel + 1);
    u((uint64_t)M.ndofs);
    p(M.vals.as<void>());
    p(M.Avals.as<void>());
    p(M.Dvals.as<void>());
    p(M.rsegs_dev.as<void>());
    u((uint64_t)split_tile_forced());
    u((uint64_t)ctx->nsm);
    u(ctx->timers ? 1 : 0);
    u(ctx->jit_broken ? 1 : 0);
    p(x.split_cols.as<void>());
    p(x.split_colexp.as<void>());
    p(x.split_error.as<void>());
    const std::vector<int> pair = cross_pairs(M, precision, nullptr);
    size_t gi = 0;
    for (auto& gp : M.groups) {
        const GroupDev& g = *gp;
        u(g.serial);
        p(g.jit_kernel);
        u(g.jit_members.size());
        for (uint64_t id : g.jit_members) u(id);
        u(symmetric_form(g) ? 1 : 0);
        u((uint64_t)(pair[gi++] + 1));
        for (int t = 0; t < 2; t++) {
            auto it = ctx->tile_choice.find(split_shape_key(g, t));
            u(it == ctx->tile_choice.end() ? 0 : (uint64_t)it->second);
        }
        for (int t = 0; t < 6; t++) {
            p(g.split[t] ? g.split[t]->slices.as<void>() : nullptr);
            p(g.split[t] ? g.split[t]->rowexp.as<void>() : nullptr);
        }
        for (int t = 0; t < 3; t++) p(g.fmt[t] ? g.fmt[t]->Mt.as<void>() : nullptr);
        auto mi = ctx->meshes.find(g.mesh);
        if (mi == ctx->meshes.end()) {
            u(~0ull);
            continue;
        }
        p(mi->second.xyz.as<void>());
        auto ti = mi->second.types.find(g.elemtype);
        p(ti == mi->second.types.end() ? nullptr : ti->second.conn.as<void>());
    }
    for (auto& f : M.frags) {
        p(f->vals.as<void>());
        u((uint64_t)f->nr);
        u((uint64_t)f->nc);
    }
    for (const Segment& sg : segs) {
        u((uint64_t)sg.coo_base);
        u((uint64_t)sg.val_base);
    }
    return s;
}

// Captures the value path into M.vgraph.  Copies the captured launches make
// from page-locked staging read blocks that the graph owns.  A capture the
// driver refuses leaves the matrix ungraphed (graph_failed).
static void capture_value_graph(Ctx* ctx, Matrix& M, int precision, bool rhs, const std::vector<int64_t>& gvb, std::vector<uint64_t> sig,
                                double* Av, double* Dv)
{
    Exec& x = *ctx->x;
    char* save_stage = x.stage;
    const size_t save_bytes = x.stage_bytes, save_used = x.stage_used, nold = x.stage_old.size();
    x.stage = nullptr;
    x.stage_bytes = x.stage_used = 0;
    auto G = std::make_unique<ValueGraph>();
    const int64_t l0 = ctx->launches;
    x.kev_tag.clear();
    cuda_check(cudaStreamBeginCapture(x.stream, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
    x.capturing = true;
    std::string err;
    try {
        launch_contractions(ctx, M, precision, gvb, M.vals.as<double>(), nullptr, float_values(M, precision));
        phase_event(ctx, ctx->x->ev[2]);
        launch_row_values(ctx, M, *M.pattern, M.rsegs_host, M.rsegs_dev.as<RowSeg>(), rhs, M.vals.as<double>(), Av, Dv);
    } catch (const std::exception& e) {
        err = e.what();
    }
    x.capturing = false;
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(x.stream, &graph);
    // Staging blocks used while capturing belong to the graph.
    if (x.stage != nullptr)
        G->stage.push_back(x.stage);
    for (size_t i = nold; i < x.stage_old.size(); i++) G->stage.push_back(x.stage_old[i]);
    x.stage_old.resize(nold);
    x.stage = save_stage;
    x.stage_bytes = save_bytes;
    x.stage_used = save_used;
    const int64_t nlaunch = ctx->launches - l0;
    ctx->launches = l0;
    if (err.empty() && ec == cudaSuccess && graph != nullptr) {
        G->graph = graph;
        if (cudaGraphInstantiate(&G->exec, graph, 0) == cudaSuccess) {
            G->kev_tag = x.kev_tag;
            G->launches = nlaunch;
            G->sig = std::move(sig);
            G->pattern = M.pattern;
            M.vgraph = std::move(G);
            return;
        }
        G->exec = nullptr;
    } else if (graph != nullptr) {
        cudaGraphDestroy(graph);
    }
    cudaGetLastError();
    M.graph_failed = true;
    M.vgraph.reset();
    x.kev_tag.clear();
}

static void process_matrix(Ctx* ctx, Matrix& M, const uint8_t* isconstrained, int precision, bool rhs, slgpu_csr_info* info)
{
    htrace_begin(ctx);
    ctx->x->kev_tag.clear();
    stage_reset(*ctx->x);
    if (ctx->record_only) {
        if (isconstrained != nullptr)
            M.rec_constrained.assign(isconstrained, isconstrained + M.ndofs);
        fail(SLGPU_E_NODEVICE, kNoDevice);
    }
    if (precision != SLGPU_PREC_FP64 && precision != SLGPU_PREC_SPLIT && precision != SLGPU_PREC_FP32)
        fail(SLGPU_E_ARG, "unknown precision mode");
    if (M.ndofs <= 0 || M.ndofs >= (int64_t(1) << 31))
        fail(SLGPU_E_ARG, "DOF count out of range");
    ev_record(ctx, 0);
    std::vector<int64_t> gvb;
    int64_t total_vals = 0;
    // FP32-level steps whose groups all go through the split kernels keep
    // their element matrices as floats: half the element-value traffic.
    const bool f32v = float_values(M, precision);
    std::vector<Segment> segs = build_segments(M, &gvb, &total_vals, f32v);

    // Constraints: device copy and content key, both reused while the array
    // is byte-identical to the previous call's.  A right-hand side uses an
    // all-zero array (every row kept).
    const uint8_t* hconstr = isconstrained;
    std::vector<uint8_t> zeros;
    if (rhs) {
        zeros.assign((size_t)M.ndofs, 0);
        hconstr = zeros.data();
    }
    const bool same = ctx->constr_host.size() == (size_t)M.ndofs &&
                      std::memcmp(ctx->constr_host.data(), hconstr, (size_t)M.ndofs) == 0;
    if (!same) {
        ctx->constr_host.assign(hconstr, hconstr + M.ndofs);
        ctx->constr_dev.alloc(ctx, (size_t)M.ndofs + 1);
        cuda_check(cudaMemcpyAsync(ctx->constr_dev.as<void>(), hconstr, M.ndofs, cudaMemcpyHostToDevice, ctx->x->stream), "H2D constr");
        ctx->bytes_h2d += M.ndofs;
        std::vector<int32_t> packed((M.ndofs + 3) / 4, 0);
        std::memcpy(packed.data(), hconstr, M.ndofs);
        uint64_t a = 0x12345, b = 0x6789;
        for (size_t i = 0; i < packed.size(); i++) {
            a = mix64(a ^ (uint64_t)(uint32_t)packed[i] ^ (uint64_t)i << 32);
            b += mix64((uint64_t)(uint32_t)packed[i] * 0x100000001b3ull + i);
        }
        ctx->constr_key[0] = a;
        ctx->constr_key[1] = b;
    }
    const uint8_t* dconstr = ctx->constr_dev.as<uint8_t>();
    uint64_t key0 = mix64(ctx->constr_key[0] ^ (uint64_t)M.ndofs ^ (rhs ? 0xABCDEFull : 0));
    uint64_t key1 = mix64(ctx->constr_key[1] ^ (uint64_t)segs.size());
    for (auto& g : M.groups) {
        key0 = mix64(key0 ^ g->addr_hash[0]);
        key1 = mix64(key1 + g->addr_hash[1]);
    }
    for (auto& f : M.frags) {
        key0 = mix64(key0 ^ f->addr_hash[0]);
        key1 = mix64(key1 + f->addr_hash[1]);
    }

    // 3: pattern (symbolic; cached while addresses and constraints are unchanged).
    bool reused = false;
    M.pattern = get_pattern(ctx, M, segs, dconstr, rhs, key0, key1, &reused);
    Pattern& P = *M.pattern;
    phase_event(ctx, ctx->x->ev[1]);

    // Output buffers, kept between calls while their sizes are unchanged.
    if (M.vals.bytes() < (size_t)std::max<int64_t>(total_vals, 1) * 8)
        M.vals.alloc(ctx, (size_t)std::max<int64_t>(total_vals, 1) * 8);
    auto keep_or_alloc = [&](DevBuf& b, int64_t n) {
        const size_t want = (((size_t)std::max<int64_t>(n, 1) * 8) + 255) & ~size_t(255);
        if (b.bytes() != want)
            b.alloc(ctx, want);
    };
    if (rhs) {
        keep_or_alloc(M.Avals, M.ndofs);
    } else {
        keep_or_alloc(M.Avals, P.nnzA);
        keep_or_alloc(M.Dvals, P.nnzD);
    }
    double* Av = M.Avals.as<double>();
    double* Dv = rhs ? nullptr : M.Dvals.as<double>();
    // Resident segment array of the value kernels (updated in place while its
    // size is unchanged, so that captured graphs stay valid).
    {
        std::vector<RowSeg> rsegs = row_segments(M, segs, f32v);
        const size_t nb = rsegs.size() * sizeof(RowSeg);
        const bool same = rsegs.size() == M.rsegs_host.size() && std::memcmp(rsegs.data(), M.rsegs_host.data(), nb) == 0;
        if (!same || M.rsegs_dev.empty()) {
            if (M.rsegs_dev.empty() || M.rsegs_dev.bytes() < std::max<size_t>(nb, 16))
                M.rsegs_dev.alloc(ctx, std::max<size_t>(nb, 16));
            if (nb > 0)
                upload_staged_into(ctx, M.rsegs_dev.as<void>(), rsegs.data(), nb);
            M.rsegs_host = std::move(rsegs);
        }
    }

    // 1+2 (coefficients, contractions into the value buffer) and 4 (CSR
    // values): replayed from a graph when the launches are the same as last
    // time's.
    bool graphed = false;
    if (ctx->graphs && reused && ctx->x == &ctx->main && !M.graph_failed) {
        prepare_value_path(ctx, M, precision);
        std::vector<uint64_t> sig = value_signature(ctx, M, precision, rhs, P, segs);
        if (!(M.vgraph && M.vgraph->sig == sig)) {
            M.vgraph.reset();
            if (M.vsig_prev == sig)
                capture_value_graph(ctx, M, precision, rhs, gvb, std::move(sig), Av, Dv);
            else
                M.vsig_prev = std::move(sig);
        }
        if (M.vgraph) {
            cuda_check(cudaGraphLaunch(M.vgraph->exec, ctx->x->stream), "cudaGraphLaunch");
            ctx->x->kev_tag = M.vgraph->kev_tag;
            ctx->launches += M.vgraph->launches;
            ctx->graph_launches++;
            graphed = true;
        }
    } else {
        M.vgraph.reset();
        M.vsig_prev.clear();
    }
    if (!graphed) {
        launch_contractions(ctx, M, precision, gvb, M.vals.as<double>(), nullptr, float_values(M, precision));
        phase_event(ctx, ctx->x->ev[2]);
        launch_row_values(ctx, M, P, M.rsegs_host, M.rsegs_dev.as<RowSeg>(), rhs, M.vals.as<double>(), Av, Dv);
    }
    ev_record(ctx, 3);
    cuda_check(cudaEventSynchronize(ctx->x->ev[3]), "sync");
    kstat_collect(ctx);
    if (precision != SLGPU_PREC_FP64) {
        unsigned int err = 0;
        cuda_check(cudaMemcpy(&err, ctx->x->split_error.as<void>(), 4, cudaMemcpyDeviceToHost), "D2H split error");
        if (err != 0)
            fail(SLGPU_E_TIMEOUT, "a split-precision contraction tile timed out waiting for its data");
    }
    float coef_ms = 0, contract_ms = 0;
    if (ctx->timers) {
        cudaEventElapsedTime(&coef_ms, ctx->x->evpool[0], ctx->x->evpool[1]);
        cudaEventElapsedTime(&contract_ms, ctx->x->evpool[1], ctx->x->evpool[2]);
    }
    ctx->x->timings[0] = coef_ms;
    ctx->x->timings[1] = contract_ms;
    ctx->x->timings[2] = ctx->timers ? ev_ms(ctx, 0, 1) : 0.0;
    ctx->x->timings[3] = ctx->timers ? ev_ms(ctx, 2, 3) : 0.0;
    ctx->x->timings[4] = ev_ms(ctx, 0, 3);
    if (info != nullptr) {
        info->nA = P.nA;
        info->nD = P.nD;
        info->nnzA = P.nnzA;
        info->nnzD = P.nnzD;
        info->ncoo = P.ncoo;
        info->pattern_reused = reused ? 1 : 0;
    }
    M.info.nA = P.nA;
    M.info.nD = P.nD;
    M.info.nnzA = P.nnzA;
    M.info.nnzD = P.nnzD;
    M.info.ncoo = P.ncoo;
    M.info.pattern_reused = reused;
}

}  // namespace slgpu

using namespace slgpu;

struct slgpu_ctx : public slgpu::Ctx {};

template <class F>
static int guarded(slgpu_ctx* ctx, F&& f)
{
    if (ctx == nullptr)
        return SLGPU_E_ARG;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    try {
        if (!ctx->record_only && ctx->device >= 0)
            cudaSetDevice(ctx->device);
        f();
        return SLGPU_OK;
    } catch (const SlgpuException& e) {
        ctx->last_error = e.e.msg;
        return e.e.code;
    } catch (const std::bad_alloc&) {
        ctx->last_error = "host allocation failed";
        return SLGPU_E_BUDGET;
    } catch (const std::exception& e) {
        ctx->last_error = e.what();
        return SLGPU_E_ARG;
    }
}

static Matrix& get_matrix(slgpu_ctx* ctx, int handle)
{
    auto it = ctx->matrices.find(handle);
    if (it == ctx->matrices.end())
        fail(SLGPU_E_ARG, "unknown matrix handle " + std::to_string(handle));
    return *it->second;
}

extern "C" {

int slgpu_ctx_create(int device, size_t hbm_budget, unsigned flags, slgpu_ctx** out)
{
    if (out == nullptr)
        return SLGPU_E_ARG;
    *out = nullptr;
    auto* ctx = new slgpu_ctx();
    ctx->budget = hbm_budget ? hbm_budget : (size_t)150 * 1000 * 1000 * 1000;
    ctx->record_only = (flags & SLGPU_CTX_RECORD_ONLY) != 0;
    if (!ctx->record_only) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0) {
            cudaGetLastError();
            delete ctx;
            return SLGPU_E_NODEVICE;
        }
        ctx->device = device;
        if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->x->stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            delete ctx;
            return SLGPU_E_CUDA;
        }
        for (auto& e : ctx->x->ev) cudaEventCreate(&e);
        cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device);
        const char* gv = std::getenv("SLGPU_GRAPHS");
        ctx->graphs = !(gv != nullptr && std::strcmp(gv, "0") == 0);
        const char* tv = std::getenv("SLGPU_KERNEL_TIMERS");
        ctx->timers = !(tv != nullptr && std::strcmp(tv, "0") == 0);
        // Keep freed blocks in the stream-ordered pool between assemblies.
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t threshold = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
        }
    }
    *out = ctx;
    return SLGPU_OK;
}

void slgpu_ctx_destroy(slgpu_ctx* ctx)
{
    if (ctx == nullptr)
        return;
    if (!ctx->record_only)
        cudaSetDevice(ctx->device);
    ctx->matrices.clear();
    ctx->patterns.clear();
    ctx->meshes.clear();
    ctx->scratch.release();
    ctx->hash_acc.release();
    ctx->constr_dev.release();
    // Every device buffer the context owns is freed on its stream, so all of
    // them must go before the stream does.
    ctx->x->split_cols.release();
    ctx->x->split_colexp.release();
    ctx->x->split_error.release();
    ctx->rhs_record.clear();
    for (cudaLibrary_t lib : ctx->jit_libs) cudaLibraryUnload(lib);
    ctx->jit_libs.clear();
    ctx->jit_kernels.clear();
    if (!ctx->record_only) {
        cudaStreamSynchronize(ctx->x->stream);
        for (auto& e : ctx->x->ev) cudaEventDestroy(e);
        for (auto& e : ctx->x->evpool) cudaEventDestroy(e);
        for (auto& e : ctx->x->kev) cudaEventDestroy(e);
        for (int b = 0; b < Ctx::kDlStages; b++) {
            if (ctx->dl_stage[b] != nullptr)
                cudaFreeHost(ctx->dl_stage[b]);
            if (ctx->dl_ev[b] != nullptr)
                cudaEventDestroy(ctx->dl_ev[b]);
        }
        for (int b = 0; b < Ctx::kUlStages; b++) {
            if (ctx->ul_stage[b] != nullptr)
                cudaFreeHost(ctx->ul_stage[b]);
            if (ctx->ul_ev[b] != nullptr)
                cudaEventDestroy(ctx->ul_ev[b]);
        }
        stage_free(ctx->main);
        cudaStreamDestroy(ctx->x->stream);
    }
    delete ctx;
}

int slgpu_last_error(const slgpu_ctx* ctx, char* buf, size_t len)
{
    if (ctx == nullptr || buf == nullptr || len == 0)
        return SLGPU_E_ARG;
    std::snprintf(buf, len, "%s", ctx->last_error.c_str());
    return SLGPU_OK;
}

int64_t slgpu_bytes_in_use(const slgpu_ctx* ctx) { return ctx ? ctx->in_use : 0; }

int slgpu_tuned_tiles(slgpu_ctx* ctx, char* buf, size_t len)
{
    return guarded(ctx, [&] {
        std::string t;
        for (const auto& kv : ctx->tile_choice) {
            const auto& k = kv.first;
            t += (k[0] == 0 ? std::string("split tier ") + std::to_string(k[1]) + " NE=" : std::string("fp64 rows/block="));
            t += std::to_string(kv.second) + " for ntf " + std::to_string(k[2]) + " ndof " + std::to_string(k[3]) + " ngp " +
                 std::to_string(k[4]) + "\n";
        }
        for (const auto& p : ctx->patterns)
            if (p)
                t += std::string("csr values kernel=") + (p->row_kernel == 0 ? "stream" : p->row_kernel == 1 ? "warp" : p->row_kernel == 2 ? "thread" : "untimed") +
                     " for " + std::to_string(p->nA) + " rows\n";
        if (buf != nullptr && len > 0)
            std::snprintf(buf, len, "%s", t.c_str());
    });
}

int slgpu_transfer_bytes(const slgpu_ctx* ctx, int64_t* h2d, int64_t* d2h)
{
    if (ctx == nullptr || h2d == nullptr || d2h == nullptr)
        return SLGPU_E_ARG;
    *h2d = ctx->bytes_h2d;
    *d2h = ctx->bytes_d2h;
    return SLGPU_OK;
}

int slgpu_host_register(slgpu_ctx* ctx, void* ptr, size_t bytes)
{
    return guarded(ctx, [&] {
        if (ptr == nullptr || bytes == 0)
            fail(SLGPU_E_ARG, "empty host range");
        if (ctx->record_only)
            fail(SLGPU_E_NODEVICE, "record-only context");
        cuda_check(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault), "cudaHostRegister");
    });
}

int slgpu_host_unregister(slgpu_ctx* ctx, void* ptr)
{
    return guarded(ctx, [&] {
        if (ptr == nullptr)
            fail(SLGPU_E_ARG, "null host pointer");
        if (ctx->record_only)
            fail(SLGPU_E_NODEVICE, "record-only context");
        cuda_check(cudaHostUnregister(ptr), "cudaHostUnregister");
    });
}

int slgpu_mesh_set_nodes(slgpu_ctx* ctx, int mesh, int64_t nnodes, const double* xyz)
{
    return guarded(ctx, [&] {
        if (nnodes < 0 || (nnodes > 0 && xyz == nullptr))
            fail(SLGPU_E_ARG, "invalid node array");
        MeshDev& m = ctx->meshes[mesh];
        const bool same = !ctx->record_only && m.nnodes == nnodes && !m.xyz.empty();
        m.nnodes = nnodes;
        if (same && nnodes > 0) {  // in place: buffers (and captured graphs) stay valid
            cuda_check(cudaMemcpyAsync(m.xyz.as<void>(), xyz, (size_t)3 * nnodes * 8, cudaMemcpyHostToDevice, ctx->x->stream),
                       "upload nodes");
            ctx->bytes_h2d += 24 * nnodes;
        }
        else if (!ctx->record_only)
            upload(ctx, m.xyz, xyz, (size_t)3 * nnodes);
        else
            m.hxyz.assign(xyz, xyz + 3 * nnodes);
    });
}

int slgpu_mesh_set_elements(slgpu_ctx* ctx, int mesh, int elemtype, int ncurvednodes, int64_t nelem, const int32_t* conn)
{
    return guarded(ctx, [&] {
        if (nelem < 0 || ncurvednodes <= 0 || (nelem > 0 && conn == nullptr))
            fail(SLGPU_E_ARG, "invalid connectivity");
        MeshDev& m = ctx->meshes[mesh];
        for (int64_t k = 0; k < nelem * ncurvednodes; k++)
            if (conn[k] < 0 || conn[k] >= m.nnodes)
                fail(SLGPU_E_ARG, "connectivity refers to a node outside the uploaded node array");
        MeshDev::Type& t = m.types[elemtype];
        t.ncn = ncurvednodes;
        t.nelem = nelem;
        if (!ctx->record_only)
            upload(ctx, t.conn, conn, (size_t)nelem * ncurvednodes);
        else
            t.hconn.assign(conn, conn + nelem * ncurvednodes);
    });
}

int slgpu_matrix_create(slgpu_ctx* ctx, int64_t ndofs, int* handle)
{
    return guarded(ctx, [&] {
        if (handle == nullptr || ndofs < 0)
            fail(SLGPU_E_ARG, "invalid matrix arguments");
        auto m = std::make_unique<Matrix>();
        m->ndofs = ndofs;
        *handle = ctx->next_handle++;
        ctx->matrices[*handle] = std::move(m);
    });
}

int slgpu_matrix_destroy(slgpu_ctx* ctx, int handle)
{
    return guarded(ctx, [&] {
        get_matrix(ctx, handle);
        ctx->matrices.erase(handle);
    });
}

int slgpu_matrix_clone(slgpu_ctx* ctx, int handle, int* new_handle)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (new_handle == nullptr)
            fail(SLGPU_E_ARG, "null handle pointer");
        auto m = std::make_unique<Matrix>();
        m->ndofs = M.ndofs;
        m->groups = M.groups;
        m->frags = M.frags;
        m->rec_constrained = M.rec_constrained;
        m->share_addresses = M.share_addresses;
        *new_handle = ctx->next_handle++;
        ctx->matrices[*new_handle] = std::move(m);
    });
}

int slgpu_matrix_share_addresses(slgpu_ctx* ctx, int handle, int enable)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        M.share_addresses = enable != 0;
        if (!M.share_addresses)
            M.shared_addresses.clear();
    });
}

int slgpu_matrix_add_group(slgpu_ctx* ctx, int handle, const slgpu_group* g, int* index)
{
    return guarded(ctx, [&] {
        if (g == nullptr)
            fail(SLGPU_E_ARG, "null group");
        Matrix& M = get_matrix(ctx, handle);
        if (g->terms == nullptr || g->nterms <= 0 || g->terms[0].dof_table < 0)
            fail(SLGPU_E_ARG, "matrix groups need dof tables (use slgpu_rhs_assemble for right-hand sides)");
        M.groups.push_back(make_group(ctx, *g, M.share_addresses ? &M.shared_addresses : nullptr));
        if (index)
            *index = (int)M.groups.size() - 1;
    });
}

int slgpu_matrix_add_fragment(slgpu_ctx* ctx, int handle, int32_t ntr, int32_t ndr, int32_t nr, int64_t nc, const int32_t* rows,
                              const int32_t* cols, const double* vals)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (nr < 0 || nc < 0 || ntr < 0 || ndr < 0)
            fail(SLGPU_E_ARG, "negative fragment size");
        if ((int64_t)nr * nc == 0)
            return;
        if ((ntr != nr || ndr != nr) && (int64_t)ntr * ndr != nr)
            fail(SLGPU_E_ARG, "fragment rows must be ntr*ndr when ntr or ndr differ from nr");
        auto f = std::make_shared<FragmentDev>();
        f->ntr = ntr;
        f->ndr = ndr;
        f->nr = nr;
        f->nc = nc;
        if (ctx->record_only) {
            f->hrows.assign(rows, rows + (size_t)ntr * nc);
            f->hcols.assign(cols, cols + (size_t)ndr * nc);
            f->hvals.assign(vals, vals + (size_t)nr * nc);
        } else {
            upload(ctx, f->rows, rows, (size_t)ntr * nc);
            upload(ctx, f->cols, cols, (size_t)ndr * nc);
            upload(ctx, f->vals, vals, (size_t)nr * nc);
            uint64_t h[2];
            hash_device(ctx, f->rows.as<int32_t>(), (int64_t)ntr * nc, 77, h);
            f->addr_hash[0] = h[0];
            f->addr_hash[1] = h[1];
            hash_device(ctx, f->cols.as<int32_t>(), (int64_t)ndr * nc, 78, h);
            f->addr_hash[0] = mix64(f->addr_hash[0] ^ h[0] ^ (uint64_t)nr << 32 ^ (uint64_t)nc);
            f->addr_hash[1] = mix64(f->addr_hash[1] ^ h[1] ^ (uint64_t)ntr << 32 ^ (uint64_t)ndr);
        }
        M.frags.push_back(std::move(f));
    });
}

int slgpu_matrix_group_count(slgpu_ctx* ctx, int handle, int* ngroups)
{
    return guarded(ctx, [&] {
        if (ngroups == nullptr)
            fail(SLGPU_E_ARG, "null output");
        *ngroups = (int)get_matrix(ctx, handle).groups.size();
    });
}

int slgpu_matrix_group_desc(slgpu_ctx* ctx, int handle, int gi, slgpu_group_desc* out)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (out == nullptr || gi < 0 || gi >= (int)M.groups.size())
            fail(SLGPU_E_ARG, "group index out of range");
        const GroupDev& g = *M.groups[gi];
        slgpu_group_desc d{};
        d.mesh = g.mesh;
        d.elemtype = g.elemtype;
        d.ntf = g.ntf;
        d.ndof = g.ndof;
        d.nterms = g.nterms;
        d.ngp = g.ngp;
        d.norient = g.norient;
        d.ndests = g.ndests;
        d.nelemdata = (int)g.elemdata_off.size();
        d.nfielddata = (int)g.field_off.size();
        for (int k = 0; k < 8 && k < d.nfielddata; k++) d.fieldrows[k] = g.field_rows[k];
        d.nelem = g.nelem;
        auto mit = ctx->meshes.find(g.mesh);
        if (mit != ctx->meshes.end() && mit->second.types.count(g.elemtype))
            d.mesh_nelem = mit->second.types.at(g.elemtype).nelem;
        *out = d;
    });
}

int slgpu_matrix_set_elemdata(slgpu_ctx* ctx, int handle, int gi, int k, const double* values)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (gi < 0 || gi >= (int)M.groups.size())
            fail(SLGPU_E_ARG, "group index out of range");
        GroupDev& g = *M.groups[gi];
        if (k < 0 || k >= (int)g.elemdata_off.size())
            fail(SLGPU_E_ARG, "element data index out of range");
        g.data_keys[k] = key_of(values, (size_t)g.nelem, 1);
        if (ctx->record_only) {
            std::copy(values, values + g.nelem, g.rec->elemdata[k].begin());
            return;
        }
        cuda_check(cudaMemcpyAsync(g.elemdata.as<double>() + g.elemdata_off[k], values, (size_t)g.nelem * 8, cudaMemcpyHostToDevice,
                                   ctx->x->stream),
                   "upload elemdata");
        ctx->bytes_h2d += g.nelem * 8;
    });
}

int slgpu_matrix_set_fielddata(slgpu_ctx* ctx, int handle, int gi, int k, const double* values)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (gi < 0 || gi >= (int)M.groups.size())
            fail(SLGPU_E_ARG, "group index out of range");
        GroupDev& g = *M.groups[gi];
        if (k < 0 || k >= (int)g.field_off.size())
            fail(SLGPU_E_ARG, "field data index out of range");
        const size_t n = (size_t)g.field_rows[k] * g.nelem;
        g.data_keys[g.elemdata_off.size() + k] = key_of(values, n, 2);
        if (ctx->record_only) {
            std::copy(values, values + n, g.rec->fielddata[k].begin());
            return;
        }
        cuda_check(cudaMemcpyAsync(g.fielddata.as<double>() + g.field_off[k], values, n * 8, cudaMemcpyHostToDevice, ctx->x->stream),
                   "upload fielddata");
        ctx->bytes_h2d += (int64_t)n * 8;
    });
}

int64_t slgpu_kernel_launches(const slgpu_ctx* ctx) { return ctx ? ctx->launches : 0; }

int slgpu_ctx_set_graphs(slgpu_ctx* ctx, int enable)
{
    return guarded(ctx, [&] {
        ctx->graphs = enable != 0;
        if (!ctx->graphs)
            for (auto& [h, m] : ctx->matrices) {
                m->vgraph.reset();
                m->vsig_prev.clear();
            }
    });
}

int64_t slgpu_graph_launches(const slgpu_ctx* ctx) { return ctx ? ctx->graph_launches : 0; }

int slgpu_ctx_set_kernel_timers(slgpu_ctx* ctx, int enable)
{
    return guarded(ctx, [&] { ctx->timers = enable != 0; });
}

int slgpu_check_coefficient_kernels(slgpu_ctx* ctx, int handle, char* log, size_t len)
{
    int st = guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        size_t k = 0;
        while (k < M.groups.size()) {
            size_t k1 = k + 1;
            while (k1 < M.groups.size() && k1 - k < (size_t)kJitBatch && M.groups[k1]->geom_hash == M.groups[k]->geom_hash) k1++;
            std::vector<const GroupDev*> batch;
            for (size_t j = k; j < k1; j++) batch.push_back(M.groups[j].get());
            try {
                if (M.groups[k]->elemdim == M.groups[k]->problemdim)
                    jit_compile(jit_coef_source(batch));
            } catch (const std::exception& e) {
                fail(SLGPU_E_CUDA, e.what());
            }
            k = k1;
        }
    });
    if (log != nullptr && len > 0)
        std::snprintf(log, len, "%s", st == SLGPU_OK ? "" : ctx->last_error.c_str());
    return st;
}

int slgpu_matrix_work(slgpu_ctx* ctx, int handle, slgpu_work* out)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (out == nullptr)
            fail(SLGPU_E_ARG, "null output");
        slgpu_work w{};
        for (auto& g : M.groups) {
            w.contraction_flops += (double)g->nelem * g->nterms * 2.0 * g->ntf * g->ndof * g->ngp;
            w.coef_points += g->nelem * (int64_t)g->ngp;
        }
        w.ngroups = (int32_t)M.groups.size();
        if (M.pattern) {
            w.ncoo = M.pattern->ncoo;
            w.nvalid = M.pattern->nvalid;
            w.nnz = M.pattern->nnzA + M.pattern->nnzD;
            w.nA = M.pattern->nA;
        }
        *out = w;
    });
}

int slgpu_matrix_set_scales(slgpu_ctx* ctx, int handle, int gi, const double* term_scales, const double* dest_multipliers)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (gi < 0 || gi >= (int)M.groups.size())
            fail(SLGPU_E_ARG, "group index out of range");
        GroupDev& g = *M.groups[gi];
        if (term_scales != nullptr) {
            g.term_scale.assign(term_scales, term_scales + g.nterms);
            if (!ctx->record_only)
                cuda_check(cudaMemcpyAsync(g.term_scale_d.as<void>(), term_scales, (size_t)g.nterms * 8, cudaMemcpyHostToDevice,
                                           ctx->x->stream),
                           "upload scales");
        }
        if (dest_multipliers != nullptr)
            g.dest_mult.assign(dest_multipliers, dest_multipliers + g.ndests);
    });
}

int slgpu_matrix_get_scales(slgpu_ctx* ctx, int handle, int gi, double* term_scales, double* dest_multipliers)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (gi < 0 || gi >= (int)M.groups.size())
            fail(SLGPU_E_ARG, "group index out of range");
        const GroupDev& g = *M.groups[gi];
        if (term_scales != nullptr)
            std::copy(g.term_scale.begin(), g.term_scale.end(), term_scales);
        if (dest_multipliers != nullptr)
            std::copy(g.dest_mult.begin(), g.dest_mult.end(), dest_multipliers);
    });
}

int slgpu_matrix_group_symmetry(slgpu_ctx* ctx, int handle, int gi, int32_t* mirror, int32_t* symmetric, int32_t* partner)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (gi < 0 || gi >= (int)M.groups.size())
            fail(SLGPU_E_ARG, "group index out of range");
        const GroupDev& g = *M.groups[gi];
        if (mirror != nullptr)
            for (int t = 0; t < g.nterms; t++) mirror[t] = g.mirror.empty() ? -1 : g.mirror[t];
        if (symmetric != nullptr)
            *symmetric = symmetric_form(g) ? (g.mirror_exact ? 1 : 2) : 0;
        if (partner != nullptr)
            *partner = cross_pairs(M, SLGPU_PREC_SPLIT, nullptr)[gi];
    });
}

int slgpu_matrix_process(slgpu_ctx* ctx, int handle, const uint8_t* isconstrained, int precision, slgpu_csr_info* info)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (isconstrained == nullptr && M.ndofs > 0)
            fail(SLGPU_E_ARG, "null constraint array");
        // Arrays given for sharing need to stay unchanged only until here.
        M.shared_addresses.clear();
        process_matrix(ctx, M, isconstrained, precision, false, info);
    });
}

namespace {

// Device -> host copy on the context's stream.  Page-locked or small
// destinations: one asynchronous copy (the caller synchronises).  Large
// pageable ones: 16 MB chunks through a ring of 32 page-locked blocks.  This
// thread issues the copies (at most 32 in flight) and up to 16 worker threads
// -- created once per call -- copy the landed chunks out, chunk i by worker
// i % 16, each worker owning two blocks.  The pageable destination, often
// freshly allocated and not yet touched, is advised to use huge pages
// (MADV_HUGEPAGE), so that its first-touch faults come 2 MB at a time.
void d2h(Ctx* ctx, void* dst, const void* src, size_t n)
{
    if (n == 0)
        return;
    ctx->bytes_d2h += (int64_t)n;
    cudaPointerAttributes a{};
    const bool pinned = cudaPointerGetAttributes(&a, dst) == cudaSuccess && a.type == cudaMemoryTypeHost;
    cudaGetLastError();
    constexpr size_t kChunk = size_t(16) << 20;
    if (pinned || n < 8 * kChunk) {
        cuda_check(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, ctx->x->stream), "D2H");
        return;
    }
    {
        const uintptr_t lo = (reinterpret_cast<uintptr_t>(dst) + (size_t(2) << 20) - 1) & ~((uintptr_t(2) << 20) - 1);
        const uintptr_t hi = (reinterpret_cast<uintptr_t>(dst) + n) & ~((uintptr_t(2) << 20) - 1);
        if (hi > lo)
            madvise(reinterpret_cast<void*>(lo), hi - lo, MADV_HUGEPAGE);  // advice only: failure changes nothing
    }
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    // First touches of a fresh destination, not the link, bound this copy
    // (measured on a 16-core host: 34 GB/s with 8 threads, 47 GB/s with 16,
    // against 56 GB/s over PCIe), so every core takes part.
    const int nw = std::max(1, std::min(std::min(hw, 16), Ctx::kDlStages / 2));
    const int nstage = 2 * nw;
    for (int b = 0; b < nstage; b++) {
        if (ctx->dl_stage[b] == nullptr)
            cuda_check(cudaHostAlloc(reinterpret_cast<void**>(&ctx->dl_stage[b]), kChunk, cudaHostAllocDefault), "cudaHostAlloc");
        if (ctx->dl_ev[b] == nullptr)
            cuda_check(cudaEventCreateWithFlags(&ctx->dl_ev[b], cudaEventDisableTiming), "cudaEventCreate");
    }
    const size_t nch = (n + kChunk - 1) / kChunk;
    // Chunk i uses block (i % nw) * 2 + (i / nw) % 2: worker i % nw alternates
    // between its two blocks.
    auto block = [&](size_t i) { return (int)((i % nw) * 2 + (i / nw) % 2); };
    std::mutex mu;
    std::condition_variable cv;
    size_t issued = 0;  // chunks [0, issued) have their copy queued
    std::vector<char> done(nch, 0);
    std::string err;
    auto issue = [&](size_t i) {
        const size_t off = i * kChunk, len = std::min(kChunk, n - off);
        const int b = block(i);
        cudaError_t e = cudaMemcpyAsync(ctx->dl_stage[b], static_cast<const char*>(src) + off, len, cudaMemcpyDeviceToHost, ctx->x->stream);
        if (e == cudaSuccess)
            e = cudaEventRecord(ctx->dl_ev[b], ctx->x->stream);
        return e;
    };
    std::vector<std::thread> workers;
    for (int w = 0; w < nw; w++)
        workers.emplace_back([&, w] {
            for (size_t i = (size_t)w; i < nch; i += (size_t)nw) {
                {
                    std::unique_lock<std::mutex> lk(mu);
                    cv.wait(lk, [&] { return issued > i || !err.empty(); });
                    if (!err.empty())
                        return;
                }
                const int b = block(i);
                const cudaError_t e = cudaEventSynchronize(ctx->dl_ev[b]);
                if (e != cudaSuccess) {
                    std::lock_guard<std::mutex> lk(mu);
                    err = std::string("D2H chunk wait: ") + cudaGetErrorString(e);
                    cv.notify_all();
                    return;
                }
                const size_t off = i * kChunk, len = std::min(kChunk, n - off);
                std::memcpy(static_cast<char*>(dst) + off, ctx->dl_stage[b], len);
                std::lock_guard<std::mutex> lk(mu);
                done[i] = 1;
                cv.notify_all();
            }
        });
    // Issue in order; chunk i may be issued once chunk i - nstage (same block) was copied out.
    for (size_t i = 0; i < nch; i++) {
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return i < (size_t)nstage || done[i - nstage] || !err.empty(); });
            if (!err.empty())
                break;
        }
        const cudaError_t e = issue(i);
        std::lock_guard<std::mutex> lk(mu);
        if (e != cudaSuccess) {
            err = std::string("D2H chunk: ") + cudaGetErrorString(e);
            cv.notify_all();
            break;
        }
        issued = i + 1;
        cv.notify_all();
    }
    for (auto& t : workers) t.join();
    if (!err.empty())
        fail(SLGPU_E_CUDA, err);
}
}  // namespace

int slgpu_matrix_download(slgpu_ctx* ctx, int handle, int32_t* Arows, int32_t* Acols, double* Avals, int32_t* Drows, int32_t* Dcols,
                          double* Dvals)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (!M.pattern)
            fail(SLGPU_E_STATE, "matrix not processed");
        Pattern& P = *M.pattern;
        d2h(ctx, Arows, P.Arows.as<void>(), (P.nA + 1) * 4);
        d2h(ctx, Acols, P.Acols.as<void>(), P.nnzA * 4);
        d2h(ctx, Avals, M.Avals.as<void>(), P.nnzA * 8);
        d2h(ctx, Drows, P.Drows.as<void>(), (P.nA + 1) * 4);
        d2h(ctx, Dcols, P.Dcols.as<void>(), P.nnzD * 4);
        d2h(ctx, Dvals, M.Dvals.as<void>(), P.nnzD * 8);
        cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync download");
    });
}

int slgpu_matrix_download_values(slgpu_ctx* ctx, int handle, double* Avals, double* Dvals)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (!M.pattern)
            fail(SLGPU_E_STATE, "matrix not processed");
        Pattern& P = *M.pattern;
        d2h(ctx, Avals, M.Avals.as<void>(), P.nnzA * 8);
        d2h(ctx, Dvals, M.Dvals.as<void>(), P.nnzD * 8);
        cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync download");
    });
}

int slgpu_matrix_pattern_serial(slgpu_ctx* ctx, int handle, uint64_t* serial)
{
    return guarded(ctx, [&] {
        if (serial == nullptr)
            fail(SLGPU_E_ARG, "null serial");
        Matrix& M = get_matrix(ctx, handle);
        *serial = M.pattern ? M.pattern->serial : 0;
    });
}

int slgpu_matrix_device_csr(slgpu_ctx* ctx, int handle, const int32_t** Arows, const int32_t** Acols, const double** Avals,
                            const int32_t** Drows, const int32_t** Dcols, const double** Dvals)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (!M.pattern)
            fail(SLGPU_E_STATE, "matrix not processed");
        Pattern& P = *M.pattern;
        *Arows = P.Arows.as<int32_t>();
        *Acols = P.Acols.as<int32_t>();
        *Avals = M.Avals.as<double>();
        *Drows = P.Drows.as<int32_t>();
        *Dcols = P.Dcols.as<int32_t>();
        *Dvals = M.Dvals.as<double>();
    });
}

int slgpu_matrix_eliminate(slgpu_ctx* ctx, int handle, const double* b, double* out)
{
    return guarded(ctx, [&] {
        Matrix& M = get_matrix(ctx, handle);
        if (!M.pattern)
            fail(SLGPU_E_STATE, "matrix not processed");
        if (b == nullptr || out == nullptr)
            fail(SLGPU_E_ARG, "null argument");
        Pattern& P = *M.pattern;
        for (const void* p : {(const void*)b, (const void*)out}) {
            cudaPointerAttributes a{};
            const bool dev = cudaPointerGetAttributes(&a, p) == cudaSuccess &&
                             (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == ctx->device;
            cudaGetLastError();
            if (!dev)
                fail(SLGPU_E_ARG, "b and out must be device memory of the context's device");
        }
        if (P.nA > 0) {
            k_eliminate<<<grid_for(P.nA, 256), 256, 0, ctx->x->stream>>>(P.Drows.as<uint32_t>(), P.Dcols.as<int32_t>(), M.Dvals.as<double>(),
                                                                       P.ainds.as<int32_t>(), P.dinds.as<int32_t>(), P.nA, b, out);
            cuda_check(cudaGetLastError(), "k_eliminate");
            ctx->launches++;
        }
        cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync eliminate");
    });
}

int slgpu_rhs_assemble(slgpu_ctx* ctx, const slgpu_group* g, int64_t ndofs, int precision, double* b_accum)
{
    return guarded(ctx, [&] {
        if (g == nullptr || b_accum == nullptr)
            fail(SLGPU_E_ARG, "null argument");
        if (g->terms == nullptr || g->nterms <= 0 || g->terms[0].dof_table >= 0 || g->ndof != 1)
            fail(SLGPU_E_ARG, "right-hand-side groups have no dof tables and ndof = 1");
        Matrix M;
        M.ndofs = ndofs;
        M.groups.push_back(make_group(ctx, *g));
        if (ctx->record_only) {
            ctx->rhs_record.push_back(M.groups.back());
            ctx->rhs_record_ndofs.push_back(ndofs);
        }
        process_matrix(ctx, M, nullptr, precision, true, nullptr);
        std::vector<double> dense((size_t)ndofs);
        if (ndofs > 0)
            cuda_check(cudaMemcpyAsync(dense.data(), M.Avals.as<void>(), (size_t)ndofs * 8, cudaMemcpyDeviceToHost, ctx->x->stream), "D2H");
        cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync rhs");
        for (int64_t i = 0; i < ndofs; i++) b_accum[i] += dense[i];
    });
}

int slgpu_rhs_assemble_rows(slgpu_ctx* ctx, const slgpu_group* g, int64_t ndofs, int precision, int32_t* rows, double* vals,
                            int64_t capacity, int64_t* count)
{
    return guarded(ctx, [&] {
        if (g == nullptr || rows == nullptr || vals == nullptr || count == nullptr || capacity < 0)
            fail(SLGPU_E_ARG, "null argument");
        if (g->terms == nullptr || g->nterms <= 0 || g->terms[0].dof_table >= 0 || g->ndof != 1)
            fail(SLGPU_E_ARG, "right-hand-side groups have no dof tables and ndof = 1");
        Matrix M;
        M.ndofs = ndofs;
        M.groups.push_back(make_group(ctx, *g));
        if (ctx->record_only) {
            ctx->rhs_record.push_back(M.groups.back());
            ctx->rhs_record_ndofs.push_back(ndofs);
        }
        process_matrix(ctx, M, nullptr, precision, true, nullptr);
        Pattern& P = *M.pattern;
        if (!P.rhs_rows_ready) {
            // Every DOF is a row of a right-hand side; the rows with incidences
            // are the ones an entry reaches.
            std::vector<uint32_t> ip((size_t)P.nA + 1);
            cuda_check(cudaMemcpyAsync(ip.data(), P.inc_ptr.as<void>(), ip.size() * 4, cudaMemcpyDeviceToHost, ctx->x->stream),
                       "D2H incidence pointers");
            cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync rhs rows");
            P.rhs_rows.clear();
            for (int64_t r = 0; r < P.nA; r++)
                if (ip[r + 1] > ip[r])
                    P.rhs_rows.push_back((int32_t)r);
            upload(ctx, P.rhs_rows_d, P.rhs_rows);
            P.rhs_rows_ready = true;
        }
        const int64_t n = (int64_t)P.rhs_rows.size();
        if (n > capacity)
            fail(SLGPU_E_ARG, "capacity smaller than the rows the right-hand side reaches");
        *count = n;
        if (n == 0)
            return;
        DevBuf out;
        out.alloc(ctx, (size_t)n * 8);
        k_gather_rows<<<grid_for(n, 256), 256, 0, ctx->x->stream>>>(M.Avals.as<double>(), P.rhs_rows_d.as<int32_t>(), n, out.as<double>());
        cuda_check(cudaGetLastError(), "k_gather_rows");
        ctx->launches++;
        cuda_check(cudaMemcpyAsync(vals, out.as<void>(), (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->x->stream), "D2H rhs rows");
        ctx->bytes_d2h += n * 8;
        cuda_check(cudaStreamSynchronize(ctx->x->stream), "sync rhs");
        std::memcpy(rows, P.rhs_rows.data(), (size_t)n * 4);
    });
}

int slgpu_last_timings(const slgpu_ctx* ctx, double* ms5)
{
    if (ctx == nullptr || ms5 == nullptr)
        return SLGPU_E_ARG;
    for (int i = 0; i < 5; i++) ms5[i] = ctx->x->timings[i];
    return SLGPU_OK;
}

int slgpu_kernel_stats(const slgpu_ctx* ctx, const char* family, double* total_ms, int64_t* launches, double* work)
{
    if (ctx == nullptr || family == nullptr)
        return SLGPU_E_ARG;
    auto it = ctx->x->kstats.find(family);
    const KernelStat none{};
    const KernelStat& k = it == ctx->x->kstats.end() ? none : it->second;
    if (total_ms != nullptr)
        *total_ms = k.ms;
    if (launches != nullptr)
        *launches = k.launches;
    if (work != nullptr)
        *work = k.work;
    return SLGPU_OK;
}

int slgpu_record_count(const slgpu_ctx* ctx, int handle, int* ngroups, int* nfragments)
{
    auto* c = const_cast<slgpu_ctx*>(ctx);
    return guarded(c, [&] {
        Matrix& M = get_matrix(c, handle);
        *ngroups = (int)M.groups.size();
        *nfragments = (int)M.frags.size();
    });
}

int slgpu_record_group(const slgpu_ctx* ctx, int handle, int gi, slgpu_group* out)
{
    auto* c = const_cast<slgpu_ctx*>(ctx);
    return guarded(c, [&] {
        if (!c->record_only)
            fail(SLGPU_E_STATE, "groups are only kept on record-only contexts");
        Matrix& M = get_matrix(c, handle);
        if (gi < 0 || gi >= (int)M.groups.size())
            fail(SLGPU_E_ARG, "group index out of range");
        *out = M.groups[gi]->rec->desc;
        out->terms = M.groups[gi]->rec->terms.data();
    });
}

int slgpu_record_fragment(const slgpu_ctx* ctx, int handle, int fi, int32_t* ntr, int32_t* ndr, int32_t* nr, int64_t* nc,
                          const int32_t** rows, const int32_t** cols, const double** vals)
{
    auto* c = const_cast<slgpu_ctx*>(ctx);
    return guarded(c, [&] {
        if (!c->record_only)
            fail(SLGPU_E_STATE, "fragments are only kept on record-only contexts");
        Matrix& M = get_matrix(c, handle);
        if (fi < 0 || fi >= (int)M.frags.size())
            fail(SLGPU_E_ARG, "fragment index out of range");
        FragmentDev& f = *M.frags[fi];
        *ntr = f.ntr;
        *ndr = f.ndr;
        *nr = f.nr;
        *nc = f.nc;
        *rows = f.hrows.data();
        *cols = f.hcols.data();
        *vals = f.hvals.data();
    });
}

int slgpu_record_rhs_count(const slgpu_ctx* ctx, int* ngroups)
{
    if (ctx == nullptr || ngroups == nullptr)
        return SLGPU_E_ARG;
    *ngroups = (int)ctx->rhs_record.size();
    return SLGPU_OK;
}

int slgpu_record_rhs_group(const slgpu_ctx* ctx, int gi, slgpu_group* out, int64_t* ndofs)
{
    auto* c = const_cast<slgpu_ctx*>(ctx);
    return guarded(c, [&] {
        if (gi < 0 || gi >= (int)c->rhs_record.size())
            fail(SLGPU_E_ARG, "rhs group index out of range");
        *out = c->rhs_record[gi]->rec->desc;
        *ndofs = c->rhs_record_ndofs[gi];
    });
}

int slgpu_record_mesh(const slgpu_ctx* ctx, int mesh, int elemtype, int64_t* nnodes, const double** xyz, int* ncurvednodes,
                      int64_t* nelem, const int32_t** conn)
{
    auto* c = const_cast<slgpu_ctx*>(ctx);
    return guarded(c, [&] {
        if (!c->record_only)
            fail(SLGPU_E_STATE, "mesh arrays are only kept on record-only contexts");
        auto it = c->meshes.find(mesh);
        if (it == c->meshes.end() || it->second.types.count(elemtype) == 0)
            fail(SLGPU_E_ARG, "no such mesh / element type");
        *nnodes = it->second.nnodes;
        *xyz = it->second.hxyz.data();
        const MeshDev::Type& t = it->second.types.at(elemtype);
        *ncurvednodes = t.ncn;
        *nelem = t.nelem;
        *conn = t.hconn.data();
    });
}

int slgpu_record_constraints(const slgpu_ctx* ctx, int handle, int64_t* ndofs, const uint8_t** isconstrained)
{
    auto* c = const_cast<slgpu_ctx*>(ctx);
    return guarded(c, [&] {
        Matrix& M = get_matrix(c, handle);
        *ndofs = M.ndofs;
        *isconstrained = M.rec_constrained.empty() ? nullptr : M.rec_constrained.data();
    });
}

}  // extern "C"

// ------------------------------------------------------------------------
// Element matrices without any device allocation.
//
// Some callers cannot allocate device memory: a host application whose own
// memory manager owns the whole device heap (allocations behind its back
// break its accounting or fail outright), or a latency-critical loop where
// cudaMalloc/cudaFree and the device-wide synchronisation they can imply are
// not acceptable.  For them slgpu_element_matrices_noalloc computes one
// group's element matrices using only the caller's input/output buffers and a
// fixed scratch array that lives in this library's device image.
//
// The scratch array below is file-scope and statically sized: every GPU that
// loads this library holds kNoAllocScratchBytes of it until the process
// exits.  All calls share it and it keeps whatever the last call left there;
// calls whose work overlaps on the GPU (different streams, or different host
// threads without ordering) race on it and must be serialised by the caller.
// Nothing in it has to start at zero: every byte a call reads was written by
// that same call first.
namespace slgpu {
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
static std::mutex g_noalloc_mutex;
static void* g_noalloc_addr[256] = {};  // device address of the scratch, per device

// Device address of the scratch array on the current device.  In host code
// the name g_noalloc_scratch is only a host-side stand-in, not a device
// address, so the address is looked up once per device (with that device
// current) and kept.  The kept address belongs to the device's primary
// context: the library must not be used across a cudaDeviceReset.
static void* noalloc_scratch_address(int* status, std::string* msg)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
        cudaGetLastError();
        *status = SLGPU_E_NODEVICE;
        *msg = "no current CUDA device";
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_addr[dev] == nullptr) {
        void* p = nullptr;
        cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (err != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            *status = SLGPU_E_CUDA;
            *msg = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(err);
            return nullptr;
        }
        g_noalloc_addr[dev] = p;
    }
    return g_noalloc_addr[dev];
}
}  // namespace slgpu

extern "C" int slgpu_element_matrices_noalloc(const slgpu_group* g, const double* xyz, int64_t nnodes, const int32_t* conn,
                                              int64_t mesh_nelem, double* K, void* stream, char* err, size_t errlen)
{
    auto report = [&](int code, const std::string& m) {
        if (err != nullptr && errlen > 0)
            std::snprintf(err, errlen, "%s", m.c_str());
        return code;
    };
    if (g == nullptr || xyz == nullptr || conn == nullptr || K == nullptr)
        return report(SLGPU_E_ARG, "null argument");
    if (nnodes <= 0 || nnodes > INT32_MAX)
        return report(SLGPU_E_ARG, "node count must be in [1, 2^31)");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    {
        // The copies below read host arrays, some of them temporaries of this
        // call, so they must not be recorded for a later replay.
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaError_t ce = cudaStreamIsCapturing(s, &cs);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            return report(SLGPU_E_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(ce));
        }
        if (cs != cudaStreamCaptureStatusNone)
            return report(SLGPU_E_UNSUPPORTED, "the stream is capturing; this call copies host arrays that do not outlive it");
    }
    try {
        validate_group(*g, false);
        for (int64_t e = 0; e < g->nelem; e++)
            if (g->elems[e] < 0 || g->elems[e] >= mesh_nelem)
                return report(SLGPU_E_ARG, "element number outside the mesh");
        std::vector<Instr> prog = compile_program(*g, g->nterms);
        std::vector<Tile> tiles;
        for (int64_t e = 0; e < g->nelem;) {
            const int o = g->orient[e];
            if (o < 0 || o >= g->norient)
                return report(SLGPU_E_ARG, "orientation index out of range");
            int64_t e1 = e;
            while (e1 < g->nelem && g->orient[e1] == o && e1 - e < kTileE) e1++;
            tiles.push_back(Tile{(int32_t)e, (int32_t)(e1 - e), o, 0});
            e = e1;
        }
        // Checked before anything is queued on the stream.
        if (tiles.size() > 65535)
            return report(SLGPU_E_UNSUPPORTED, "more than 65535 orientation-uniform runs of elements in one group");
        // Scratch layout: each block 256-byte aligned.
        struct Block {
            const void* src;
            size_t bytes;
            size_t off;
        };
        std::vector<Block> blocks;
        size_t top = 0;
        auto place = [&](const void* src, size_t bytes) {
            top = (top + 255) & ~size_t(255);
            blocks.push_back(Block{src, bytes, top});
            top += bytes;
            return blocks.size() - 1;
        };
        std::vector<int64_t> tab_off(g->ntables), field_off(g->nfielddata);
        std::vector<int32_t> tab_rows(g->ntables);
        int64_t tot = 0;
        for (int k = 0; k < g->ntables; k++) {
            tab_off[k] = tot;
            tab_rows[k] = g->tables[k].rows;
            tot += (int64_t)g->norient * g->tables[k].rows * g->ngp;
        }
        const int64_t tables_total = tot;
        tot = 0;
        for (int k = 0; k < g->nfielddata; k++) {
            field_off[k] = tot;
            tot += (int64_t)g->fieldrows[k] * g->nelem;
        }
        const int64_t field_total = tot;
        std::vector<double> term_scale(g->nterms);
        std::vector<int32_t> term_tf(g->nterms), term_dof(g->nterms);
        for (int t = 0; t < g->nterms; t++) {
            term_scale[t] = g->terms[t].scale;
            term_tf[t] = g->terms[t].tf_table;
            term_dof[t] = g->terms[t].dof_table;
        }
        const size_t b_prog = place(prog.data(), prog.size() * sizeof(Instr));
        const size_t b_consts = place(g->consts, (size_t)g->nconsts * 8);
        const size_t b_tables = place(nullptr, (size_t)tables_total * 8);
        const size_t b_weights = place(g->weights, (size_t)g->ngp * 8);
        const size_t b_lag = place(g->lagrange, (size_t)(1 + g->elemdim) * g->ncurvednodes * g->ngp * 8);
        const size_t b_elems = place(g->elems, (size_t)g->nelem * 4);
        const size_t b_orient = place(g->orient, (size_t)g->nelem * 4);
        const size_t b_elemdata = place(nullptr, (size_t)g->nelemdata * g->nelem * 8);
        const size_t b_field = place(nullptr, (size_t)field_total * 8);
        const size_t b_fieldoff = place(field_off.data(), field_off.size() * 8);
        const size_t b_taboff = place(tab_off.data(), tab_off.size() * 8);
        const size_t b_tabrows = place(tab_rows.data(), tab_rows.size() * 4);
        const size_t b_scale = place(term_scale.data(), term_scale.size() * 8);
        const size_t b_ttf = place(term_tf.data(), term_tf.size() * 4);
        const size_t b_tdof = place(term_dof.data(), term_dof.size() * 4);
        const size_t b_tiles = place(tiles.data(), tiles.size() * sizeof(Tile));
        const size_t b_C = place(nullptr, (size_t)g->nterms * g->ngp * g->nelem * 8);
        if (top > kNoAllocScratchBytes)
            return report(SLGPU_E_BUDGET, "group needs " + std::to_string(top) + " bytes of scratch; the allocation-free path has " +
                                              std::to_string(kNoAllocScratchBytes) + " (use slgpu_matrix_* for larger groups)");
        int status = SLGPU_OK;
        std::string msg;
        unsigned char* base = static_cast<unsigned char*>(noalloc_scratch_address(&status, &msg));
        if (base == nullptr)
            return report(status, msg);
        auto h2d = [&](size_t off, const void* src, size_t bytes) {
            if (bytes > 0)
                cuda_check(cudaMemcpyAsync(base + off, src, bytes, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync to scratch");
        };
        for (const Block& b : blocks)
            if (b.src != nullptr)
                h2d(b.off, b.src, b.bytes);
        for (int k = 0; k < g->ntables; k++)
            h2d(blocks[b_tables].off + (size_t)tab_off[k] * 8, g->tables[k].vals, (size_t)g->norient * g->tables[k].rows * g->ngp * 8);
        for (int k = 0; k < g->nelemdata; k++)
            h2d(blocks[b_elemdata].off + (size_t)k * g->nelem * 8, g->elemdata[k], (size_t)g->nelem * 8);
        for (int k = 0; k < g->nfielddata; k++)
            h2d(blocks[b_field].off + (size_t)field_off[k] * 8, g->fielddata[k], (size_t)g->fieldrows[k] * g->nelem * 8);
        if (g->nelem == 0)
            return report(SLGPU_OK, "");
        auto at = [&](size_t b) { return (void*)(base + blocks[b].off); };
        CoefParams cp{};
        cp.xyz = xyz;
        cp.conn = conn;
        cp.ncn = g->ncurvednodes;
        cp.elems = (const int32_t*)at(b_elems);
        cp.orient = (const int32_t*)at(b_orient);
        cp.nelem = g->nelem;
        cp.ngp = g->ngp;
        cp.weights = (const double*)at(b_weights);
        cp.lagrange = (const double*)at(b_lag);
        cp.dim = g->problemdim;
        cp.edim = g->elemdim;
        cp.prog = (const Instr*)at(b_prog);
        cp.nprog = (int)prog.size();
        cp.consts = (const double*)at(b_consts);
        cp.tables = (const double*)at(b_tables);
        cp.tab_off = (const int64_t*)at(b_taboff);
        cp.tab_rows = (const int32_t*)at(b_tabrows);
        cp.elemdata = (const double*)at(b_elemdata);
        cp.fielddata = (const double*)at(b_field);
        cp.field_off = (const int64_t*)at(b_fieldoff);
        cp.term_scale = (const double*)at(b_scale);
        cp.nterms = g->nterms;
        cp.C = (double*)at(b_C);
        cp.nnodes = nnodes;
        const int64_t n = g->nelem * (int64_t)g->ngp;
        k_geometry_coef<<<grid_for(n, 128), 128, 0, s>>>(cp);
        cuda_check(cudaGetLastError(), "k_geometry_coef");
        ContractParams kp{};
        kp.tables = cp.tables;
        kp.tab_off = cp.tab_off;
        kp.term_tf = (const int32_t*)at(b_ttf);
        kp.term_dof = (const int32_t*)at(b_tdof);
        kp.nterms = g->nterms;
        kp.ngp = g->ngp;
        kp.ntf = g->ntf;
        kp.ndof = g->ndof;
        kp.nelem = g->nelem;
        kp.C = cp.C;
        kp.tiles = (const Tile*)at(b_tiles);
        kp.out = K;
        const int64_t P = (int64_t)g->ntf * g->ndof;
        dim3 grid((unsigned)((P + kTileP - 1) / kTileP), (unsigned)tiles.size());
        k_contract_fp64<<<grid, dim3(16, 16), 0, s>>>(kp);
        cuda_check(cudaGetLastError(), "k_contract_fp64");
        return report(SLGPU_OK, "");
    } catch (const SlgpuException& e) {
        return report(e.e.code, e.e.msg);
    } catch (const std::exception& e) {
        return report(SLGPU_E_ARG, e.what());
    }
}
