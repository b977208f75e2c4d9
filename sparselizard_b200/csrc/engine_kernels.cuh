// Device kernels of the slgpu assembly engine (FP64 path and COO -> CSR).
#pragma once

#include "engine_internal.h"

#include <cstdint>

namespace slgpu {

constexpr int kTileE = 64;  // elements per contraction tile
constexpr int kTileP = 64;  // element-matrix entries (tf*ndof+dof) per contraction tile
constexpr int kTileQ = 16;  // (term, Gauss point) pairs staged per step

__device__ __forceinline__ unsigned long long dmix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Order-sensitive 128-bit content hash of an int32 array (sum and xor of
// per-position mixes; both are exact integer reductions, so deterministic).
__global__ void k_hash_i32(const int32_t* __restrict__ data, int64_t n, unsigned long long salt, unsigned long long* acc)
{
    unsigned long long s = 0, x = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long v = ((unsigned long long)i << 32) ^ (unsigned long long)(uint32_t)data[i] ^ (salt * 0xD6E8FEB86659FD93ull);
        s += dmix64(v);
        x ^= dmix64(v + 0x632BE59BD9B4E019ull);
    }
    for (int off = 16; off > 0; off >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, off);
        x ^= __shfl_down_sync(0xffffffffu, x, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc[0], s);
        atomicXor(&acc[1], x);
    }
}

struct CoefParams {
    const double* xyz;
    const int32_t* conn;
    int ncn;
    const int32_t* elems;
    const int32_t* orient;
    int64_t nelem;
    int ngp;
    const double* weights;
    const double* lagrange;  // [1+dim][ncn][ngp]
    int dim;
    const Instr* prog;
    int nprog;
    const double* consts;
    const double* tables;
    const int64_t* tab_off;
    const int32_t* tab_rows;
    const double* elemdata;
    const double* fielddata;
    const int64_t* field_off;
    const double* term_scale;
    int nterms;
    double* C;  // [nterms][ngp][nelem]
};

// Geometry (J, detJ, invJ; src/field/jacobian.cpp:248-349 and :396-504 for
// elements of the mesh dimension) and the coefficient program at one
// (element, Gauss point).  Thread n handles g = n / nelem, e = n % nelem so
// that the C writes are coalesced over elements.
__global__ void __launch_bounds__(128) k_geometry_coef(CoefParams p)
{
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= p.nelem * p.ngp)
        return;
    const int g = (int)(n / p.nelem);
    const int64_t e = n - (int64_t)g * p.nelem;
    const int elem = p.elems[e];
    const int o = p.orient[e];
    const int dim = p.dim;

    double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double X[3] = {0, 0, 0};
    const int32_t* cn = p.conn + (int64_t)elem * p.ncn;
    for (int k = 0; k < p.ncn; k++) {
        const int node = cn[k];
        const double x0 = p.xyz[3 * (int64_t)node + 0], x1 = p.xyz[3 * (int64_t)node + 1], x2 = p.xyz[3 * (int64_t)node + 2];
        const double nv = p.lagrange[(int64_t)k * p.ngp + g];
        X[0] += nv * x0;
        X[1] += nv * x1;
        X[2] += nv * x2;
        for (int a = 0; a < dim; a++) {
            const double dn = p.lagrange[((int64_t)(1 + a) * p.ncn + k) * p.ngp + g];
            J[a][0] += dn * x0;
            if (dim > 1) J[a][1] += dn * x1;
            if (dim > 2) J[a][2] += dn * x2;
        }
    }
    double det, inv[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (dim == 1) {
        det = J[0][0];
        inv[0][0] = 1.0 / J[0][0];
    } else if (dim == 2) {
        det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        inv[0][0] = J[1][1] / det;
        inv[0][1] = -J[0][1] / det;
        inv[1][0] = -J[1][0] / det;
        inv[1][1] = J[0][0] / det;
    } else {
        det = J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) - J[0][1] * (J[1][0] * J[2][2] - J[2][0] * J[1][2]) +
              J[0][2] * (J[1][0] * J[2][1] - J[2][0] * J[1][1]);
        inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
        inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
        inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
        inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
        inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
        inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
        inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
        inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
        inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    }
    const double wdet = p.weights[g] * fabs(det);

    double s[kMaxSlots];
    for (int k = 0; k < p.nprog; k++) {
        const Instr in = p.prog[k];
        double v = 0;
        switch (in.op) {
        case SLGPU_OP_CONST: v = p.consts[in.a]; break;
        case SLGPU_OP_JAC: v = J[in.a][in.b]; break;
        case SLGPU_OP_INVJAC: v = inv[in.a][in.b]; break;
        case SLGPU_OP_DETJAC: v = det; break;
        case SLGPU_OP_ELEM: v = p.elemdata[(int64_t)in.a * p.nelem + e]; break;
        case SLGPU_OP_FIELD: {
            const int rows = p.tab_rows[in.b];
            const double* fd = p.fielddata + p.field_off[in.a] + e;
            const double* tb = p.tables + p.tab_off[in.b] + (int64_t)o * rows * p.ngp + g;
            for (int f = 0; f < rows; f++) v += fd[(int64_t)f * p.nelem] * tb[(int64_t)f * p.ngp];
            break;
        }
        case SLGPU_OP_COORD: v = X[in.a]; break;
        case SLGPU_OP_ADD: v = s[in.a] + s[in.b]; break;
        case SLGPU_OP_MUL: v = s[in.a] * s[in.b]; break;
        case SLGPU_OP_INV: v = 1.0 / s[in.a]; break;
        case SLGPU_OP_NEG: v = -s[in.a]; break;
        case SLGPU_OP_POW: v = pow(s[in.a], s[in.b]); break;
        case INSTR_STORE:
            p.C[((int64_t)in.b * p.ngp + g) * p.nelem + e] = s[in.a] * p.term_scale[in.b] * wdet;
            continue;
        }
        s[in.dst] = v;
    }
}

struct ContractParams {
    const double* tables;
    const int64_t* tab_off;
    const int32_t* term_tf;
    const int32_t* term_dof;
    int nterms, ngp, ntf, ndof;
    int64_t nelem;
    const double* C;
    const Tile* tiles;
    double* out;  // [ntf*ndof][nelem]
};

// FP64 contraction: out[p][e] = sum_q M[p][q] C[q][e] with
// M[(i,j)][(t,g)] = T_t[o][i][g] * D_t[o][j][g] built in shared memory per
// tile (o = the tile's orientation).  Block 16x16 threads, 64 p x 64 e tile,
// each thread 4 x 4 outputs strided by 16.
__global__ void __launch_bounds__(256) k_contract_fp64(ContractParams p)
{
    __shared__ double Ms[kTileQ][kTileP];
    __shared__ double Cs[kTileQ][kTileE];
    const Tile tile = p.tiles[blockIdx.x];
    const int p0 = blockIdx.y * kTileP;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 16 + tx;
    const int P = p.ntf * p.ndof;
    const int Q = p.nterms * p.ngp;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0;

    for (int q0 = 0; q0 < Q; q0 += kTileQ) {
#pragma unroll
        for (int r = 0; r < (kTileQ * kTileP) / 256; r++) {
            const int idx = tid + 256 * r;
            const int qq = idx / kTileP, pp = idx % kTileP;
            const int q = q0 + qq, pe = p0 + pp;
            double val = 0;
            if (q < Q && pe < P) {
                const int t = q / p.ngp, g = q - t * p.ngp;
                const int i = pe / p.ndof, j = pe - i * p.ndof;
                const double tv = p.tables[p.tab_off[p.term_tf[t]] + ((int64_t)tile.orient * p.ntf + i) * p.ngp + g];
                const int dt = p.term_dof[t];
                const double dv = dt >= 0 ? p.tables[p.tab_off[dt] + ((int64_t)tile.orient * p.ndof + j) * p.ngp + g] : 1.0;
                val = tv * dv;
            }
            Ms[qq][pp] = val;
        }
#pragma unroll
        for (int r = 0; r < (kTileQ * kTileE) / 256; r++) {
            const int idx = tid + 256 * r;
            const int qq = idx / kTileE, ee = idx % kTileE;
            const int q = q0 + qq;
            Cs[qq][ee] = (q < Q && ee < tile.ne) ? p.C[(int64_t)q * p.nelem + tile.e0 + ee] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int qq = 0; qq < kTileQ; qq++) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = Ms[qq][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Cs[qq][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int pe = p0 + ty + 16 * i;
        if (pe >= P)
            continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int ee = tx + 16 * j;
            if (ee < tile.ne)
                p.out[(int64_t)pe * p.nelem + tile.e0 + ee] = acc[i][j];
        }
    }
}

struct KeyParams {
    const int32_t* tfaddr;
    const int32_t* dofaddr;  // null: right-hand side (column 0)
    int ndof;
    int64_t nelem, count, coo_base, ndofs;
    int colbits;
    const uint8_t* constrained;  // null: keep constrained rows
    unsigned long long invalid;
    unsigned long long* keys;
    uint32_t* idx;
    unsigned long long* nvalid;  // [0] valid count, [1] out-of-range address count
};

__device__ __forceinline__ void count_valid(unsigned long long* ctr, bool valid)
{
    const unsigned mask = __ballot_sync(__activemask(), valid);
    if ((threadIdx.x & 31) == (__ffs(__activemask()) - 1) && mask != 0)
        atomicAdd(ctr, (unsigned long long)__popc(mask));
}

// COO keys of one (group, destination) block in COO order (p-major, element
// minor), with the drop rules of rawmat::process (src/formulation/rawmat.cpp:162):
// negative row or column address, or a constrained row.
__global__ void k_group_keys(KeyParams p)
{
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool valid = false;
    if (k < p.count) {
        const int64_t pe = k / p.nelem, e = k - pe * p.nelem;
        const int64_t i = pe / p.ndof, j = pe - i * p.ndof;
        const int row = p.tfaddr[i * p.nelem + e];
        const int col = p.dofaddr ? p.dofaddr[j * p.nelem + e] : 0;
        bool bad = row >= p.ndofs || (p.dofaddr && col >= p.ndofs);
        if (bad)
            atomicAdd(&p.nvalid[1], 1ull);
        valid = !bad && row >= 0 && col >= 0 && (p.constrained == nullptr || !p.constrained[row]);
        p.keys[p.coo_base + k] = valid ? (((unsigned long long)row << p.colbits) | (unsigned long long)col) : p.invalid;
        p.idx[p.coo_base + k] = (uint32_t)(p.coo_base + k);
    }
    count_valid(&p.nvalid[0], valid);
}

struct FragKeyParams {
    const int32_t* rows;
    const int32_t* cols;
    int ntr, ndr, nr;
    int64_t nc, coo_base, ndofs;
    int colbits;
    const uint8_t* constrained;
    unsigned long long invalid;
    unsigned long long* keys;
    uint32_t* idx;
    unsigned long long* nvalid;
};

// Raw fragments decode rows as rawmat::process does (rawmat.cpp:150-155).
__global__ void k_frag_keys(FragKeyParams p)
{
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool valid = false;
    if (k < (int64_t)p.nr * p.nc) {
        const int64_t r = k / p.nc, c = k - r * p.nc;
        int64_t ctr = r, cdr = r;
        if (p.ntr != p.nr || p.ndr != p.nr) {
            ctr = r / p.ndr;
            cdr = r % p.ndr;
        }
        const int row = p.rows[ctr * p.nc + c];
        const int col = p.cols[cdr * p.nc + c];
        bool bad = row >= p.ndofs || col >= p.ndofs;
        if (bad)
            atomicAdd(&p.nvalid[1], 1ull);
        valid = !bad && row >= 0 && col >= 0 && (p.constrained == nullptr || !p.constrained[row]);
        p.keys[p.coo_base + k] = valid ? (((unsigned long long)row << p.colbits) | (unsigned long long)col) : p.invalid;
        p.idx[p.coo_base + k] = (uint32_t)(p.coo_base + k);
    }
    count_valid(&p.nvalid[0], valid);
}

__global__ void k_run_heads(const unsigned long long* __restrict__ sk, int64_t n, uint32_t* head)
{
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < n)
        head[k] = (k == 0 || sk[k] != sk[k - 1]) ? 1u : 0u;
}

__global__ void k_run_starts(const uint32_t* head, const uint32_t* runidx, int64_t n, uint32_t* run_start)
{
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < n && head[k])
        run_start[runidx[k]] = (uint32_t)k;
}

__global__ void k_constraint_flags(const uint8_t* c, int64_t ndofs, uint32_t* fA, uint32_t* fD)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i > ndofs)
        return;
    const bool con = i < ndofs && c[i];
    fA[i] = (i < ndofs && !con) ? 1u : 0u;
    fD[i] = con ? 1u : 0u;
}

// renumtolocalindex of gentools::findtruefalse as used by rawmat::process
// (src/formulation/rawmat.cpp:133): index among constrained or unconstrained DOFs.
__global__ void k_renumber(const uint8_t* c, int64_t ndofs, const uint32_t* sA, const uint32_t* sD, int32_t* renum)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < ndofs)
        renum[i] = c[i] ? (int32_t)sD[i] : (int32_t)sA[i];
}

__global__ void k_rhs_runs(const unsigned long long* sk, const uint32_t* run_start, int64_t nruns, int32_t* run_row, int32_t* run_target)
{
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r < nruns) {
        run_row[r] = (int32_t)sk[run_start[r]];
        run_target[r] = (int32_t)r;
    }
}

__global__ void k_classify_runs(const unsigned long long* sk, const uint32_t* run_start, int64_t nruns, int colbits, const uint8_t* c,
                                const int32_t* renum, uint32_t* isA, uint32_t* isD, uint32_t* rowcA, uint32_t* rowcD)
{
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r > nruns)
        return;
    if (r == nruns) {
        isA[r] = 0;
        isD[r] = 0;
        return;
    }
    const unsigned long long key = sk[run_start[r]];
    const int64_t row = (int64_t)(key >> colbits);
    const int64_t col = (int64_t)(key & ((1ull << colbits) - 1));
    const bool con = c[col] != 0;
    isA[r] = con ? 0u : 1u;
    isD[r] = con ? 1u : 0u;
    atomicAdd(con ? &rowcD[renum[row]] : &rowcA[renum[row]], 1u);
}

__global__ void k_fill_runs(const unsigned long long* sk, const uint32_t* run_start, int64_t nruns, int colbits, const uint32_t* isA,
                            const uint32_t* slotA, const uint32_t* slotD, const int32_t* renum, int32_t* run_target, int32_t* Acols,
                            int32_t* Dcols)
{
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= nruns)
        return;
    const unsigned long long key = sk[run_start[r]];
    const int64_t col = (int64_t)(key & ((1ull << colbits) - 1));
    if (isA[r]) {
        const uint32_t s = slotA[r];
        Acols[s] = renum[col];
        run_target[r] = (int32_t)s;
    } else {
        const uint32_t s = slotD[r];
        Dcols[s] = renum[col];
        run_target[r] = -(int32_t)s - 1;
    }
}

struct ValueParams {
    const uint32_t* perm;
    const uint32_t* run_start;
    const int32_t* run_target;
    int64_t nruns;
    const Segment* segs;
    int nsegs;
    const double* vals;
    double* Avals;
    double* Dvals;
    int negate;
};

// One CSR entry per thread: its COO contributions in sorted order (stable
// sort keeps COO order within a (row, col)), summed in FP64.
__global__ void k_csr_values(ValueParams p)
{
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= p.nruns)
        return;
    const uint32_t s = p.run_start[r], t = p.run_start[r + 1];
    double acc = 0;
    for (uint32_t k = s; k < t; k++) {
        const int64_t coo = p.perm[k];
        int lo = 0, hi = p.nsegs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (p.segs[mid].coo_base <= coo)
                lo = mid;
            else
                hi = mid - 1;
        }
        const Segment sg = p.segs[lo];
        acc += p.vals[sg.val_base + (coo - sg.coo_base)] * sg.mult;
    }
    const int32_t target = p.run_target[r];
    if (p.Dvals == nullptr)
        p.Avals[target] = p.negate ? -acc : acc;
    else if (target >= 0)
        p.Avals[target] = acc;
    else
        p.Dvals[-target - 1] = acc;
}

}  // namespace slgpu
