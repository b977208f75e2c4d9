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
    const double* lagrange;  // [1+edim][ncn][ngp]
    int dim;                 // mesh (problem) dimension
    int edim;                // element dimension (<= dim)
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
    int32_t* elemexp;  // nullptr, or [nelem]: atomicMax of the frexp exponents of |C|
    int64_t nnodes;    // > 0: node numbers outside [0, nnodes) are not read and give NaN coefficients
};

// Rows edim .. dim-1 of the Jacobian of an element of lower dimension than
// the mesh, completed as src/field/jacobian.cpp:19-235 does: points get the
// identity; a line in 2D the normed perpendicular of its tangent; a surface
// in 3D the normed cross product of its two rows; a line in 3D a normed
// perpendicular (the larger of [-b a 0] and [0 -c b] for row [a b c]), then
// the normed cross product.
__device__ __forceinline__ void complete_jacobian(double (&J)[3][3], int edim, int dim)
{
    if (edim == 0) {
        for (int a = 0; a < dim; a++)
            for (int b = 0; b < dim; b++) J[a][b] = a == b ? 1.0 : 0.0;
        return;
    }
    if (dim == 2 && edim == 1) {
        J[1][0] = -J[0][1];
        J[1][1] = J[0][0];
        const double nv = sqrt(J[1][0] * J[1][0] + J[1][1] * J[1][1]);
        J[1][0] = J[1][0] / nv;
        J[1][1] = J[1][1] / nv;
        return;
    }
    if (dim == 3 && edim == 1) {
        if (sqrt(J[0][0] * J[0][0] + J[0][1] * J[0][1]) > sqrt(J[0][1] * J[0][1] + J[0][2] * J[0][2])) {
            J[1][0] = -J[0][1];
            J[1][1] = J[0][0];
            J[1][2] = 0;
        } else {
            J[1][0] = 0;
            J[1][1] = -J[0][2];
            J[1][2] = J[0][1];
        }
        const double nv = sqrt(J[1][0] * J[1][0] + J[1][1] * J[1][1] + J[1][2] * J[1][2]);
        J[1][0] = J[1][0] / nv;
        J[1][1] = J[1][1] / nv;
        J[1][2] = J[1][2] / nv;
    }
    if (dim == 3 && edim <= 2) {
        J[2][0] = J[0][1] * J[1][2] - J[1][1] * J[0][2];
        J[2][1] = J[0][2] * J[1][0] - J[1][2] * J[0][0];
        J[2][2] = J[0][0] * J[1][1] - J[1][0] * J[0][1];
        const double nv = sqrt(J[2][0] * J[2][0] + J[2][1] * J[2][1] + J[2][2] * J[2][2]);
        J[2][0] = J[2][0] / nv;
        J[2][1] = J[2][1] / nv;
        J[2][2] = J[2][2] / nv;
    }
}

// Geometry (J, detJ, invJ; src/field/jacobian.cpp:4-349 and :396-504) and
// the coefficient program at one (element, Gauss point).  Thread n handles
// g = n / nelem, e = n % nelem so that the C writes are coalesced over
// elements.
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
    bool bad_node = false;
    for (int k = 0; k < p.ncn; k++) {
        const int node = cn[k];
        if (p.nnodes > 0 && (node < 0 || node >= p.nnodes)) {
            bad_node = true;
            continue;
        }
        const double x0 = p.xyz[3 * (int64_t)node + 0], x1 = p.xyz[3 * (int64_t)node + 1], x2 = p.xyz[3 * (int64_t)node + 2];
        const double nv = p.lagrange[(int64_t)k * p.ngp + g];
        X[0] += nv * x0;
        X[1] += nv * x1;
        X[2] += nv * x2;
        for (int a = 0; a < p.edim; a++) {
            const double dn = p.lagrange[((int64_t)(1 + a) * p.ncn + k) * p.ngp + g];
            J[a][0] += dn * x0;
            if (dim > 1) J[a][1] += dn * x1;
            if (dim > 2) J[a][2] += dn * x2;
        }
    }
    if (p.edim < dim)
        complete_jacobian(J, p.edim, dim);
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
    double cmax = 0;

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
        case INSTR_STORE: {
            const double c = bad_node ? __longlong_as_double(0x7ff8000000000000ll) : s[in.a] * p.term_scale[in.b] * wdet;
            p.C[((int64_t)in.b * p.ngp + g) * p.nelem + e] = c;
            cmax = fmax(cmax, fabs(c));
            continue;
        }
        }
        s[in.dst] = v;
    }
    if (p.elemexp != nullptr && cmax > 0) {
        int ex;
        frexp(cmax, &ex);
        atomicMax(p.elemexp + e, ex);
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
    double* out;  // [nelem][ntf*ndof]
};

// FP64 contraction: out[e][p] = sum_q M[p][q] C[q][e] with
// M[(i,j)][(t,g)] = T_t[o][i][g] * D_t[o][j][g] built in shared memory per
// tile (o = the tile's orientation).  Block 16x16 threads, 64 p x 64 e tile,
// each thread 4 x 4 outputs strided by 16; the tile is transposed through
// shared memory so that the element-major output rows are written whole.
// Grid: x = p tiles (adjacent blocks share the C columns in L2), y = tiles.
__global__ void __launch_bounds__(256) k_contract_fp64(ContractParams p)
{
    __shared__ double sm[kTileE * (kTileP + 1)];
    double(*Ms)[kTileP] = reinterpret_cast<double(*)[kTileP]>(sm);
    double(*Cs)[kTileE] = reinterpret_cast<double(*)[kTileE]>(sm + kTileQ * kTileP);
    const Tile tile = p.tiles[blockIdx.y];
    const int p0 = blockIdx.x * kTileP;
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
    // Transpose through shared memory: Out[e][p].
    double(*Out)[kTileP + 1] = reinterpret_cast<double(*)[kTileP + 1]>(sm);
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) Out[tx + 16 * j][ty + 16 * i] = acc[i][j];
    __syncthreads();
    const int pw = min(kTileP, P - p0);
    for (int idx = tid; idx < kTileE * kTileP; idx += 256) {
        const int ee = idx / kTileP, pp = idx % kTileP;
        if (ee < tile.ne && pp < pw)
            p.out[(int64_t)(tile.e0 + ee) * P + p0 + pp] = Out[ee][pp];
    }
}

// FP64 contraction for small element matrices (ntf*ndof <= 32): one thread
// per element, M of every orientation in shared memory.  Each output is
// accumulated in (term, Gauss point) order with the same fma operands as
// k_contract_fp64, so both kernels give the same values.  The block's outputs
// are staged in shared memory and stored as contiguous [e][p] rows.
constexpr int kSmallE = 128;
constexpr int kSmallP = 32;
constexpr int kSmallSmem = 96 * 1024;

__global__ void __launch_bounds__(kSmallE) k_contract_small(ContractParams p, const int32_t* __restrict__ orient, int norient)
{
    extern __shared__ double sm_small[];
    const int P = p.ntf * p.ndof, Q = p.nterms * p.ngp;
    double* Ms = sm_small;                             // [norient][Q][P]
    double* Os = sm_small + (int64_t)norient * Q * P;  // [kSmallE][P + 1]
    for (int idx = threadIdx.x; idx < norient * Q * P; idx += blockDim.x) {
        const int o = idx / (Q * P), rem = idx - o * (Q * P), q = rem / P, pe = rem - q * P;
        const int t = q / p.ngp, g = q - t * p.ngp;
        const int i = pe / p.ndof, j = pe - i * p.ndof;
        const double tv = p.tables[p.tab_off[p.term_tf[t]] + ((int64_t)o * p.ntf + i) * p.ngp + g];
        const int dt = p.term_dof[t];
        const double dv = dt >= 0 ? p.tables[p.tab_off[dt] + ((int64_t)o * p.ndof + j) * p.ngp + g] : 1.0;
        Ms[idx] = tv * dv;
    }
    __syncthreads();
    const int64_t e0 = (int64_t)blockIdx.x * kSmallE;
    const int64_t e = e0 + threadIdx.x;
    double acc[kSmallP];
#pragma unroll
    for (int pe = 0; pe < kSmallP; pe++) acc[pe] = 0.0;
    if (e < p.nelem) {
        const double* M = Ms + (int64_t)orient[e] * Q * P;
        // Coefficients eight at a time, all loads issued before their use.
        for (int q0 = 0; q0 < Q; q0 += 8) {
            double c[8];
#pragma unroll
            for (int u = 0; u < 8; u++) c[u] = q0 + u < Q ? p.C[(int64_t)(q0 + u) * p.nelem + e] : 0.0;
#pragma unroll
            for (int u = 0; u < 8; u++) {
                if (q0 + u >= Q)
                    break;
                const double* Mq = M + (q0 + u) * P;
#pragma unroll
                for (int pe = 0; pe < kSmallP; pe++)
                    if (pe < P)
                        acc[pe] = fma(Mq[pe], c[u], acc[pe]);
            }
        }
    }
#pragma unroll
    for (int pe = 0; pe < kSmallP; pe++)
        if (pe < P)
            Os[threadIdx.x * (P + 1) + pe] = acc[pe];
    __syncthreads();
    const int ne = (int)min((int64_t)kSmallE, p.nelem - e0);
    for (int idx = threadIdx.x; idx < ne * P; idx += blockDim.x) {
        const int ee = idx / P, pe = idx - ee * P;
        p.out[(e0 + ee) * P + pe] = Os[ee * (P + 1) + pe];
    }
}

struct KeyParams {
    const int32_t* tfaddr;
    const int32_t* dofaddr;  // null: right-hand side (column 0)
    int ndof, ntf;
    int64_t nelem, count, coo_base, ndofs;
    int colbits;
    const uint8_t* constrained;
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

// COO keys of one (group, destination) block in COO order (element-major:
// e, then i*ndof+j), with the drop rules of rawmat::process
// (src/formulation/rawmat.cpp:162): negative row or column address, or a
// constrained row.
__global__ void k_group_keys(KeyParams p)
{
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool valid = false;
    if (k < p.count) {
        const int64_t P = (int64_t)p.ntf * p.ndof;
        const int64_t e = k / P, pe = k - e * P;
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

__device__ __forceinline__ void frag_decode(int64_t k, int ntr, int ndr, int nr, int64_t nc, int64_t* ctr, int64_t* cdr, int64_t* c)
{
    const int64_t r = k / nc;
    *c = k - r * nc;
    *ctr = r;
    *cdr = r;
    if (ntr != nr || ndr != nr) {
        *ctr = r / ndr;
        *cdr = r % ndr;
    }
}

// Raw fragments decode rows as rawmat::process does (rawmat.cpp:150-155).
__global__ void k_frag_keys(FragKeyParams p)
{
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool valid = false;
    if (k < (int64_t)p.nr * p.nc) {
        int64_t ctr, cdr, c;
        frag_decode(k, p.ntr, p.ndr, p.nr, p.nc, &ctr, &cdr, &c);
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

// Ainds / Dinds of gentools::findtruefalse (src/formulation/rawmat.cpp:133):
// the unconstrained and the constrained DOFs, each in increasing order.
__global__ void k_dof_split(const uint8_t* c, int64_t ndofs, const uint32_t* sA, const uint32_t* sD, int32_t* ainds, int32_t* dinds)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= ndofs)
        return;
    if (c[i])
        dinds[sD[i]] = (int32_t)i;
    else
        ainds[sA[i]] = (int32_t)i;
}

// mat::eliminate (src/formulation/mat.cpp:78-103) on the device:
// out[r] = b[ainds[r]] - (D b_D)[r], (D b_D)[r] summed over the row in column
// order with separate roundings (the sequential product-then-add of a CSR
// SpMV on the host, MatMult_SeqAIJ), then subtracted as VecAXPY(ba, -1, prod).
// A thread per row: rows of D hold the few constrained neighbours of a DOF.
__global__ void k_eliminate(const uint32_t* __restrict__ Drows, const int32_t* __restrict__ Dcols, const double* __restrict__ Dvals,
                            const int32_t* __restrict__ ainds, const int32_t* __restrict__ dinds, int64_t nA,
                            const double* __restrict__ b, double* __restrict__ out)
{
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= nA)
        return;
    double s = 0.0;
    for (uint32_t k = Drows[r]; k < Drows[r + 1]; k++)
        s = __dadd_rn(s, __dmul_rn(Dvals[k], b[dinds[Dcols[k]]]));
    out[r] = __dadd_rn(b[ainds[r]], __dmul_rn(-1.0, s));
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

// Position of every kept COO entry inside its row's value segment
// ([A part | D part]); entries that are dropped keep -1.
// runidx is the exclusive scan of the run heads, so position k belongs to
// run runidx[k] + head[k] - 1 (a head starts its own run; any other
// position's exclusive count already includes its run's head).
// COO segment bounds used to tell which incidence (element-matrix row) a COO
// entry belongs to.
struct CooSeg {
    int64_t coo_base;
    int64_t width;
};

__device__ __forceinline__ int64_t incidence_of(const CooSeg* segs, int nsegs, int64_t coo, int* seg)
{
    int lo = 0, hi = nsegs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segs[mid].coo_base <= coo)
            lo = mid;
        else
            hi = mid - 1;
    }
    *seg = lo;
    return (coo - segs[lo].coo_base) / segs[lo].width;
}

// Also flags (dup[coo] = 1) an entry that falls on the same CSR entry as the
// previous entry of its own incidence -- two dof functions of one element
// with the same address.  Within a run entries keep COO order and the
// entries of one incidence are contiguous in COO order, so such pairs are
// adjacent.
__global__ void k_slotmap(const unsigned long long* sk, const uint32_t* perm, const uint32_t* head, const uint32_t* runidx, int64_t nvalid,
                          int colbits, const int32_t* run_target, const int32_t* renum, const uint32_t* Arows, const uint32_t* Drows,
                          int16_t* slotmap, unsigned long long* overflow, const CooSeg* csegs, int ncsegs, uint8_t* dup)
{
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= nvalid)
        return;
    if (k > 0 && head[k] == 0) {
        int sa, sb;
        const int64_t ia = incidence_of(csegs, ncsegs, perm[k], &sa);
        const int64_t ib = incidence_of(csegs, ncsegs, perm[k - 1], &sb);
        if (sa == sb && ia == ib)
            dup[perm[k]] = 1;
    }
    const int64_t row = (int64_t)(sk[k] >> colbits);
    const int32_t lr = renum[row];
    const int32_t t = run_target[(int64_t)runidx[k] + head[k] - 1];
    int64_t off;
    if (t >= 0)
        off = (int64_t)t - Arows[lr];
    else
        off = (int64_t)(Arows[lr + 1] - Arows[lr]) + (-(int64_t)t - 1 - Drows[lr]);
    if (off > 32767) {
        atomicAdd(overflow, 1ull);
        off = -1;
    }
    slotmap[perm[k]] = (int16_t)off;
}

// One incidence = one (segment, element, test function) row of an element
// matrix (width ndof), or one raw fragment entry (width 1).
struct IncSeg {
    int64_t inc_base;  // first incidence id of the segment
    int64_t count;     // incidences in the segment
    int64_t coo_base;  // first COO index of the segment
    int64_t val_base;  // first value of the segment in the value buffer
    double mult;       // destination multiplier
    int32_t width;     // entries per incidence (ndof, or 1 for fragments)
    int32_t ntf;       // group segments: test functions per element
    int32_t kind;      // 0 group, 1 fragment
    int32_t ntr, ndr, nr;
    int64_t nelem, nc;
    const int32_t* rows;  // group: tfaddr [ntf][nelem]; fragment: rows
    const int32_t* cols;  // fragment: cols
};

__global__ void k_inc_keys(const IncSeg* segs, int s, const uint8_t* constrained, int64_t ndofs, uint32_t* keys, uint32_t* ids,
                           unsigned long long* nvalid)
{
    const IncSeg sg = segs[s];
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool valid = false;
    if (k < sg.count) {
        int row;
        if (sg.kind == 0) {
            const int64_t e = k / sg.ntf, i = k - e * sg.ntf;
            row = sg.rows[i * sg.nelem + e];
        } else {
            int64_t ctr, cdr, c;
            frag_decode(k, sg.ntr, sg.ndr, sg.nr, sg.nc, &ctr, &cdr, &c);
            row = sg.rows[ctr * sg.nc + c];
            if (sg.cols[cdr * sg.nc + c] < 0)
                row = -1;
        }
        valid = row >= 0 && row < ndofs && !constrained[row];
        keys[sg.inc_base + k] = valid ? (uint32_t)row : 0xFFFFFFFFu;
        ids[sg.inc_base + k] = (uint32_t)(sg.inc_base + k);
    }
    count_valid(nvalid, valid);
}

// inc[k] = (serial << 63) | (segment << 40) | COO index of the incidence's
// first entry; serial marks an incidence with repeated addresses, whose
// entries must be added one after the other.
__global__ void k_inc_finalize(const uint32_t* skeys, const uint32_t* sids, int64_t ninc, const IncSeg* segs, int nsegs,
                               const int32_t* renum, const uint8_t* dup, unsigned long long* inc, uint32_t* rowcount)
{
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= ninc)
        return;
    const int64_t id = sids[k];
    int lo = 0, hi = nsegs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segs[mid].inc_base <= id)
            lo = mid;
        else
            hi = mid - 1;
    }
    const IncSeg& sg = segs[lo];
    const int64_t local = id - sg.inc_base;
    int64_t coo;
    if (sg.kind == 0) {
        const int64_t e = local / sg.ntf, i = local - e * sg.ntf;
        coo = sg.coo_base + e * (int64_t)sg.ntf * sg.width + i * sg.width;
    } else {
        coo = sg.coo_base + local;
    }
    unsigned long long serial = 0;
    for (int j = 0; j < sg.width; j++) serial |= dup[coo + j];
    inc[k] = (serial << 63) | ((unsigned long long)lo << 40) | (unsigned long long)coo;
    atomicAdd(&rowcount[renum[skeys[k]]], 1u);
}

// out[k] = v[rows[k]] for k < n.
__global__ void k_gather_rows(const double* __restrict__ v, const int32_t* __restrict__ rows, int64_t n, double* __restrict__ out)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n)
        out[k] = v[rows[k]];
}

__global__ void k_max_rowlen(const uint32_t* Arows, const uint32_t* Drows, int64_t nrows, unsigned long long* out)
{
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    unsigned long long len = 0;
    if (r < nrows)
        len = (unsigned long long)(Arows[r + 1] - Arows[r]) + (unsigned long long)(Drows[r + 1] - Drows[r]);
    for (int off = 16; off > 0; off >>= 1) len = max(len, __shfl_down_sync(0xffffffffu, len, off));
    if ((threadIdx.x & 31) == 0)
        atomicMax(out, len);
}

struct RowParams {
    const uint32_t* inc_ptr;
    const unsigned long long* inc;
    const RowSeg* segs;
    const int16_t* slotmap;
    const double* vals;
    const uint32_t* Arows;
    const uint32_t* Drows;
    int64_t nrows;
    int lmax;
    double* Avals;
    double* Dvals;
    double* dense;  // right-hand side: dense[row] = -value (Avals unused)
    int rows_per_warp;  // k_row_values: consecutive rows per warp (1 .. kRowsPerWarp)
    int uniform_width;  // every segment this width (<= 32) with multiplier 1, else 0
};

// CSR values, one warp per row: the row's incidences are visited in a fixed
// order and each adds its element-matrix row (contiguous in the element-major
// value buffer) into a shared-memory copy of the row through the slot map.
// Within one incidence every lane hits a different slot, so the sum of each
// CSR entry is formed in incidence order: deterministic, no atomics.
//
// Lane l decodes incidence l of each group of 32 (segment lookup, value and
// slot offsets) once; the other lanes receive it by shuffle.  The loads of
// kRowBatch incidences are issued before any of them is added (lane j holds
// entry j of each), so a warp keeps that many element-matrix rows in flight;
// the additions still run in incidence order.  Incidences flagged serial
// (duplicate addresses) or wider than a warp are added by their own loop at
// their place in the order.
constexpr int kRowBatch = 4;

template <class V>
__device__ __forceinline__ void row_add_generic(double* buf, int width, double mult, const V* v, const int16_t* sm, bool serial,
                                                int lane)
{
    if (serial) {
        if (lane == 0)
            for (int j = 0; j < width; j++) {
                const int s = sm[j];
                if (s >= 0)
                    buf[s] = fma((double)v[j], mult, buf[s]);
            }
    } else {
        for (int j = lane; j < width; j += 32) {
            const int s = sm[j];
            if (s >= 0)
                buf[s] = fma((double)v[j], mult, buf[s]);
        }
    }
}

// CSR values for short rows (lmax <= kThreadRowMax): one thread per row, its
// row buffer a column of a [lmax][kThreadRows] shared array.  The thread adds
// its incidences in order and each incidence's columns in order, so the
// results equal the warp kernels' (every slot is touched once per incidence
// except in serial incidences, which every kernel adds in column order).
constexpr int kThreadRows = 128;
constexpr int kThreadRowMax = 32;

template <class V>
__global__ void __launch_bounds__(kThreadRows) k_row_thread(RowParams p)
{
    const V* vals = reinterpret_cast<const V*>(p.vals);
    constexpr int64_t kScale = sizeof(double) / sizeof(V);  // values of type V per double of the buffer
    extern __shared__ double tbuf[];
    const int64_t r = (int64_t)blockIdx.x * kThreadRows + threadIdx.x;
    if (r >= p.nrows)
        return;
    double* buf = tbuf + threadIdx.x;  // slot s at buf[s * kThreadRows]
    const uint32_t a0 = p.Arows[r], a1 = p.Arows[r + 1];
    const uint32_t d0 = p.Drows ? p.Drows[r] : 0u, d1 = p.Drows ? p.Drows[r + 1] : 0u;
    const int la = (int)(a1 - a0), L = la + (int)(d1 - d0);
    for (int s = 0; s < L; s++) buf[s * kThreadRows] = 0.0;
    const uint32_t k0 = p.inc_ptr[r], k1 = p.inc_ptr[r + 1];
    for (uint32_t k = k0; k < k1; k++) {
        const unsigned long long pk = p.inc[k];
        const RowSeg sg = p.segs[(pk >> 40) & ((1ull << 23) - 1)];
        const long long co = (long long)(pk & ((1ull << 40) - 1));
        const V* v = vals + (sg.val_base * kScale + (co - sg.coo_base));
        const int16_t* sl = p.slotmap + co;
        for (int j = 0; j < sg.width; j++) {
            const int s = sl[j];
            if (s >= 0)
                buf[s * kThreadRows] = fma((double)v[j], sg.mult, buf[s * kThreadRows]);
        }
    }
    if (p.dense != nullptr) {
        p.dense[r] = L > 0 ? -buf[0] : 0.0;
        return;
    }
    for (int s = 0; s < L; s++) {
        if (s < la)
            p.Avals[a0 + s] = buf[s * kThreadRows];
        else
            p.Dvals[d0 + (s - la)] = buf[s * kThreadRows];
    }
}

// Most rows per warp of k_row_values: their 32 row bounds fit one per lane.
constexpr int kRowsPerWarp = 31;

template <class V, bool U>
__global__ void __launch_bounds__(256, 6) k_row_values(RowParams p)
{
    const V* vals = reinterpret_cast<const V*>(p.vals);
    constexpr long long kScale = sizeof(double) / sizeof(V);  // values of type V per double of the buffer
    extern __shared__ double rowbuf[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t r0 = ((int64_t)blockIdx.x * (blockDim.x >> 5) + warp) * p.rows_per_warp;
    if (r0 >= p.nrows)
        return;
    const int nr = (int)min((int64_t)p.rows_per_warp, p.nrows - r0);
    double* buf = rowbuf + (int64_t)warp * p.lmax;
    // The row buffer is kept zero between rows (the write-back clears it).
    for (int s = lane; s < p.lmax; s += 32) buf[s] = 0.0;
    // Row bounds of the warp's rows, one per lane (lane nr: the end).
    uint32_t a_lo = 0, d_lo = 0, i_lo = 0;
    if (lane <= nr) {
        a_lo = p.Arows[r0 + lane];
        d_lo = p.Drows ? p.Drows[r0 + lane] : 0u;
        i_lo = p.inc_ptr[r0 + lane];
    }
    __syncwarp();
    constexpr int kGeneric = 1 << 17, kSerial = 1 << 16;
    for (int rr = 0; rr < nr; rr++) {
        // The CSR bounds are fetched after the incidences (only the
        // write-back needs them): fewer registers live in the loop below.
        const uint32_t k0 = __shfl_sync(0xffffffffu, i_lo, rr), k1 = __shfl_sync(0xffffffffu, i_lo, rr + 1);
        for (uint32_t kb = k0; kb < k1; kb += 32) {
            const int nkb = (int)min(32u, k1 - kb);
            // Lane l decodes incidence kb + l.  Value and COO offsets fit 32
            // bits (fewer than 2^32 COO entries per matrix).
            uint32_t voff = 0, coo = 0;
            double mult = 0.0;
            int info = 0;  // width | kSerial | kGeneric
            if (lane < nkb) {
                const unsigned long long pk = p.inc[kb + lane];
                const RowSeg sg = p.segs[(pk >> 40) & ((1ull << 23) - 1)];
                coo = (uint32_t)(pk & ((1ull << 40) - 1));
                voff = (uint32_t)(sg.val_base * kScale + ((long long)coo - sg.coo_base));
                mult = sg.mult;
                const bool serial = (pk >> 63) != 0;
                info = sg.width | (serial ? kSerial : 0) | ((serial || sg.width > 32) ? kGeneric : 0);
            }
            if (!__any_sync(0xffffffffu, (info & kGeneric) != 0)) {
                // Batches of kRowBatch incidences: every load issued before
                // the ordered additions.
                for (int u = 0; u < nkb; u += kRowBatch) {
                    double val[kRowBatch];
                    int slot[kRowBatch];
#pragma unroll
                    for (int x = 0; x < kRowBatch; x++) {
                        const int src = (u + x) & 31;
                        const uint32_t vo = __shfl_sync(0xffffffffu, voff, src);
                        const uint32_t co = __shfl_sync(0xffffffffu, coo, src);
                        const int w = U ? p.uniform_width : (__shfl_sync(0xffffffffu, info, src) & 0xffff);
                        slot[x] = -1;
                        val[x] = 0.0;
                        if (u + x < nkb && lane < w) {
                            slot[x] = p.slotmap[(uint64_t)co + lane];
                            val[x] = (double)vals[(uint64_t)vo + lane];
                        }
                    }
#pragma unroll
                    for (int x = 0; x < kRowBatch; x++) {
                        if (u + x < nkb) {
                            if constexpr (U) {
                                // Multiplier 1: val + buf is fma(val, 1, buf) bit for bit.
                                if (slot[x] >= 0)
                                    buf[slot[x]] = val[x] + buf[slot[x]];
                            } else {
                                const double m = __shfl_sync(0xffffffffu, mult, (u + x) & 31);
                                if (slot[x] >= 0)
                                    buf[slot[x]] = fma(val[x], m, buf[slot[x]]);
                            }
                            __syncwarp();
                        }
                    }
                }
            } else {
                for (int x = 0; x < nkb; x++) {
                    const uint32_t vo = __shfl_sync(0xffffffffu, voff, x);
                    const uint32_t co = __shfl_sync(0xffffffffu, coo, x);
                    const double m = __shfl_sync(0xffffffffu, mult, x);
                    const int inf = __shfl_sync(0xffffffffu, info, x);
                    row_add_generic(buf, inf & 0xffff, m, vals + vo, p.slotmap + co, (inf & kSerial) != 0, lane);
                    __syncwarp();
                }
            }
        }
        const uint32_t a0 = __shfl_sync(0xffffffffu, a_lo, rr), a1 = __shfl_sync(0xffffffffu, a_lo, rr + 1);
        const uint32_t d0 = __shfl_sync(0xffffffffu, d_lo, rr), d1 = __shfl_sync(0xffffffffu, d_lo, rr + 1);
        const int la = (int)(a1 - a0), L = la + (int)(d1 - d0);
        const int64_t r = r0 + rr;
        if (p.dense != nullptr) {
            if (lane == 0)
                p.dense[r] = L > 0 ? -buf[0] : 0.0;
            __syncwarp();
            for (int s = lane; s < L; s += 32) buf[s] = 0.0;
        } else {
            for (int s = lane; s < L; s += 32) {
                const double v = buf[s];
                buf[s] = 0.0;
                if (s < la)
                    p.Avals[a0 + s] = v;
                else
                    p.Dvals[d0 + (s - la)] = v;
            }
        }
        __syncwarp();
    }
}

}  // namespace slgpu
