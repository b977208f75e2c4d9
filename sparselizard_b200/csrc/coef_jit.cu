// Runtime-compiled geometry + coefficient kernels.
//
// The interpreter kernel (k_geometry_coef) walks a group's coefficient program
// instruction by instruction with its values in local memory.  Here the
// programs of all groups that share the same elements and Gauss points (the
// slices of one contribution) are turned into one straight-line CUDA kernel,
// compiled for sm_100a with NVRTC and cached by source text: the Jacobian is
// computed once per (element, Gauss point) and every program value lives in
// a register.  Results are written in the same [term][gp][element] layout.
#include "engine_internal.h"

#include <nvrtc.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <sstream>
#include <stdexcept>

namespace slgpu {

namespace {

const char* kPrelude = R"(
typedef long long i64;
struct JitGeom {
    const double* xyz;
    const int* conn;
    const int* elems;
    const int* orient;
    i64 nelem;
    const double* weights;
    const double* lagrange;
};
struct JitGroup {
    const double* tables;
    const double* elemdata;
    const double* fielddata;
    const double* term_scale;
    double* C;
    int* elemexp;
};
)";

std::string lit(double v)
{
    char buf[64];
    std::snprintf(buf, sizeof(buf), "(%a)", v);
    return buf;
}

}  // namespace

namespace {

// X, J, det J, the cofactor inverse I and wdet = w_g |det J| at element e,
// Gauss point g (as in src/field/jacobian.cpp:308-349, :396-504).
void emit_geometry(std::ostringstream& s, int dim, int ncn, int ngp, const char* indent)
{
    s << indent << "const int* cn = p.conn + (i64)p.elems[e] * " << ncn << ";\n";
    s << indent << "double X0 = 0, X1 = 0, X2 = 0;\n";
    for (int a = 0; a < dim; a++)
        for (int b = 0; b < dim; b++) s << indent << "double J" << a << b << " = 0;\n";
    s << indent << "#pragma unroll\n" << indent << "for (int k = 0; k < " << ncn << "; k++) {\n";
    s << indent << "  const i64 nd = 3 * (i64)cn[k];\n";
    s << indent << "  const double x0 = p.xyz[nd], x1 = p.xyz[nd + 1], x2 = p.xyz[nd + 2];\n";
    s << indent << "  const double nv = p.lagrange[k * " << ngp << " + g];\n";
    s << indent << "  X0 = fma(nv, x0, X0); X1 = fma(nv, x1, X1); X2 = fma(nv, x2, X2);\n";
    for (int a = 0; a < dim; a++) {
        s << indent << "  { const double dn = p.lagrange[(" << (1 + a) * ncn << " + k) * " << ngp << " + g];";
        for (int b = 0; b < dim; b++) s << " J" << a << b << " = fma(dn, x" << b << ", J" << a << b << ");";
        s << " }\n";
    }
    s << indent << "}\n";
    if (dim == 1) {
        s << indent << "const double det = J00;\n" << indent << "const double I00 = 1.0 / J00;\n";
    } else if (dim == 2) {
        s << indent << "const double det = J00 * J11 - J01 * J10;\n";
        s << indent << "const double I00 = J11 / det, I01 = -J01 / det, I10 = -J10 / det, I11 = J00 / det;\n";
    } else {
        s << indent << "const double det = J00 * (J11 * J22 - J21 * J12) - J01 * (J10 * J22 - J20 * J12) + J02 * (J10 * J21 - J20 * J11);\n";
        s << indent << "const double I00 = (J11 * J22 - J12 * J21) / det, I01 = (J02 * J21 - J01 * J22) / det, I02 = (J01 * J12 - J02 * J11) / det;\n";
        s << indent << "const double I10 = (J12 * J20 - J10 * J22) / det, I11 = (J00 * J22 - J02 * J20) / det, I12 = (J02 * J10 - J00 * J12) / det;\n";
        s << indent << "const double I20 = (J10 * J21 - J11 * J20) / det, I21 = (J01 * J20 - J00 * J21) / det, I22 = (J00 * J11 - J01 * J10) / det;\n";
    }
    s << indent << "const double wdet = p.weights[g] * fabs(det);\n";
}

// Program nodes the given terms depend on.
std::vector<char> node_closure(const GroupDev& G, const std::vector<int>& terms)
{
    const int n = (int)G.nodes.size();
    std::vector<char> needed(n, 0);
    for (int t : terms) needed[G.term_node[t]] = 1;
    for (int i = n - 1; i >= 0; i--) {
        if (!needed[i])
            continue;
        const slgpu_node& nd = G.nodes[i];
        if (nd.op == SLGPU_OP_ADD || nd.op == SLGPU_OP_MUL || nd.op == SLGPU_OP_POW)
            needed[nd.a] = needed[nd.b] = 1;
        if (nd.op == SLGPU_OP_INV || nd.op == SLGPU_OP_NEG)
            needed[nd.a] = 1;
    }
    return needed;
}

// `const double v<i> = ...;` for the needed nodes (q: the group's descriptor;
// e, o, g, J.., I.., det, X.. in scope).
void emit_nodes(std::ostringstream& s, const GroupDev& G, const std::vector<char>& needed, int ngp, const char* indent)
{
    for (int i = 0; i < (int)G.nodes.size(); i++) {
        if (!needed[i])
            continue;
        const slgpu_node& nd = G.nodes[i];
        if (nd.op == SLGPU_OP_FIELD) {
            // sum_f coefficient[f][e] * form function f at (orientation, gp)
            const int rows = G.tab_rows[nd.b];
            s << indent << "double v" << i << " = 0;\n";
            s << indent << "for (int f = 0; f < " << rows << "; f++) v" << i << " = fma(q.fielddata[(i64)" << G.field_off[nd.a]
              << " + (i64)f * p.nelem + e], q.tables[(i64)" << G.tab_off[nd.b] << " + ((i64)o * " << rows << " + f) * " << ngp
              << " + g], v" << i << ");\n";
            continue;
        }
        s << indent << "const double v" << i << " = ";
        switch (nd.op) {
        case SLGPU_OP_CONST: s << lit(G.hconsts[nd.a]); break;
        case SLGPU_OP_JAC: s << "J" << nd.a << nd.b; break;
        case SLGPU_OP_INVJAC: s << "I" << nd.a << nd.b; break;
        case SLGPU_OP_DETJAC: s << "det"; break;
        case SLGPU_OP_ELEM: s << "q.elemdata[(i64)" << nd.a << " * p.nelem + e]"; break;
        case SLGPU_OP_COORD: s << "X" << nd.a; break;
        case SLGPU_OP_ADD: s << "v" << nd.a << " + v" << nd.b; break;
        case SLGPU_OP_MUL: s << "v" << nd.a << " * v" << nd.b; break;
        case SLGPU_OP_INV: s << "1.0 / v" << nd.a; break;
        case SLGPU_OP_NEG: s << "-v" << nd.a; break;
        case SLGPU_OP_POW: s << "pow(v" << nd.a << ", v" << nd.b << ")"; break;
        default: throw std::runtime_error("unknown coefficient op");
        }
        s << ";\n";
    }
}

std::vector<int> all_terms(const GroupDev& G)
{
    std::vector<int> t(G.nterms);
    for (int k = 0; k < G.nterms; k++) t[k] = k;
    return t;
}

}  // namespace

std::string jit_coef_source(const std::vector<const GroupDev*>& batch)
{
    const GroupDev& g0 = *batch[0];
    const int dim = g0.problemdim, ncn = g0.ncn, ngp = g0.ngp;
    std::ostringstream s;
    s << kPrelude;
    // The batch's group descriptors are passed by value (kernel parameter
    // space), so that a launch needs no argument upload.
    s << "struct JitGroups { JitGroup g[" << batch.size() << "]; };\n";
    s << "extern \"C\" __global__ void __launch_bounds__(128) slgpu_coef(JitGeom p, const JitGroups grp)\n{\n";
    s << "  const i64 n = blockIdx.x * (i64)blockDim.x + threadIdx.x;\n";
    s << "  if (n >= p.nelem * " << ngp << ") return;\n";
    s << "  const int g = (int)(n / p.nelem);\n  const i64 e = n - (i64)g * p.nelem;\n";
    s << "  const int o = p.orient[e];\n";
    emit_geometry(s, dim, ncn, ngp, "  ");
    s << "  (void)o; (void)X0; (void)X1; (void)X2;\n";
    for (size_t k = 0; k < batch.size(); k++) {
        const GroupDev& G = *batch[k];
        // A group whose coefficients are not needed in this launch (the
        // second group of a transposed pair) gets C = null.
        s << "  if (grp.g[" << k << "].C != nullptr) {\n    const JitGroup q = grp.g[" << k << "];\n";
        emit_nodes(s, G, node_closure(G, all_terms(G)), ngp, "    ");
        s << "    double cmax = 0;\n";
        for (int t = 0; t < G.nterms; t++) {
            const int c = G.term_node[t];
            s << "    { const double c = v" << c << " * q.term_scale[" << t << "] * wdet; q.C[((i64)" << t << " * " << ngp
              << " + g) * p.nelem + e] = c; cmax = fmax(cmax, fabs(c)); }\n";
        }
        // Exponent of the element's largest coefficient for split precision.
        s << "    if (q.elemexp != nullptr && cmax > 0) { int ex; frexp(cmax, &ex); atomicMax(q.elemexp + e, ex); }\n";
        s << "  }\n";
    }
    s << "}\n";
    return s.str();
}

std::vector<char> jit_compile(const std::string& src)
{
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), "slgpu_coef.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
        throw std::runtime_error("nvrtcCreateProgram failed");
    // No implicit multiply-add contraction: a coefficient program rounds the
    // same however the compiler schedules it; the sums of products (Jacobian,
    // coordinates, field values) are written as explicit fma.
    const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-default-device", "--fmad=false"};
    nvrtcResult r = nvrtcCompileProgram(prog, 4, opts);
    if (r != NVRTC_SUCCESS) {
        size_t n = 0;
        nvrtcGetProgramLogSize(prog, &n);
        std::string log(n, '\0');
        nvrtcGetProgramLog(prog, &log[0]);
        nvrtcDestroyProgram(&prog);
        throw std::runtime_error("NVRTC compile of a coefficient kernel failed: " + log.substr(0, 2000));
    }
    size_t n = 0;
    nvrtcGetCUBINSize(prog, &n);
    std::vector<char> cubin(n);
    nvrtcGetCUBIN(prog, cubin.data());
    nvrtcDestroyProgram(&prog);
    return cubin;
}

cudaKernel_t jit_coef_kernel(Ctx* ctx, const std::string& src)
{
    auto it = ctx->jit_kernels.find(src);
    if (it != ctx->jit_kernels.end())
        return it->second;
    std::vector<char> cubin = jit_compile(src);
    cudaLibrary_t lib;
    cudaError_t e = cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e != cudaSuccess)
        throw std::runtime_error(std::string("cudaLibraryLoadData: ") + cudaGetErrorString(e));
    cudaKernel_t k;
    e = cudaLibraryGetKernel(&k, lib, "slgpu_coef");
    if (e != cudaSuccess)
        throw std::runtime_error(std::string("cudaLibraryGetKernel: ") + cudaGetErrorString(e));
    ctx->jit_libs.push_back(lib);
    ctx->jit_kernels[src] = k;
    return k;
}

}  // namespace slgpu
