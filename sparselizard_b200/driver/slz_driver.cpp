// Assembly workloads written as ordinary sparselizard user programs.
//
// Each workload builds a mesh, fields and a formulation with sparselizard's
// public API and then runs generate(), A() and b()
// (src/formulation/formulation.h:68-111).  The same source is compiled twice:
// once against stock sparselizard and once against sparselizard with the two
// GPU translation units (contribution.cpp, rawmat.cpp) swapped in, so both
// builds answer the same calls.  The results (A/D CSR blocks, Ainds/Dinds and
// b) and the per-phase wall times are exposed through the extern "C" functions
// at the end of the file for the Python harness.
#include "sparselizard.h"
#ifdef SLZ_GPU_BUILD
#include "slgpu_adapter.h"
#endif

#include <chrono>
#include <memory>
#include <stdexcept>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

using namespace sl;

namespace {

// Physical regions written by sparselizard_b200/meshgen.py.
const int VOL = 1, BOUNDARY = 2, CLAMP = 3, ORDER_REGION_BASE = 10, MATERIAL_REGION_BASE = 20;

struct Result {
    std::vector<int> Arows, Acols, Drows, Dcols, Ainds, Dinds;
    std::vector<double> Avals, Dvals, b;
    long long ndofs = 0;
};

Result g_result;
std::string g_error;
// The last captured matrix and right-hand side (kept for slz_eliminate).
mat g_lastA;
vec g_lastb;

double now_s(void)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Deterministic standard normal draws (SplitMix64 + Box-Muller) so that both
// builds see identical coefficients without depending on a library RNG.
struct Normal {
    uint64_t s;
    explicit Normal(uint64_t seed) : s(seed) {}
    uint64_t next(void)
    {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform(void) { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    double draw(void)
    {
        double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
    // Both normals of one Box-Muller step.
    void draw2(double& a, double& b)
    {
        const double r = std::sqrt(-2.0 * std::log(uniform())), t = 6.283185307179586 * uniform();
        a = r * std::cos(t);
        b = r * std::sin(t);
    }
};

void capture(mat& A, vec& b)
{
    Result r;
    std::shared_ptr<rawmat> raw = A.getpointer();
    indexmat ainds = raw->getainds(), dinds = raw->getdinds();
    r.Ainds.assign(ainds.getvalues(), ainds.getvalues() + ainds.count());
    r.Dinds.assign(dinds.getvalues(), dinds.getvalues() + dinds.count());
    r.ndofs = raw->countrows();
    PetscInt m, n;
    const PetscInt *rows, *cols;
    const PetscScalar* vals;
    if (slshim_mat_csr(raw->getapetsc(), &m, &n, &rows, &cols, &vals) == 0) {
        r.Arows.assign(rows, rows + m + 1);
        r.Acols.assign(cols, cols + rows[m]);
        r.Avals.assign(vals, vals + rows[m]);
    }
    if (slshim_mat_csr(raw->getdpetsc(), &m, &n, &rows, &cols, &vals) == 0) {
        r.Drows.assign(rows, rows + m + 1);
        r.Dcols.assign(cols, cols + rows[m]);
        r.Dvals.assign(vals, vals + rows[m]);
    }
    Vec bp = b.getpetsc();
    PetscInt blen;
    VecGetSize(bp, &blen);
    r.b.assign(slshim_vec_array(bp), slshim_vec_array(bp) + blen);
    g_result = std::move(r);
    g_lastA = A;
    g_lastb = b;
}

// Runs generate(), A(), b() `reps` times; times[3*i + {0,1,2}] receive the
// wall seconds of each phase of repetition i.  The last repetition's output
// is kept.
void run_reps(formulation& f, int reps, double* times)
{
    for (int i = 0; i < reps; i++) {
        double t0 = now_s();
        f.generate();
        double t1 = now_s();
        mat A = f.A();
        double t2 = now_s();
        vec b = f.b();
        double t3 = now_s();
        if (times != nullptr) {
            times[3 * i + 0] = t1 - t0;
            times[3 * i + 1] = t2 - t1;
            times[3 * i + 2] = t3 - t2;
        }
        if (i == reps - 1)
            capture(A, b);
    }
}

struct Problem {
    mesh m;
    std::vector<field> fields;
    std::vector<parameter> params;  // created after the mesh
    formulation f;
};

// Poisson on quadrangles: integral(vol, -grad(dof(v))*grad(tf(v)), -2) +
// integral(vol, 1*tf(v), -2), v = 0 on the boundary.
void poisson_quad(Problem& P, const char* msh, int order)
{
    P.m = mesh(msh, 0);
    field v("h1");
    v.setorder(VOL, order);
    v.setconstraint(BOUNDARY);
    P.f += integral(VOL, -grad(dof(v)) * grad(tf(v)), -2);
    P.f += integral(VOL, 1 * tf(v), -2);
    P.fields = {v};
}

// Sets a "one" field to one value per element of region `reg` (element order of
// the field's DOF numbering, as used by sparselizard's hp-adaptivity,
// src/mesh/rawmesh.cpp:880-910).
void set_per_element(field& E, int reg, const std::vector<double>& values)
{
    formulation fe;
    fe += integral(reg, dof(E) * tf(E));
    vec v(fe);
    int n = v.size();
    densemat vals(n, 1);
    for (int i = 0; i < n; i++)
        vals.getvalues()[i] = values[i % values.size()];
    v.setvalues(indexmat(n, 1, 0, 1), vals);
    E.setdata(reg, v);
}

// 3D linear elasticity, vector h1 field, per-element lognormal E, nu = 0.3,
// bottom face clamped: integral(vol, predefinedelasticity(dof(u), tf(u), E, nu), delta).
void elasticity_hex(Problem& P, const char* msh, int order, int delta)
{
    P.m = mesh(msh, 0);
    field u("h1xyz"), E("one");
    u.setorder(VOL, order);
    u.setconstraint(CLAMP);
    Normal rng(12345);
    std::vector<double> evals(1 << 22);
    for (double& e : evals) e = 150e9 * std::exp(0.3 * rng.draw());
    set_per_element(E, VOL, evals);
    P.f += integral(VOL, predefinedelasticity(dof(u), tf(u), E, 0.3), delta);
    P.fields = {u, E};
}

// p-adaptive scalar Helmholtz on tets: region ORDER_REGION_BASE+p holds the
// order-p elements (p = 1..5); orders are set in descending order.
void helmholtz_tet(Problem& P, const char* msh)
{
    P.m = mesh(msh, 0);
    int vol = selectunion({ORDER_REGION_BASE + 1, ORDER_REGION_BASE + 2, ORDER_REGION_BASE + 3, ORDER_REGION_BASE + 4, ORDER_REGION_BASE + 5});
    field p("h1");
    for (int ord = 5; ord >= 1; ord--)
        p.setorder(ORDER_REGION_BASE + ord, ord);
    P.f += integral(vol, grad(dof(p)) * grad(tf(p)) - 400.0 * dof(p) * tf(p));
    P.fields = {p};
}

// Harmonic eddy currents on tets, hcurl order 2 with harmonics {2,3}:
// integral(vol, curl(dof(a))*curl(tf(a))/mu + sigma*dt(dof(a))*tf(a)),
// sigma per material region, at fundamental frequency `freq`.
void eddy_tet(Problem& P, const char* msh, int order, const double* sigmas, double freq)
{
    P.m = mesh(msh, 0);
    int vol = selectunion({MATERIAL_REGION_BASE, MATERIAL_REGION_BASE + 1, MATERIAL_REGION_BASE + 2, MATERIAL_REGION_BASE + 3});
    setfundamentalfrequency(freq);
    field a("hcurl", {2, 3});
    a.setorder(vol, order);
    parameter sigma;
    for (int r = 0; r < 4; r++)
        sigma.setvalue(MATERIAL_REGION_BASE + r, sigmas[r]);
    double mu = 4.0 * 3.141592653589793 * 1e-7;
    P.f += integral(vol, curl(dof(a)) * curl(tf(a)) / mu + sigma * dt(dof(a)) * tf(a));
    P.params = {sigma};
    P.fields = {a};
}

// Poisson on quads as workload 1, with the non-zero Dirichlet value
// v = 1 + x*y + 2*x^2 on the boundary: b() then projects it onto the
// boundary form functions (rawvec::updatedisjregconstraints,
// src/formulation/rawvec.cpp:142-214).
void poisson_quad_dirichlet(Problem& P, const char* msh, int order)
{
    P.m = mesh(msh, 0);
    field v("h1"), x("x"), y("y");
    v.setorder(VOL, order);
    v.setconstraint(BOUNDARY, 1 + x * y + 2 * x * x);
    P.f += integral(VOL, -grad(dof(v)) * grad(tf(v)), -2);
    P.f += integral(VOL, 1 * tf(v), -2);
    P.fields = {v};
}

// Elasticity on hexes as workload 2 with a prescribed displacement
// u = (1e-3 x y, 0, 2e-3 x) on the z = 0 face (projected onto the face,
// edge and node form functions of that face).
void elasticity_hex_dirichlet(Problem& P, const char* msh, int order)
{
    P.m = mesh(msh, 0);
    field u("h1xyz"), E("one"), x("x"), y("y");
    u.setorder(VOL, order);
    u.setconstraint(CLAMP, array3x1(1e-3 * x * y, 0, 2e-3 * x));
    Normal rng(12345);
    std::vector<double> evals(1 << 16);
    for (double& e : evals) e = 150e9 * std::exp(0.3 * rng.draw());
    set_per_element(E, VOL, evals);
    P.f += integral(VOL, predefinedelasticity(dof(u), tf(u), E, 0.3));
    P.fields = {u, E};
}

// Per-element values for workload 7 (slz_set_element_values).
std::vector<double> g_element_values;

// Poisson on quads with a per-element coefficient field k (a "one" field set
// from g_element_values): integral(VOL, -k*grad(dof(v))*grad(tf(v))), v = 0
// on the boundary -- the formulation of the serving pool's Poisson templates.
void poisson_quad_kfield(Problem& P, const char* msh, int order)
{
    P.m = mesh(msh, 0);
    field v("h1"), k("one");
    v.setorder(VOL, order);
    v.setconstraint(BOUNDARY);
    set_per_element(k, VOL, g_element_values.empty() ? std::vector<double>{1.0} : g_element_values);
    P.f += integral(VOL, -k * grad(dof(v)) * grad(tf(v)));
    P.fields = {v, k};
}

// Workload 8: Poisson on quads (as workload 1, at order `order`) assembled
// after another formulation on the same mesh -- a field of order `order` + 1
// with its own dofmanager -- was generated and left unprocessed.
void poisson_quad_after_other(Problem& P, const char* msh, int order)
{
    P.m = mesh(msh, 0);
    field v("h1"), w("h1");
    v.setorder(VOL, order);
    w.setorder(VOL, order + 1);
    v.setconstraint(BOUNDARY);
    w.setconstraint(BOUNDARY);
    formulation other;
    other += integral(VOL, grad(dof(w)) * grad(tf(w)) + dof(w) * tf(w));
    other.generate();
    P.f += integral(VOL, -grad(dof(v)) * grad(tf(v)), -2);
    P.f += integral(VOL, 1 * tf(v), -2);
    P.fields = {v, w};
}

std::unique_ptr<Problem> build(int workload, const char* msh, const double* params)
{
    auto P = std::make_unique<Problem>();
    switch (workload) {
    case 1: poisson_quad(*P, msh, (int)params[0]); break;
    case 2: elasticity_hex(*P, msh, (int)params[0], (int)params[1]); break;
    case 3: helmholtz_tet(*P, msh); break;
    case 4: eddy_tet(*P, msh, (int)params[0], params + 2, params[1]); break;
    case 5: poisson_quad_dirichlet(*P, msh, (int)params[0]); break;
    case 6: elasticity_hex_dirichlet(*P, msh, (int)params[0]); break;
    case 7: poisson_quad_kfield(*P, msh, (int)params[0]); break;
    case 8: poisson_quad_after_other(*P, msh, (int)params[0]); break;
    default: throw std::runtime_error("unknown workload");
    }
    return P;
}

} // namespace

extern "C" {

// Workload ids: 1 Poisson quads (param0 = order), 2 elasticity hexes
// (param0 = order, param1 = integration delta), 3 p-adaptive Helmholtz tets,
// 4 harmonic eddy current tets (param0 = order, param1 = frequency,
// param2..5 = sigma per material region), 5 Poisson quads with a non-zero
// Dirichlet value (param0 = order), 6 elasticity hexes with a prescribed
// face displacement (param0 = order), 7 Poisson quads with a per-element
// coefficient field from slz_set_element_values (param0 = order).
int slz_run(int workload, const char* msh, const double* params, int reps, double* times)
{
    g_error.clear();
    try {
        std::unique_ptr<Problem> P = build(workload, msh, params);
        run_reps(P->f, reps, times);
    } catch (const std::exception& e) {
        g_error = e.what();
        if (g_error.empty())
            g_error = "sparselizard raised an error (message printed on stdout)";
        return 2;
    }
    return 0;
}

const char* slz_last_error(void) { return g_error.c_str(); }

// 0 ndofs, 1 len(Arows), 2 nnzA, 3 len(Drows), 4 nnzD, 5 len(Ainds), 6 len(Dinds), 7 len(b)
long long slz_result_size(int which)
{
    const Result& r = g_result;
    switch (which) {
    case 0: return r.ndofs;
    case 1: return (long long)r.Arows.size();
    case 2: return (long long)r.Acols.size();
    case 3: return (long long)r.Drows.size();
    case 4: return (long long)r.Dcols.size();
    case 5: return (long long)r.Ainds.size();
    case 6: return (long long)r.Dinds.size();
    case 7: return (long long)r.b.size();
    }
    return -1;
}

void slz_result_copy(int* Arows, int* Acols, double* Avals, int* Drows, int* Dcols, double* Dvals, int* Ainds, int* Dinds, double* b)
{
    const Result& r = g_result;
    std::memcpy(Arows, r.Arows.data(), r.Arows.size() * sizeof(int));
    std::memcpy(Acols, r.Acols.data(), r.Acols.size() * sizeof(int));
    std::memcpy(Avals, r.Avals.data(), r.Avals.size() * sizeof(double));
    std::memcpy(Drows, r.Drows.data(), r.Drows.size() * sizeof(int));
    std::memcpy(Dcols, r.Dcols.data(), r.Dcols.size() * sizeof(int));
    std::memcpy(Dvals, r.Dvals.data(), r.Dvals.size() * sizeof(double));
    std::memcpy(Ainds, r.Ainds.data(), r.Ainds.size() * sizeof(int));
    std::memcpy(Dinds, r.Dinds.data(), r.Dinds.size() * sizeof(int));
    std::memcpy(b, r.b.data(), r.b.size() * sizeof(double));
}

void slz_set_threads(int n) { setmaxnumthreads(n); }

// Per-element coefficient values of workload 7, in element order.
void slz_set_element_values(const double* v, long long n) { g_element_values.assign(v, v + n); }

// mat::eliminate (src/formulation/mat.cpp:78-103) of the last captured matrix
// applied to the vector x [ndofs]: out [nA] = x_A - D x_D.  Returns nA, or -1.
long long slz_eliminate(const double* x, double* out)
{
    g_error.clear();
    try {
        const int n = g_lastb.size();
        vec xv = g_lastb.copy();
        densemat vals(n, 1);
        std::memcpy(vals.getvalues(), x, (size_t)n * sizeof(double));
        xv.setvalues(indexmat(n, 1, 0, 1), vals);
        vec e = g_lastA.eliminate(xv);
        densemat ev = e.getallvalues();
        if (out != nullptr)
            std::memcpy(out, ev.getvalues(), (size_t)ev.count() * sizeof(double));
        return ev.count();
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// Field interpolation and integration: v (h1, order `order`) is set on the
// quadrangle mesh by projection (rawfield::setvalue), then
// e = v*v*x + 3*y - 2 is integrated over the volume at Gauss order 4.
// out[0]: expression::integrate (sparselizard's own, on the host); in the
// GPU drop-in build out[1]: the same integral through the GPU lowering
// (slgpu_adapter::integrate), else out[1] = out[0].
int slz_integrate(const char* msh, int order, double* out)
{
    g_error.clear();
    try {
        mesh m(msh, 0);
        field v("h1"), x("x"), y("y");
        v.setorder(VOL, order);
        v.setvalue(VOL, 1 + x * y + 2 * x * x);
        expression e = v * v * x + 3 * y - 2;
        out[0] = e.integrate(VOL, 4);
#ifdef SLZ_GPU_BUILD
        out[1] = slgpu_adapter::integrate(e, VOL, 4);
#else
        out[1] = out[0];
#endif
    } catch (const std::exception& e) {
        g_error = e.what();
        return 2;
    }
    return 0;
}

// Releases the last captured matrix and right-hand side.
void slz_release_last(void)
{
    g_lastA = mat();
    g_lastb = vec();
}

}

#ifdef SLZ_GPU_BUILD
// Benchmark support (GPU drop-in build only): keeps one problem resident after
// a first generate()/A()/b() so that the engine matrix it produced can be
// re-assembled on its resident pattern through the C ABI.
#include "slgpu_adapter.h"

namespace {
struct BenchState {
    std::unique_ptr<Problem> P;
    mat A;
    vec b;
    std::vector<unsigned char> constrained;
};
std::unique_ptr<BenchState> g_bench;
}  // namespace

extern "C" {

// times3: generate / A / b wall seconds of the first assembly; info4: engine
// matrix handle, ndofs, nnzA, nnzD.
int slz_bench_prepare(int workload, const char* msh, const double* params, double* times3, long long* info4)
{
    g_error.clear();
    try {
        g_bench.reset();
        auto B = std::make_unique<BenchState>();
        B->P = build(workload, msh, params);
        double t0 = now_s();
        B->P->f.generate();
        double t1 = now_s();
        B->A = B->P->f.A();
        double t2 = now_s();
        B->b = B->P->f.b();
        double t3 = now_s();
        times3[0] = t1 - t0;
        times3[1] = t2 - t1;
        times3[2] = t3 - t2;
        std::shared_ptr<rawmat> raw = B->A.getpointer();
        std::vector<bool> c = raw->getdofmanager()->isconstrained();
        B->constrained.assign(c.begin(), c.end());
        info4[0] = slgpu_adapter::find_matrix_handle(raw.get());
        info4[1] = raw->countrows();
        info4[2] = raw->countnnz();
        info4[3] = B->A.getdinds().count();
        g_bench = std::move(B);
    } catch (const std::exception& e) {
        g_error = e.what();
        return 2;
    }
    return 0;
}

// Warm generate(), A(), b() of the resident problem, `reps` times: the drop-in's
// repeated path (the pattern is found in the engine's resident cache).
// times[3*i + {0,1,2}] receive the phase wall seconds of repetition i; info4
// as for slz_bench_prepare (the matrix handle changes with every A()).
int slz_bench_reassemble(int reps, double* times, long long* info4)
{
    g_error.clear();
    try {
        if (!g_bench)
            throw std::runtime_error("no resident problem");
        for (int i = 0; i < reps; i++) {
            g_bench->A = mat();
            g_bench->b = vec();
            double t0 = now_s();
            g_bench->P->f.generate();
            double t1 = now_s();
            g_bench->A = g_bench->P->f.A();
            double t2 = now_s();
            g_bench->b = g_bench->P->f.b();
            double t3 = now_s();
            times[3 * i + 0] = t1 - t0;
            times[3 * i + 1] = t2 - t1;
            times[3 * i + 2] = t3 - t2;
        }
        std::shared_ptr<rawmat> raw = g_bench->A.getpointer();
        info4[0] = slgpu_adapter::find_matrix_handle(raw.get());
        info4[1] = raw->countrows();
        info4[2] = raw->countnnz();
        info4[3] = g_bench->A.getdinds().count();
    } catch (const std::exception& e) {
        g_error = e.what();
        return 2;
    }
    return 0;
}

// Engine handle of the last matrix captured by slz_run.
int slz_last_matrix_handle(void)
{
    std::shared_ptr<rawmat> raw = g_lastA.getpointer();
    return raw ? slgpu_adapter::find_matrix_handle(raw.get()) : 0;
}

const unsigned char* slz_bench_constraints(void) { return g_bench ? g_bench->constrained.data() : nullptr; }

// Node coordinates of the resident mesh in sparselizard's numbering.
long long slz_bench_nodes(const double** xyz)
{
    std::vector<double>* c = universe::getrawmesh()->getnodes()->getcoordinates();
    *xyz = c->data();
    return (long long)c->size() / 3;
}

void slz_bench_release(void) { g_bench.reset(); }
}

// ---------------------------------------------------------------- serving
// A pool of resident problems (each assembled once through generate()/A(),
// which leaves its mesh, tables, addresses and pattern on the device) and a
// stream of requests that re-assemble them with new per-element coefficient
// fields through the engine's request server.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>

namespace {
struct ServeProblem {
    std::unique_ptr<Problem> P;
    mat A;
    int handle = 0;
    long long nnzA = 0, nnzD = 0, nmesh = 0, ndofs = 0;
    double median = 1.0;
    std::vector<int> groups;  // groups whose fielddata array 0 is the coefficient field
};
std::vector<std::unique_ptr<ServeProblem>> g_serve;

// exp(0.3 z) at the 65536 quantiles z_i = Phi^-1((i + 0.5) / 65536) of the
// standard normal: a request's per-element lognormal field (sigma 0.3) is one
// uniform 16-bit draw per element into this table (Phi^-1 by bisection on
// erfc, exact to double rounding).
const std::vector<double>& lognormal_table(void)
{
    static const std::vector<double> T = [] {
        std::vector<double> t(65536);
        for (int i = 0; i < 65536; i++) {
            const double p = (i + 0.5) / 65536.0;
            double lo = -10, hi = 10;
            for (int it = 0; it < 80; it++) {
                const double mid = 0.5 * (lo + hi);
                (0.5 * std::erfc(-mid / std::sqrt(2.0)) < p ? lo : hi) = mid;
            }
            t[i] = std::exp(0.3 * 0.5 * (lo + hi));
        }
        return t;
    }();
    return T;
}
}  // namespace

extern "C" {

// kind 1: Poisson, integral(VOL, -k*grad(dof(v))*grad(tf(v))), v = 0 on
// BOUNDARY (2D) or CLAMP (3D); kind 2: elasticity,
// integral(VOL, predefinedelasticity(dof(u), tf(u), E, 0.3)) (plane strain in
// 2D), u = 0 on the same region.  k / E is a "one" field with one value per
// element.  info6: handle, nnzA, nnzD, mesh elements, groups, ndofs.
int slz_serve_add(int kind, const char* msh, int dim, int order, long long* info6)
{
    g_error.clear();
    try {
        auto S = std::make_unique<ServeProblem>();
        S->P = std::make_unique<Problem>();
        Problem& P = *S->P;
        P.m = mesh(msh, 0);
        field c("one");
        const int fixreg = dim == 2 ? BOUNDARY : CLAMP;
        S->median = kind == 1 ? 1.0 : 150e9;
        set_per_element(c, VOL, {S->median});
        if (kind == 1) {
            field v("h1");
            v.setorder(VOL, order);
            v.setconstraint(fixreg);
            P.f += integral(VOL, -c * grad(dof(v)) * grad(tf(v)));
            P.fields = {v, c};
        } else {
            field u(dim == 2 ? "h1xy" : "h1xyz");
            u.setorder(VOL, order);
            u.setconstraint(fixreg);
            P.f += integral(VOL, predefinedelasticity(dof(u), tf(u), c, 0.3, dim == 2 ? "planestrain" : ""));
            P.fields = {u, c};
        }
        P.f.generate();
        S->A = P.f.A();
        std::shared_ptr<rawmat> raw = S->A.getpointer();
        S->handle = slgpu_adapter::find_matrix_handle(raw.get());
        S->ndofs = raw->countrows();
        slgpu_ctx* ctx = slgpu_adapter_ctx();
        int ng = 0;
        if (slgpu_matrix_group_count(ctx, S->handle, &ng) != SLGPU_OK)
            throw std::runtime_error("template has no engine matrix");
        for (int gi = 0; gi < ng; gi++) {
            slgpu_group_desc d;
            slgpu_matrix_group_desc(ctx, S->handle, gi, &d);
            if (d.nfielddata != 1 || d.fieldrows[0] != 1)
                throw std::runtime_error("a served group must hold exactly the per-element coefficient field");
            if (S->nmesh != 0 && S->nmesh != d.mesh_nelem)
                throw std::runtime_error("groups of one template on different element types");
            S->nmesh = d.mesh_nelem;
            S->groups.push_back(gi);
        }
        // nnzA and nnzD of the resident pattern (the engine's last process).
        slgpu_work w;
        if (slgpu_matrix_work(ctx, S->handle, &w) != SLGPU_OK)
            throw std::runtime_error("slgpu_matrix_work failed");
        S->nnzA = raw->countnnz();
        S->nnzD = w.nnz - S->nnzA;
        info6[0] = S->handle;
        info6[1] = S->nnzA;
        info6[2] = S->nnzD;
        info6[3] = S->nmesh;
        info6[4] = (long long)S->groups.size();
        info6[5] = S->ndofs;
        g_serve.push_back(std::move(S));
        return (int)g_serve.size() - 1;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -2;
    }
}

// Relative Frobenius error of pool problem `idx`'s assembled values (A and D)
// in split precision (err2[0]) and in the FP32-level tier (err2[1]) against
// the plain FP64 path, each re-assembled on the resident pattern.
int slz_serve_error(int idx, double* err2)
{
    g_error.clear();
    try {
        if (idx < 0 || idx >= (int)g_serve.size())
            throw std::runtime_error("no such pool problem");
        ServeProblem& S = *g_serve[idx];
        slgpu_ctx* ctx = slgpu_adapter_ctx();
        std::shared_ptr<rawmat> raw = S.A.getpointer();
        std::vector<bool> cb = raw->getdofmanager()->isconstrained();
        std::vector<unsigned char> con(cb.begin(), cb.end());
        auto values = [&](int prec) {
            slgpu_csr_info info{};
            if (slgpu_matrix_process(ctx, S.handle, con.data(), prec, &info) != SLGPU_OK)
                throw std::runtime_error("process failed");
            std::vector<double> v((size_t)(info.nnzA + info.nnzD) + 1);
            if (slgpu_matrix_download_values(ctx, S.handle, v.data(), v.data() + info.nnzA) != SLGPU_OK)
                throw std::runtime_error("download failed");
            v.pop_back();
            return v;
        };
        const std::vector<double> ref = values(SLGPU_PREC_FP64);
        const int precs[2] = {SLGPU_PREC_SPLIT, SLGPU_PREC_FP32};
        for (int k = 0; k < 2; k++) {
            const std::vector<double> v = values(precs[k]);
            double num = 0, den = 0;
            for (size_t i = 0; i < ref.size(); i++) {
                num += (v[i] - ref[i]) * (v[i] - ref[i]);
                den += ref[i] * ref[i];
            }
            err2[k] = den > 0 ? std::sqrt(num / den) : 0.0;
        }
    } catch (const std::exception& e) {
        g_error = e.what();
        return 2;
    }
    return 0;
}

// Runs `nreq` requests arriving as a Poisson process of `rate` per second
// (seeded), each on a problem drawn uniformly from the pool with a new
// lognormal coefficient field (median of the problem, sigma 0.3, one seeded
// draw per element from 65536 quantile levels), through a
// server with `nslots` slots.  ngen threads prepare the coefficient fields
// ahead of their arrival times.  Per request: latency (scheduled arrival to
// results in host memory), completion time and device time (seconds, ms);
// summary: [0] wall seconds from the first arrival to the last completion,
// [1] sum of nnz, [2] sum of device ms, [3] requests whose submission was late
// by more than 1 ms, [4] mean host ms the server spent issuing a request,
// [5] mean ms a request waited in the queue, [6..8] mean host ms of the
// launch parts (inputs, contractions, values and copies).
int slz_serve_run_warm(int nwarm, int nreq, double rate, int nslots, int precision, unsigned long long seed, int ngen, double* latency_out,
                       double* done_out, double* device_out, int* problem_out, double* detail_out, double* summary);

int slz_serve_run(int nreq, double rate, int nslots, int precision, unsigned long long seed, int ngen, double* latency, double* done_s,
                  double* device_ms, int* problem, double* summary)
{
    return slz_serve_run_warm(0, nreq, rate, nslots, precision, seed, ngen, latency, done_s, device_ms, problem, nullptr, summary);
}

// As slz_serve_run, with `nwarm` requests of the same stream before the
// measured ones (same server, so page-locked pools and split-precision
// tables are warm); the outputs and summary cover the last `nreq` requests.
// detail_out (optional): per measured request, server-thread launch time and
// its three parts (ms), queueing time (ms) and submission delay behind the
// scheduled arrival (ms).
int slz_serve_run_warm(int nwarm, int nreq, double rate, int nslots, int precision, unsigned long long seed, int ngen, double* latency_out,
                       double* done_out, double* device_out, int* problem_out, double* detail_out, double* summary)
{
    const int ntot = nwarm + nreq;
    constexpr int kDetail = 6;
    std::vector<double> latency(ntot), done_s(ntot), device_ms(ntot), detail((size_t)ntot * kDetail);
    std::vector<int> problem(ntot);
    g_error.clear();
    const int np = (int)g_serve.size();
    if (np == 0 || ntot <= 0) {
        g_error = "no served problems";
        return -1;
    }
    slgpu_ctx* ctx = slgpu_adapter_ctx();
    slgpu_server* srv = nullptr;
    if (slgpu_server_create(ctx, nslots, &srv) != SLGPU_OK) {
        g_error = "slgpu_server_create failed";
        return -1;
    }
    // Every slot's device scratch sized for every problem before the stream.
    for (int p = 0; p < np; p++)
        if (slgpu_server_prepare(srv, g_serve[p]->handle, precision) != SLGPU_OK) {
            char buf[512];
            slgpu_last_error(ctx, buf, sizeof(buf));
            g_error = std::string("slgpu_server_prepare: ") + buf;
            slgpu_server_destroy(srv);
            return -1;
        }
    // Schedule.
    Normal rs(seed);
    std::vector<double> arrival(ntot);
    double t = 0.05;
    for (int k = 0; k < ntot; k++) {
        t += -std::log(rs.uniform()) / rate;
        arrival[k] = t;
        problem[k] = (int)(rs.next() % (uint64_t)np);
    }
    // Output buffers: page-locked pairs per problem, enough for about half a
    // second of its arrivals (at least 4), so that a slow request does not
    // hold back the submission of later ones.  Input buffers likewise:
    // page-locked, so that the server reads them in place (no copy at submit).
    std::vector<int> nbuf(np);
    for (int p = 0; p < np; p++) nbuf[p] = std::max(4, (int)std::ceil(0.5 * rate / np) + 2);
    std::vector<std::vector<std::pair<double*, double*>>> free_out(np);
    std::vector<std::vector<double*>> free_in(np);
    std::vector<void*> pinned;
    for (int p = 0; p < np; p++)
        for (int b = 0; b < nbuf[p]; b++) {
            void *a = nullptr, *d = nullptr, *in = nullptr;
            slgpu_host_alloc(ctx, (size_t)std::max(1LL, g_serve[p]->nnzA) * 8, &a);
            slgpu_host_alloc(ctx, (size_t)std::max(1LL, g_serve[p]->nnzD) * 8, &d);
            slgpu_host_alloc(ctx, (size_t)std::max(1LL, g_serve[p]->nmesh) * 8, &in);
            if (a == nullptr || d == nullptr || in == nullptr) {
                g_error = "page-locked request buffers";
                for (void* q : {a, d, in})
                    if (q != nullptr)
                        slgpu_host_free(q);
                for (void* q : pinned) slgpu_host_free(q);
                slgpu_server_destroy(srv);
                return -1;
            }
            pinned.push_back(a);
            pinned.push_back(d);
            pinned.push_back(in);
            free_out[p].push_back({(double*)a, (double*)d});
            free_in[p].push_back((double*)in);
        }
    lognormal_table();
    // Time origin of the arrivals: after the set-up above.
    const auto t_create = std::chrono::steady_clock::now();
    const double offset = slgpu_server_clock(srv);  // server time at t_create
    std::mutex mu;
    std::condition_variable cv;
    // Prepared inputs (lookahead window of L requests).  Input buffers are
    // taken in request order (next_take), so that the earliest unsubmitted
    // request never waits for a buffer held by a later one.
    const int L = 64;
    std::vector<double*> inputs(ntot, nullptr);
    std::vector<int> ready(ntot, 0);
    std::atomic<int> consumed{0};
    int next_take = 0;
    std::vector<std::thread> gens;
    for (int gth = 0; gth < ngen; gth++)
        gens.emplace_back([&, gth] {
            for (int k = gth; k < ntot; k += ngen) {
                double* v = nullptr;
                {
                    std::unique_lock<std::mutex> lk(mu);
                    cv.wait(lk, [&] { return k < consumed.load() + L && next_take == k && !free_in[problem[k]].empty(); });
                    v = free_in[problem[k]].back();
                    free_in[problem[k]].pop_back();
                    next_take = k + 1;
                    cv.notify_all();
                }
                const ServeProblem& S = *g_serve[problem[k]];
                Normal r(seed * 1000003ull + (uint64_t)k * 7919ull + 17);
                const double* T = lognormal_table().data();
                for (int64_t i = 0; i < S.nmesh; i++) v[i] = S.median * T[r.next() >> 48];
                std::lock_guard<std::mutex> lk(mu);
                inputs[k] = v;
                ready[k] = 1;
                cv.notify_all();
            }
        });
    std::vector<int64_t> tickets(ntot, 0);
    std::vector<std::pair<double*, double*>> outs(ntot);
    std::vector<int> submitted(ntot, 0);
    double late = 0, late_measured = 0, launch_ms_sum = 0, queue_s_sum = 0, parts_sum[3] = {0, 0, 0};
    // Waiter: collects completions in any order (a long request does not
    // hold back the buffers of shorter ones behind it) and frees buffers.
    std::thread waiter([&] {
        std::vector<int> open;  // submitted, not yet collected
        int next = 0, collected = 0;
        while (collected < ntot) {
            {
                std::unique_lock<std::mutex> lk(mu);
                if (open.empty())
                    cv.wait(lk, [&] { return next < ntot && submitted[next] != 0; });
                while (next < ntot && submitted[next] != 0) open.push_back(next++);
            }
            bool any = false;
            for (size_t i = 0; i < open.size();) {
                const int k = open[i];
                slgpu_request_stats st{};
                st.status = -1;
                if (tickets[k] <= 0)  // rejected at submit
                    st.status = SLGPU_E_ARG;
                else  // oldest open request: a short blocking wait; the rest are polled
                    slgpu_server_wait(srv, tickets[k], i == 0 && !any ? 2e-3 : 0.0, &st);
                if (st.status < 0) {
                    i++;
                    continue;
                }
                any = true;
                latency[k] = st.status == SLGPU_OK ? st.done_s - (arrival[k] + offset) : -1.0;
                done_s[k] = st.done_s;
                device_ms[k] = st.device_ms;
                launch_ms_sum += st.launch_ms;
                for (int j = 0; j < 3; j++) parts_sum[j] += st.launch_parts_ms[j];
                queue_s_sum += st.start_s - st.submit_s;
                double* d = &detail[(size_t)k * kDetail];
                d[0] = st.launch_ms;
                for (int j = 0; j < 3; j++) d[1 + j] = st.launch_parts_ms[j];
                d[4] = (st.start_s - st.submit_s) * 1e3;
                d[5] = std::max(0.0, (st.submit_s - (arrival[k] + offset)) * 1e3);
                if (tickets[k] > 0)
                    slgpu_server_release(srv, tickets[k]);
                open.erase(open.begin() + (long)i);
                collected++;
                std::lock_guard<std::mutex> lk(mu);
                free_out[problem[k]].push_back(outs[k]);
                free_in[problem[k]].push_back(inputs[k]);
                cv.notify_all();
            }
        }
    });
    // Submitter: on the server clock (t_create ~ the server's start).
    for (int k = 0; k < ntot; k++) {
        const ServeProblem& S = *g_serve[problem[k]];
        const double* v = nullptr;
        std::pair<double*, double*> o;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return ready[k] != 0 && !free_out[problem[k]].empty(); });
            v = inputs[k];
            o = free_out[problem[k]].back();
            free_out[problem[k]].pop_back();
        }
        std::this_thread::sleep_until(t_create + std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                                                     std::chrono::duration<double>(arrival[k])));
        const double now = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_create).count();
        if (now > arrival[k] + 1e-3) {
            late += 1;
            if (k >= nwarm)
                late_measured += 1;
        }
        std::vector<slgpu_update> ups;
        for (int gi : S.groups) ups.push_back(slgpu_update{gi, SLGPU_UPDATE_FIELDDATA, 0, 1, v, S.nmesh});
        slgpu_request rq{S.handle, precision, (int32_t)ups.size(), 0, ups.data(), o.first, o.second};
        int64_t tk = 0;
        if (slgpu_server_submit(srv, &rq, &tk) != SLGPU_OK) {
            char buf[512];
            slgpu_last_error(ctx, buf, sizeof(buf));
            g_error = buf;
        }
        std::lock_guard<std::mutex> lk(mu);
        tickets[k] = tk;
        outs[k] = o;
        submitted[k] = 1;
        consumed.store(k + 1);
        cv.notify_all();
    }
    waiter.join();
    for (auto& g : gens) g.join();
    double last = 0, nnz = 0, dev = 0;
    for (int k = nwarm; k < ntot; k++) {
        last = std::max(last, done_s[k]);
        nnz += (double)(g_serve[problem[k]]->nnzA + g_serve[problem[k]]->nnzD);
        dev += device_ms[k];
        latency_out[k - nwarm] = latency[k];
        done_out[k - nwarm] = done_s[k];
        device_out[k - nwarm] = device_ms[k];
        problem_out[k - nwarm] = problem[k];
        if (detail_out != nullptr)
            for (int j = 0; j < kDetail; j++) detail_out[(size_t)(k - nwarm) * kDetail + j] = detail[(size_t)k * kDetail + j];
    }
    summary[0] = last - (arrival[nwarm] + offset);
    summary[1] = nnz;
    summary[2] = dev;
    summary[3] = late_measured;
    summary[4] = launch_ms_sum / ntot;
    summary[5] = queue_s_sum / ntot * 1e3;
    for (int i = 0; i < 3; i++) summary[6 + i] = parts_sum[i] / ntot;
    slgpu_server_destroy(srv);
    for (void* p : pinned) slgpu_host_free(p);
    return g_error.empty() ? 0 : -1;
}

void slz_serve_release(void) { g_serve.clear(); }
}

// ---------------------------------------------------------------- frequency sweep
// The harmonic eddy-current problem assembled at two fundamental frequencies
// through generate()/A(); every term scale and destination multiplier of its
// resident groups is then known as a + b*omega (the harmonic derivation
// factor of dt(), src/harmonic.cpp:110-135, is linear in omega), so a sweep
// sets the scales for each frequency and re-processes on the resident
// pattern instead of re-running generate().
namespace {
struct SweepState {
    std::unique_ptr<Problem> P;
    mat A1, A2;
    int handle = 0;
    std::vector<unsigned char> constrained;
    std::vector<std::vector<double>> ta, tb, da, db;  // per group: a and b of term scales and multipliers
    long long nnzA = 0, nnz = 0;
};
std::unique_ptr<SweepState> g_sweep;

void read_scales(int handle, std::vector<std::vector<double>>& t, std::vector<std::vector<double>>& d)
{
    slgpu_ctx* ctx = slgpu_adapter_ctx();
    int ng = 0;
    slgpu_matrix_group_count(ctx, handle, &ng);
    t.assign(ng, {});
    d.assign(ng, {});
    for (int gi = 0; gi < ng; gi++) {
        slgpu_group_desc g;
        slgpu_matrix_group_desc(ctx, handle, gi, &g);
        t[gi].resize(g.nterms);
        d[gi].resize(g.ndests);
        slgpu_matrix_get_scales(ctx, handle, gi, t[gi].data(), d[gi].data());
    }
}
}  // namespace

extern "C" {

// info4: template handle, ndofs, nnz, groups.
int slz_sweep_prepare(const char* msh, int order, const double* sigmas, double f1, double f2, long long* info4)
{
    g_error.clear();
    try {
        g_sweep.reset();
        auto W = std::make_unique<SweepState>();
        W->P = std::make_unique<Problem>();
        eddy_tet(*W->P, msh, order, sigmas, f1);
        W->P->f.generate();
        W->A1 = W->P->f.A();
        const int h1 = slgpu_adapter::find_matrix_handle(W->A1.getpointer().get());
        std::vector<std::vector<double>> t1, d1, t2, d2;
        read_scales(h1, t1, d1);
        setfundamentalfrequency(f2);
        W->P->f.generate();
        W->A2 = W->P->f.A();
        std::shared_ptr<rawmat> raw = W->A2.getpointer();
        W->handle = slgpu_adapter::find_matrix_handle(raw.get());
        read_scales(W->handle, t2, d2);
        if (t1.size() != t2.size())
            throw std::runtime_error("the two assemblies have different groups");
        const double w1 = 2 * 3.141592653589793 * f1, w2 = 2 * 3.141592653589793 * f2;
        auto fit = [&](const std::vector<std::vector<double>>& s1, const std::vector<std::vector<double>>& s2,
                       std::vector<std::vector<double>>& a, std::vector<std::vector<double>>& b) {
            a = s1;
            b = s1;
            for (size_t g = 0; g < s1.size(); g++) {
                if (s1[g].size() != s2[g].size())
                    throw std::runtime_error("the two assemblies have different terms");
                for (size_t k = 0; k < s1[g].size(); k++) {
                    b[g][k] = (s2[g][k] - s1[g][k]) / (w2 - w1);
                    a[g][k] = s1[g][k] - b[g][k] * w1;
                }
            }
        };
        fit(t1, t2, W->ta, W->tb);
        fit(d1, d2, W->da, W->db);
        std::vector<bool> c = raw->getdofmanager()->isconstrained();
        W->constrained.assign(c.begin(), c.end());
        slgpu_work w;
        slgpu_matrix_work(slgpu_adapter_ctx(), W->handle, &w);
        W->nnzA = raw->countnnz();
        W->nnz = w.nnz;
        info4[0] = W->handle;
        info4[1] = raw->countrows();
        info4[2] = W->nnz;
        info4[3] = (long long)t1.size();
        g_sweep = std::move(W);
    } catch (const std::exception& e) {
        g_error = e.what();
        return 2;
    }
    return 0;
}

// Re-assembles the template at each frequency; device_ms: engine device time
// of the process, host_ms: wall time of the scale update and the process.
int slz_sweep_run(int nfreq, const double* freqs, int precision, double* device_ms, double* host_ms)
{
    if (!g_sweep)
        return 1;
    SweepState& W = *g_sweep;
    slgpu_ctx* ctx = slgpu_adapter_ctx();
    for (int i = 0; i < nfreq; i++) {
        const double t0 = now_s();
        const double w = 2 * 3.141592653589793 * freqs[i];
        for (size_t g = 0; g < W.ta.size(); g++) {
            std::vector<double> ts(W.ta[g].size()), ds(W.da[g].size());
            for (size_t k = 0; k < ts.size(); k++) ts[k] = W.ta[g][k] + W.tb[g][k] * w;
            for (size_t k = 0; k < ds.size(); k++) ds[k] = W.da[g][k] + W.db[g][k] * w;
            if (slgpu_matrix_set_scales(ctx, W.handle, (int)g, ts.data(), ds.data()) != SLGPU_OK)
                return 2;
        }
        slgpu_csr_info info;
        if (slgpu_matrix_process(ctx, W.handle, W.constrained.data(), precision, &info) != SLGPU_OK) {
            char buf[512];
            slgpu_last_error(ctx, buf, sizeof(buf));
            g_error = buf;
            return 3;
        }
        double ms[5];
        slgpu_last_timings(ctx, ms);
        device_ms[i] = ms[4];
        host_ms[i] = (now_s() - t0) * 1e3;
    }
    return 0;
}

// A and D values of the template after the last sweep step (nnzA + nnzD).
long long slz_sweep_values(double* Avals, double* Dvals)
{
    if (!g_sweep)
        return -1;
    if (Avals != nullptr)
        slgpu_matrix_download_values(slgpu_adapter_ctx(), g_sweep->handle, Avals, Dvals);
    return g_sweep->nnzA;
}

void slz_sweep_release(void) { g_sweep.reset(); }
}
#endif
