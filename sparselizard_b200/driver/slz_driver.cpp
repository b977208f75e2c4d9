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

std::unique_ptr<Problem> build(int workload, const char* msh, const double* params)
{
    auto P = std::make_unique<Problem>();
    switch (workload) {
    case 1: poisson_quad(*P, msh, (int)params[0]); break;
    case 2: elasticity_hex(*P, msh, (int)params[0], (int)params[1]); break;
    case 3: helmholtz_tet(*P, msh); break;
    case 4: eddy_tet(*P, msh, (int)params[0], params + 2, params[1]); break;
    default: throw std::runtime_error("unknown workload");
    }
    return P;
}

} // namespace

extern "C" {

// Workload ids: 1 Poisson quads (param0 = order), 2 elasticity hexes
// (param0 = order, param1 = integration delta), 3 p-adaptive Helmholtz tets,
// 4 harmonic eddy current tets (param0 = order, param1 = frequency,
// param2..5 = sigma per material region).
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
#endif
