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

// Poisson on quadrangles: integral(vol, -grad(dof(v))*grad(tf(v)), -2) +
// integral(vol, 1*tf(v), -2), v = 0 on the boundary.
void poisson_quad(const char* msh, int order, int reps, double* times)
{
    mesh m(msh, 0);
    field v("h1");
    v.setorder(VOL, order);
    v.setconstraint(BOUNDARY);
    formulation f;
    f += integral(VOL, -grad(dof(v)) * grad(tf(v)), -2);
    f += integral(VOL, 1 * tf(v), -2);
    run_reps(f, reps, times);
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
void elasticity_hex(const char* msh, int order, int delta, int reps, double* times)
{
    mesh m(msh, 0);
    field u("h1xyz"), E("one");
    u.setorder(VOL, order);
    u.setconstraint(CLAMP);
    Normal rng(12345);
    std::vector<double> evals(1 << 22);
    for (double& e : evals) e = 150e9 * std::exp(0.3 * rng.draw());
    set_per_element(E, VOL, evals);
    formulation f;
    f += integral(VOL, predefinedelasticity(dof(u), tf(u), E, 0.3), delta);
    run_reps(f, reps, times);
}

// p-adaptive scalar Helmholtz on tets: region ORDER_REGION_BASE+p holds the
// order-p elements (p = 1..5); orders are set in descending order.
void helmholtz_tet(const char* msh, int reps, double* times)
{
    mesh m(msh, 0);
    int vol = selectunion({ORDER_REGION_BASE + 1, ORDER_REGION_BASE + 2, ORDER_REGION_BASE + 3, ORDER_REGION_BASE + 4, ORDER_REGION_BASE + 5});
    field p("h1");
    for (int ord = 5; ord >= 1; ord--)
        p.setorder(ORDER_REGION_BASE + ord, ord);
    formulation f;
    f += integral(vol, grad(dof(p)) * grad(tf(p)) - 400.0 * dof(p) * tf(p));
    run_reps(f, reps, times);
}

// Harmonic eddy currents on tets, hcurl order 2 with harmonics {2,3}:
// integral(vol, curl(dof(a))*curl(tf(a))/mu + sigma*dt(dof(a))*tf(a)),
// sigma per material region, at fundamental frequency `freq`.
void eddy_tet(const char* msh, int order, const double* sigmas, double freq, int reps, double* times)
{
    mesh m(msh, 0);
    int vol = selectunion({MATERIAL_REGION_BASE, MATERIAL_REGION_BASE + 1, MATERIAL_REGION_BASE + 2, MATERIAL_REGION_BASE + 3});
    setfundamentalfrequency(freq);
    field a("hcurl", {2, 3});
    a.setorder(vol, order);
    parameter sigma;
    for (int r = 0; r < 4; r++)
        sigma.setvalue(MATERIAL_REGION_BASE + r, sigmas[r]);
    double mu = 4.0 * 3.141592653589793 * 1e-7;
    formulation f;
    f += integral(vol, curl(dof(a)) * curl(tf(a)) / mu + sigma * dt(dof(a)) * tf(a));
    run_reps(f, reps, times);
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
        switch (workload) {
        case 1:
            poisson_quad(msh, (int)params[0], reps, times);
            break;
        case 2:
            elasticity_hex(msh, (int)params[0], (int)params[1], reps, times);
            break;
        case 3:
            helmholtz_tet(msh, reps, times);
            break;
        case 4:
            eddy_tet(msh, (int)params[0], params + 2, params[1], reps, times);
            break;
        default:
            g_error = "unknown workload";
            return 1;
        }
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
