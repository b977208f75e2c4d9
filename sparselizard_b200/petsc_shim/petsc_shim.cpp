// Implementation of the PETSc / SLEPc / CBLAS stand-in declared in
// include/slshim_petsc.h and include/cblas.h.  Vectors and borrowed-CSR
// matrices work; every solver entry point raises std::runtime_error so that a
// program reaching a linear or eigen solve fails loudly instead of returning
// garbage.
#include "slshim_petsc.h"
#include "cblas.h"

#include <dlfcn.h>
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

struct slshim_Vec {
    std::vector<double> v;
};

struct slshim_Mat {
    int m = 0, n = 0;
    // SeqAIJ: borrowed (caller-owned) or owned copies.
    const int* rows = nullptr;
    const int* cols = nullptr;
    double* vals = nullptr;
    std::vector<int> own_rows, own_cols;
    std::vector<double> own_vals;
    bool dense = false;
};

struct slshim_IS {
    std::vector<int> idx;
};

struct slshim_Viewer {
    int dummy = 0;
};

static slshim_Viewer g_stdout_viewer;
static bool g_initialized = false;

[[noreturn]] static void unsupported(const char* name)
{
    throw std::runtime_error(std::string("PETSc stand-in: '") + name +
                             "' is a solver/IO entry point that this build does not provide");
}

PetscViewer slshim_viewer_stdout_self(void) { return &g_stdout_viewer; }

PetscErrorCode PetscInitialized(PetscBool* isinit)
{
    *isinit = g_initialized ? PETSC_TRUE : PETSC_FALSE;
    return 0;
}
PetscErrorCode SlepcInitialize(int*, char***, const char*, const char*)
{
    g_initialized = true;
    return 0;
}
PetscErrorCode PetscFinalize(void) { g_initialized = false; return 0; }
PetscErrorCode SlepcFinalize(void) { g_initialized = false; return 0; }

// ------------------------------------------------------------------ Vec
PetscErrorCode VecCreate(MPI_Comm, Vec* v) { *v = new slshim_Vec(); return 0; }
PetscErrorCode VecSetSizes(Vec v, PetscInt n, PetscInt N)
{
    v->v.assign(N >= 0 ? N : n, 0.0);
    return 0;
}
PetscErrorCode VecSetFromOptions(Vec) { return 0; }
PetscErrorCode VecSetValues(Vec v, PetscInt ni, const PetscInt ix[], const PetscScalar y[], InsertMode iora)
{
    for (PetscInt i = 0; i < ni; i++) {
        if (ix[i] < 0)
            continue;
        if (iora == ADD_VALUES)
            v->v[ix[i]] += y[i];
        else
            v->v[ix[i]] = y[i];
    }
    return 0;
}
PetscErrorCode VecSetValue(Vec v, PetscInt i, PetscScalar va, InsertMode mode)
{
    return VecSetValues(v, 1, &i, &va, mode);
}
PetscErrorCode VecGetValues(Vec v, PetscInt ni, const PetscInt ix[], PetscScalar y[])
{
    for (PetscInt i = 0; i < ni; i++)
        y[i] = v->v[ix[i]];
    return 0;
}
PetscErrorCode VecAssemblyBegin(Vec) { return 0; }
PetscErrorCode VecAssemblyEnd(Vec) { return 0; }
PetscErrorCode VecDestroy(Vec* v)
{
    delete *v;
    *v = nullptr;
    return 0;
}
PetscErrorCode VecDuplicate(Vec v, Vec* newv)
{
    *newv = new slshim_Vec();
    (*newv)->v.assign(v->v.size(), 0.0);
    return 0;
}
PetscErrorCode VecCopy(Vec x, Vec y) { y->v = x->v; return 0; }
PetscErrorCode VecSet(Vec x, PetscScalar alpha)
{
    for (auto& e : x->v) e = alpha;
    return 0;
}
PetscErrorCode VecAXPY(Vec y, PetscScalar alpha, Vec x)
{
    for (size_t i = 0; i < y->v.size(); i++) y->v[i] += alpha * x->v[i];
    return 0;
}
PetscErrorCode VecGetSize(Vec x, PetscInt* size) { *size = (PetscInt)x->v.size(); return 0; }
PetscErrorCode VecNorm(Vec x, NormType type, PetscReal* val)
{
    double r = 0;
    for (double e : x->v) {
        if (type == NORM_1) r += std::fabs(e);
        else if (type == NORM_INFINITY) r = std::fmax(r, std::fabs(e));
        else r += e * e;
    }
    *val = (type == NORM_2 || type == NORM_FROBENIUS) ? std::sqrt(r) : r;
    return 0;
}
PetscErrorCode VecSum(Vec v, PetscScalar* sum)
{
    double s = 0;
    for (double e : v->v) s += e;
    *sum = s;
    return 0;
}
PetscErrorCode VecView(Vec vec, PetscViewer)
{
    for (size_t i = 0; i < vec->v.size(); i++) std::cout << vec->v[i] << "\n";
    return 0;
}
PetscErrorCode VecPermute(Vec x, IS row, PetscBool inv)
{
    std::vector<double> out(x->v.size());
    for (size_t i = 0; i < out.size(); i++) {
        if (inv) out[row->idx[i]] = x->v[i];
        else out[i] = x->v[row->idx[i]];
    }
    x->v = out;
    return 0;
}
PetscErrorCode VecLoad(Vec, PetscViewer) { unsupported("VecLoad"); }
PetscScalar* slshim_vec_array(Vec v) { return v->v.data(); }

// ------------------------------------------------------------------ Mat
PetscErrorCode MatCreateSeqAIJWithArrays(MPI_Comm, PetscInt m, PetscInt n, PetscInt i[], PetscInt j[], PetscScalar a[], Mat* mat)
{
    Mat M = new slshim_Mat();
    M->m = m;
    M->n = n;
    M->rows = i;
    M->cols = j;
    M->vals = a;
    *mat = M;
    return 0;
}
PetscErrorCode MatCreateSeqDense(MPI_Comm, PetscInt m, PetscInt n, PetscScalar* data, Mat* A)
{
    Mat M = new slshim_Mat();
    M->m = m;
    M->n = n;
    M->vals = data;
    M->dense = true;
    *A = M;
    return 0;
}
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatDestroy(Mat* A)
{
    delete *A;
    *A = nullptr;
    return 0;
}
PetscErrorCode MatDuplicate(Mat mat, MatDuplicateOption op, Mat* out)
{
    if (mat->dense)
        unsupported("MatDuplicate(dense)");
    Mat M = new slshim_Mat();
    M->m = mat->m;
    M->n = mat->n;
    int nnz = mat->rows[mat->m];
    M->own_rows.assign(mat->rows, mat->rows + mat->m + 1);
    M->own_cols.assign(mat->cols, mat->cols + nnz);
    if (op == MAT_COPY_VALUES)
        M->own_vals.assign(mat->vals, mat->vals + nnz);
    else
        M->own_vals.assign(nnz, 0.0);
    M->rows = M->own_rows.data();
    M->cols = M->own_cols.data();
    M->vals = M->own_vals.data();
    *out = M;
    return 0;
}
PetscErrorCode MatAXPY(Mat Y, PetscScalar a, Mat X, MatStructure)
{
    if (Y->dense || X->dense || Y->m != X->m)
        unsupported("MatAXPY(shape)");
    int nnz = Y->rows[Y->m];
    bool same = X->rows[X->m] == nnz && std::memcmp(X->rows, Y->rows, sizeof(int) * (Y->m + 1)) == 0 &&
                std::memcmp(X->cols, Y->cols, sizeof(int) * nnz) == 0;
    if (!same)
        unsupported("MatAXPY(different pattern)");
    for (int k = 0; k < nnz; k++)
        Y->vals[k] += a * X->vals[k];
    return 0;
}
PetscErrorCode MatMult(Mat A, Vec x, Vec y)
{
    if (A->dense)
        unsupported("MatMult(dense)");
    y->v.assign(A->m, 0.0);
    for (int r = 0; r < A->m; r++) {
        double s = 0;
        for (int k = A->rows[r]; k < A->rows[r + 1]; k++)
            s += A->vals[k] * x->v[A->cols[k]];
        y->v[r] = s;
    }
    return 0;
}
PetscErrorCode MatMultAdd(Mat A, Vec v1, Vec v2, Vec v3)
{
    std::vector<double> base = v2->v;
    MatMult(A, v1, v3);
    for (size_t i = 0; i < base.size(); i++) v3->v[i] += base[i];
    return 0;
}
PetscErrorCode MatView(Mat mat, PetscViewer)
{
    if (mat->dense)
        return 0;
    for (int r = 0; r < mat->m; r++) {
        std::cout << "row " << r << ":";
        for (int k = mat->rows[r]; k < mat->rows[r + 1]; k++)
            std::cout << " (" << mat->cols[k] << ", " << mat->vals[k] << ")";
        std::cout << "\n";
    }
    return 0;
}
PetscErrorCode MatMatMult(Mat, Mat, MatReuse, PetscReal, Mat*) { unsupported("MatMatMult"); }
PetscErrorCode MatMatSolve(Mat, Mat, Mat) { unsupported("MatMatSolve"); }
// B(i, j) = A(rperm[i], cperm[j]) (each new row i is old row rperm[i], old
// column c becomes column cinv[c]); rows of B sorted by column.
PetscErrorCode MatPermute(Mat A, IS rperm, IS cperm, Mat* out)
{
    if (A->dense)
        unsupported("MatPermute(dense)");
    if ((PetscInt)rperm->idx.size() != A->m || (PetscInt)cperm->idx.size() != A->n)
        unsupported("MatPermute(permutation size)");
    std::vector<int> cinv(A->n);
    for (int j = 0; j < A->n; j++) cinv[cperm->idx[j]] = j;
    Mat M = new slshim_Mat();
    M->m = A->m;
    M->n = A->n;
    M->own_rows.assign(A->m + 1, 0);
    for (int i = 0; i < A->m; i++) {
        const int r = rperm->idx[i];
        M->own_rows[i + 1] = M->own_rows[i] + (A->rows[r + 1] - A->rows[r]);
    }
    M->own_cols.resize(M->own_rows[A->m]);
    M->own_vals.resize(M->own_rows[A->m]);
    std::vector<std::pair<int, double>> row;
    for (int i = 0; i < A->m; i++) {
        const int r = rperm->idx[i];
        row.clear();
        for (int k = A->rows[r]; k < A->rows[r + 1]; k++) row.emplace_back(cinv[A->cols[k]], A->vals[k]);
        std::sort(row.begin(), row.end(), [](const std::pair<int, double>& a, const std::pair<int, double>& b) { return a.first < b.first; });
        for (size_t k = 0; k < row.size(); k++) {
            M->own_cols[M->own_rows[i] + k] = row[k].first;
            M->own_vals[M->own_rows[i] + k] = row[k].second;
        }
    }
    M->rows = M->own_rows.data();
    M->cols = M->own_cols.data();
    M->vals = M->own_vals.data();
    *out = M;
    return 0;
}

// Inverses of the consecutive diagonal blocks of sizes bsizes[0..nb), each
// stored column-major one after the other (the layout
// densemat::blockdiagonaltimesvector reads, src/densemat.cpp:788-818).
// Gauss-Jordan elimination with partial pivoting.
PetscErrorCode MatInvertVariableBlockDiagonal(Mat A, PetscInt nb, const PetscInt* bsizes, PetscScalar* diag)
{
    if (A->dense)
        unsupported("MatInvertVariableBlockDiagonal(dense)");
    long long r0 = 0, off = 0;
    std::vector<double> a, inv;
    for (PetscInt b = 0; b < nb; b++) {
        const int n = bsizes[b];
        a.assign((size_t)n * n, 0.0);  // row-major block
        for (int i = 0; i < n; i++) {
            const long long r = r0 + i;
            for (int k = A->rows[r]; k < A->rows[r + 1]; k++) {
                const long long c = A->cols[k];
                if (c >= r0 && c < r0 + n)
                    a[(size_t)i * n + (c - r0)] = A->vals[k];
            }
        }
        inv.assign((size_t)n * n, 0.0);
        for (int i = 0; i < n; i++) inv[(size_t)i * n + i] = 1.0;
        for (int col = 0; col < n; col++) {
            int piv = col;
            for (int i = col + 1; i < n; i++)
                if (std::fabs(a[(size_t)i * n + col]) > std::fabs(a[(size_t)piv * n + col]))
                    piv = i;
            if (a[(size_t)piv * n + col] == 0.0)
                unsupported("MatInvertVariableBlockDiagonal(singular block)");
            if (piv != col)
                for (int k = 0; k < n; k++) {
                    std::swap(a[(size_t)piv * n + k], a[(size_t)col * n + k]);
                    std::swap(inv[(size_t)piv * n + k], inv[(size_t)col * n + k]);
                }
            const double d = a[(size_t)col * n + col];
            for (int k = 0; k < n; k++) {
                a[(size_t)col * n + k] /= d;
                inv[(size_t)col * n + k] /= d;
            }
            for (int i = 0; i < n; i++) {
                if (i == col)
                    continue;
                const double f = a[(size_t)i * n + col];
                if (f == 0.0)
                    continue;
                for (int k = 0; k < n; k++) {
                    a[(size_t)i * n + k] -= f * a[(size_t)col * n + k];
                    inv[(size_t)i * n + k] -= f * inv[(size_t)col * n + k];
                }
            }
        }
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) diag[off + (size_t)j * n + i] = inv[(size_t)i * n + j];
        off += (long long)n * n;
        r0 += n;
    }
    return 0;
}

int slshim_mat_csr(Mat m, PetscInt* nrows, PetscInt* ncols, const PetscInt** rows, const PetscInt** cols, const PetscScalar** vals)
{
    if (m == nullptr || m->dense)
        return 1;
    *nrows = m->m;
    *ncols = m->n;
    *rows = m->rows;
    *cols = m->cols;
    *vals = m->vals;
    return 0;
}

// ------------------------------------------------------------------ IS
PetscErrorCode ISCreateGeneral(MPI_Comm, PetscInt n, const PetscInt idx[], PetscCopyMode, IS* is)
{
    *is = new slshim_IS();
    (*is)->idx.assign(idx, idx + n);
    return 0;
}
PetscErrorCode ISDestroy(IS* is)
{
    delete *is;
    *is = nullptr;
    return 0;
}
PetscErrorCode ISGetSize(IS is, PetscInt* size) { *size = (PetscInt)is->idx.size(); return 0; }
PetscErrorCode ISGetIndices(IS is, const PetscInt* ptr[]) { *ptr = is->idx.data(); return 0; }
PetscErrorCode ISRestoreIndices(IS, const PetscInt* ptr[]) { *ptr = nullptr; return 0; }
PetscErrorCode ISSetPermutation(IS) { return 0; }

// ------------------------------------------------------------------ Viewer
PetscErrorCode PetscViewerDestroy(PetscViewer* v)
{
    if (*v != &g_stdout_viewer)
        delete *v;
    *v = nullptr;
    return 0;
}
PetscErrorCode PetscViewerBinaryOpen(MPI_Comm, const char[], PetscFileMode, PetscViewer*) { unsupported("PetscViewerBinaryOpen"); }
PetscErrorCode PetscViewerASCIIOpen(MPI_Comm, const char[], PetscViewer*) { unsupported("PetscViewerASCIIOpen"); }
PetscErrorCode PetscViewerPushFormat(PetscViewer, PetscViewerFormat) { unsupported("PetscViewerPushFormat"); }

// ------------------------------------------------------------------ KSP / PC
PetscErrorCode KSPCreate(MPI_Comm, KSP*) { unsupported("KSPCreate"); }
PetscErrorCode KSPDestroy(KSP* ksp) { *ksp = nullptr; return 0; }
PetscErrorCode KSPSetOperators(KSP, Mat, Mat) { unsupported("KSPSetOperators"); }
PetscErrorCode KSPGetPC(KSP, PC*) { unsupported("KSPGetPC"); }
PetscErrorCode KSPSetType(KSP, KSPType) { unsupported("KSPSetType"); }
PetscErrorCode KSPSetFromOptions(KSP) { unsupported("KSPSetFromOptions"); }
PetscErrorCode KSPSolve(KSP, Vec, Vec) { unsupported("KSPSolve"); }
PetscErrorCode KSPSetDiagonalScale(KSP, PetscBool) { unsupported("KSPSetDiagonalScale"); }
PetscErrorCode KSPSetTolerances(KSP, PetscReal, PetscReal, PetscReal, PetscInt) { unsupported("KSPSetTolerances"); }
PetscErrorCode KSPSetInitialGuessNonzero(KSP, PetscBool) { unsupported("KSPSetInitialGuessNonzero"); }
PetscErrorCode KSPMonitorSet(KSP, PetscErrorCode (*)(KSP, PetscInt, PetscReal, void*), void*, PetscErrorCode (*)(void**)) { unsupported("KSPMonitorSet"); }
PetscErrorCode KSPGetResidualNorm(KSP, PetscReal*) { unsupported("KSPGetResidualNorm"); }
PetscErrorCode KSPGetIterationNumber(KSP, PetscInt*) { unsupported("KSPGetIterationNumber"); }
PetscErrorCode PCSetType(PC, PCType) { unsupported("PCSetType"); }
PetscErrorCode PCFactorSetMatSolverType(PC, MatSolverType) { unsupported("PCFactorSetMatSolverType"); }
PetscErrorCode PCSetUp(PC) { unsupported("PCSetUp"); }
PetscErrorCode PCFactorGetMatrix(PC, Mat*) { unsupported("PCFactorGetMatrix"); }

// ------------------------------------------------------------------ DMPlex
PetscErrorCode DMPlexCreateFromFile(MPI_Comm, const char[], PetscBool, DM*) { unsupported("DMPlexCreateFromFile"); }
PetscErrorCode DMPlexCreateFromFile(MPI_Comm, const char[], const char[], PetscBool, DM*) { unsupported("DMPlexCreateFromFile"); }
PetscErrorCode DMDestroy(DM* dm) { *dm = nullptr; return 0; }
PetscErrorCode DMView(DM, PetscViewer) { unsupported("DMView"); }
PetscErrorCode DMGetDimension(DM, PetscInt*) { unsupported("DMGetDimension"); }
PetscErrorCode DMGetCoordinates(DM, Vec*) { unsupported("DMGetCoordinates"); }
PetscErrorCode DMGetNumLabels(DM, PetscInt*) { unsupported("DMGetNumLabels"); }
PetscErrorCode DMGetLabelByNum(DM, PetscInt, DMLabel*) { unsupported("DMGetLabelByNum"); }
PetscErrorCode DMLabelGetNumValues(DMLabel, PetscInt*) { unsupported("DMLabelGetNumValues"); }
PetscErrorCode DMLabelGetValueIS(DMLabel, IS*) { unsupported("DMLabelGetValueIS"); }
PetscErrorCode DMLabelGetStratumIS(DMLabel, PetscInt, IS*) { unsupported("DMLabelGetStratumIS"); }
PetscErrorCode DMPlexGetDepthStratum(DM, PetscInt, PetscInt*, PetscInt*) { unsupported("DMPlexGetDepthStratum"); }
PetscErrorCode DMPlexGetTransitiveClosure(DM, PetscInt, PetscBool, PetscInt*, PetscInt*[]) { unsupported("DMPlexGetTransitiveClosure"); }
PetscErrorCode DMPlexRestoreTransitiveClosure(DM, PetscInt, PetscBool, PetscInt*, PetscInt*[]) { unsupported("DMPlexRestoreTransitiveClosure"); }

// ------------------------------------------------------------------ SLEPc
PetscErrorCode EPSCreate(MPI_Comm, EPS*) { unsupported("EPSCreate"); }
PetscErrorCode EPSDestroy(EPS* eps) { *eps = nullptr; return 0; }
PetscErrorCode EPSSetOperators(EPS, Mat, Mat) { unsupported("EPSSetOperators"); }
PetscErrorCode EPSSetProblemType(EPS, EPSProblemType) { unsupported("EPSSetProblemType"); }
PetscErrorCode EPSSetType(EPS, EPSType) { unsupported("EPSSetType"); }
PetscErrorCode EPSSetWhichEigenpairs(EPS, EPSWhich) { unsupported("EPSSetWhichEigenpairs"); }
PetscErrorCode EPSSetTarget(EPS, PetscScalar) { unsupported("EPSSetTarget"); }
PetscErrorCode EPSSetDimensions(EPS, PetscInt, PetscInt, PetscInt) { unsupported("EPSSetDimensions"); }
PetscErrorCode EPSSetTolerances(EPS, PetscReal, PetscInt) { unsupported("EPSSetTolerances"); }
PetscErrorCode EPSSetFromOptions(EPS) { unsupported("EPSSetFromOptions"); }
PetscErrorCode EPSGetST(EPS, ST*) { unsupported("EPSGetST"); }
PetscErrorCode EPSSolve(EPS) { unsupported("EPSSolve"); }
PetscErrorCode EPSGetConverged(EPS, PetscInt*) { unsupported("EPSGetConverged"); }
PetscErrorCode EPSGetEigenpair(EPS, PetscInt, PetscScalar*, PetscScalar*, Vec, Vec) { unsupported("EPSGetEigenpair"); }
PetscErrorCode PEPCreate(MPI_Comm, PEP*) { unsupported("PEPCreate"); }
PetscErrorCode PEPDestroy(PEP* pep) { *pep = nullptr; return 0; }
PetscErrorCode PEPSetOperators(PEP, PetscInt, Mat[]) { unsupported("PEPSetOperators"); }
PetscErrorCode PEPSetProblemType(PEP, PEPProblemType) { unsupported("PEPSetProblemType"); }
PetscErrorCode PEPSetType(PEP, PEPType) { unsupported("PEPSetType"); }
PetscErrorCode PEPSetWhichEigenpairs(PEP, PEPWhich) { unsupported("PEPSetWhichEigenpairs"); }
PetscErrorCode PEPSetTarget(PEP, PetscScalar) { unsupported("PEPSetTarget"); }
PetscErrorCode PEPSetDimensions(PEP, PetscInt, PetscInt, PetscInt) { unsupported("PEPSetDimensions"); }
PetscErrorCode PEPSetTolerances(PEP, PetscReal, PetscInt) { unsupported("PEPSetTolerances"); }
PetscErrorCode PEPSetScale(PEP, PEPScale, PetscReal, Vec, Vec, PetscInt, PetscReal) { unsupported("PEPSetScale"); }
PetscErrorCode PEPSTOARSetDetectZeros(PEP, PetscBool) { unsupported("PEPSTOARSetDetectZeros"); }
PetscErrorCode PEPSetFromOptions(PEP) { unsupported("PEPSetFromOptions"); }
PetscErrorCode PEPSetUp(PEP) { unsupported("PEPSetUp"); }
PetscErrorCode PEPGetST(PEP, ST*) { unsupported("PEPGetST"); }
PetscErrorCode PEPSolve(PEP) { unsupported("PEPSolve"); }
PetscErrorCode PEPGetConverged(PEP, PetscInt*) { unsupported("PEPGetConverged"); }
PetscErrorCode PEPGetEigenpair(PEP, PetscInt, PetscScalar*, PetscScalar*, Vec, Vec) { unsupported("PEPGetEigenpair"); }
PetscErrorCode STSetType(ST, STType) { unsupported("STSetType"); }
PetscErrorCode STGetKSP(ST, KSP*) { unsupported("STGetKSP"); }

// ------------------------------------------------------------------ CBLAS
typedef void (*dgemm_fn)(int, int, int, int, int, int, double, const double*, int, const double*, int, double, double*, int);

// The BLAS behind cblas_dgemm: the library named by SLSHIM_OPENBLAS (an
// OpenBLAS build exporting scipy_cblas_dgemm, e.g. the one bundled with scipy)
// when it loads, else the plain loop below.  slshim_dgemm_name() reports which.
static std::string g_dgemm_name = "loop (no BLAS library loaded)";

static dgemm_fn load_openblas_dgemm(void)
{
    const char* path = std::getenv("SLSHIM_OPENBLAS");
    if (path == nullptr || path[0] == 0)
        return nullptr;
    void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (h == nullptr)
        return nullptr;
    void* f = dlsym(h, "scipy_cblas_dgemm");
    if (f == nullptr)
        return nullptr;
    g_dgemm_name = std::string("OpenBLAS scipy_cblas_dgemm from ") + path;
    return (dgemm_fn)f;
}

static dgemm_fn dgemm_impl(void)
{
    static std::once_flag once;
    static dgemm_fn fn = nullptr;
    std::call_once(once, [] { fn = load_openblas_dgemm(); });
    return fn;
}

extern "C" const char* slshim_dgemm_name(void)
{
    dgemm_impl();
    return g_dgemm_name.c_str();
}

void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE transa, enum CBLAS_TRANSPOSE transb,
                 int m, int n, int k, double alpha, const double* a, int lda, const double* b, int ldb,
                 double beta, double* c, int ldc)
{
    dgemm_fn fn = dgemm_impl();
    if (fn != nullptr) {
        fn((int)order, (int)transa, (int)transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
        return;
    }
    if (order != CblasRowMajor)
        unsupported("cblas_dgemm(column-major)");
    // Plain row-major triple loop when no BLAS library could be loaded.
    for (int i = 0; i < m; i++)
        for (int j = 0; j < n; j++) {
            double s = 0;
            for (int p = 0; p < k; p++) {
                double av = (transa == CblasNoTrans) ? a[(long)i * lda + p] : a[(long)p * lda + i];
                double bv = (transb == CblasNoTrans) ? b[(long)p * ldb + j] : b[(long)j * ldb + p];
                s += av * bv;
            }
            c[(long)i * ldc + j] = alpha * s + (beta == 0 ? 0 : beta * c[(long)i * ldc + j]);
        }
}
