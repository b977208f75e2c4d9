// Minimal stand-in for the PETSc / SLEPc / CBLAS C APIs that sparselizard's
// sources include.  It exists only so that sparselizard compiles in an image
// without those libraries: the assembly path (Vec*, MatCreateSeqAIJWithArrays,
// Mat assembly/duplicate/AXPY/Mult) is functional, while the solver families
// (KSP, PC, EPS, PEP, ST, DMPlex) raise std::runtime_error when called.
//
// Types follow a real-valued, 32-bit-index PETSc build, which is what
// sparselizard's rawmat expects (int* row pointers handed to
// MatCreateSeqAIJWithArrays, src/formulation/rawmat.cpp:292).
#ifndef SLSHIM_PETSC_H
#define SLSHIM_PETSC_H

#include <cstddef>
#include <cstdio>

typedef int PetscErrorCode;
typedef int PetscInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef int PetscMPIInt;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef int MPI_Comm;

#define PETSC_COMM_SELF 0
#define PETSC_COMM_WORLD 0
#define PETSC_NULLPTR nullptr
#define PETSC_NULL nullptr
#define PETSC_DECIDE (-1)
#define PETSC_DETERMINE (-1)
#define PETSC_DEFAULT (-2)
#define PETSC_VERSION_GE(a, b, c) 1
#define PETSC_VERSION_LT(a, b, c) 0

typedef struct slshim_Vec* Vec;
typedef struct slshim_Mat* Mat;
typedef struct slshim_KSP* KSP;
typedef struct slshim_PC* PC;
typedef struct slshim_IS* IS;
typedef struct slshim_DM* DM;
typedef struct slshim_DMLabel* DMLabel;
typedef struct slshim_Viewer* PetscViewer;
typedef struct slshim_EPS* EPS;
typedef struct slshim_PEP* PEP;
typedef struct slshim_ST* ST;

typedef enum { NOT_SET_VALUES, INSERT_VALUES, ADD_VALUES } InsertMode;
typedef enum { NORM_1 = 0, NORM_2 = 1, NORM_FROBENIUS = 2, NORM_INFINITY = 3 } NormType;
typedef enum { MAT_FLUSH_ASSEMBLY = 1, MAT_FINAL_ASSEMBLY = 0 } MatAssemblyType;
typedef enum { DIFFERENT_NONZERO_PATTERN, SUBSET_NONZERO_PATTERN, SAME_NONZERO_PATTERN, UNKNOWN_NONZERO_PATTERN } MatStructure;
typedef enum { MAT_INITIAL_MATRIX, MAT_REUSE_MATRIX, MAT_IGNORE_MATRIX, MAT_INPLACE_MATRIX } MatReuse;
typedef enum { MAT_DO_NOT_COPY_VALUES, MAT_COPY_VALUES, MAT_SHARE_NONZERO_PATTERN } MatDuplicateOption;
typedef enum { PETSC_COPY_VALUES, PETSC_OWN_POINTER, PETSC_USE_POINTER } PetscCopyMode;
typedef enum { FILE_MODE_UNDEFINED = -1, FILE_MODE_READ = 0, FILE_MODE_WRITE, FILE_MODE_APPEND } PetscFileMode;
typedef enum { PETSC_VIEWER_DEFAULT, PETSC_VIEWER_ASCII_CSV = 100 } PetscViewerFormat;

typedef const char* MatSolverType;
typedef const char* PCType;
typedef const char* KSPType;
typedef const char* EPSType;
typedef const char* PEPType;
typedef const char* STType;

#define PCLU "lu"
#define PCCHOLESKY "cholesky"
#define PCILU "ilu"
#define PCSOR "sor"
#define PCGAMG "gamg"
#define KSPGMRES "gmres"
#define KSPBCGS "bcgs"
#define KSPPREONLY "preonly"
#define EPSKRYLOVSCHUR "krylovschur"
#define PEPTOAR "toar"
#define STSINVERT "sinvert"

typedef enum { EPS_HEP = 1, EPS_GHEP, EPS_NHEP, EPS_GNHEP, EPS_PGNHEP, EPS_GHIEP } EPSProblemType;
typedef enum { EPS_LARGEST_MAGNITUDE = 1, EPS_SMALLEST_MAGNITUDE, EPS_TARGET_MAGNITUDE = 7 } EPSWhich;
typedef enum { PEP_GENERAL = 1, PEP_HERMITIAN, PEP_HYPERBOLIC, PEP_GYROSCOPIC } PEPProblemType;
typedef enum { PEP_LARGEST_MAGNITUDE = 1, PEP_TARGET_MAGNITUDE = 7 } PEPWhich;
typedef enum { PEP_SCALE_NONE, PEP_SCALE_SCALAR, PEP_SCALE_DIAGONAL, PEP_SCALE_BOTH } PEPScale;

PetscViewer slshim_viewer_stdout_self(void);
#define PETSC_VIEWER_STDOUT_SELF slshim_viewer_stdout_self()

// ---- library state
PetscErrorCode PetscInitialized(PetscBool* isinit);
PetscErrorCode SlepcInitialize(int* argc, char*** args, const char file[], const char help[]);
PetscErrorCode PetscFinalize(void);
PetscErrorCode SlepcFinalize(void);

// ---- Vec (functional)
PetscErrorCode VecCreate(MPI_Comm comm, Vec* v);
PetscErrorCode VecSetSizes(Vec v, PetscInt n, PetscInt N);
PetscErrorCode VecSetFromOptions(Vec v);
PetscErrorCode VecSetValues(Vec v, PetscInt ni, const PetscInt ix[], const PetscScalar y[], InsertMode iora);
PetscErrorCode VecSetValue(Vec v, PetscInt i, PetscScalar va, InsertMode mode);
PetscErrorCode VecGetValues(Vec v, PetscInt ni, const PetscInt ix[], PetscScalar y[]);
PetscErrorCode VecAssemblyBegin(Vec v);
PetscErrorCode VecAssemblyEnd(Vec v);
PetscErrorCode VecDestroy(Vec* v);
PetscErrorCode VecDuplicate(Vec v, Vec* newv);
PetscErrorCode VecCopy(Vec x, Vec y);
PetscErrorCode VecSet(Vec x, PetscScalar alpha);
PetscErrorCode VecAXPY(Vec y, PetscScalar alpha, Vec x);
PetscErrorCode VecGetSize(Vec x, PetscInt* size);
PetscErrorCode VecNorm(Vec x, NormType type, PetscReal* val);
PetscErrorCode VecSum(Vec v, PetscScalar* sum);
PetscErrorCode VecView(Vec vec, PetscViewer viewer);
PetscErrorCode VecPermute(Vec x, IS row, PetscBool inv);
PetscErrorCode VecLoad(Vec vec, PetscViewer viewer);

// Direct access used by tools built on this stand-in (not a PETSc name).
PetscScalar* slshim_vec_array(Vec v);

// ---- Mat (CSR borrowed from the caller, as in PETSc's SeqAIJ WithArrays)
PetscErrorCode MatCreateSeqAIJWithArrays(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt i[], PetscInt j[], PetscScalar a[], Mat* mat);
PetscErrorCode MatCreateSeqDense(MPI_Comm comm, PetscInt m, PetscInt n, PetscScalar* data, Mat* A);
PetscErrorCode MatAssemblyBegin(Mat mat, MatAssemblyType type);
PetscErrorCode MatAssemblyEnd(Mat mat, MatAssemblyType type);
PetscErrorCode MatDestroy(Mat* A);
PetscErrorCode MatDuplicate(Mat mat, MatDuplicateOption op, Mat* M);
PetscErrorCode MatAXPY(Mat Y, PetscScalar a, Mat X, MatStructure str);
PetscErrorCode MatMult(Mat mat, Vec x, Vec y);
PetscErrorCode MatMultAdd(Mat mat, Vec v1, Vec v2, Vec v3);
PetscErrorCode MatView(Mat mat, PetscViewer viewer);
PetscErrorCode MatMatMult(Mat A, Mat B, MatReuse scall, PetscReal fill, Mat* C);
PetscErrorCode MatMatSolve(Mat A, Mat B, Mat X);
PetscErrorCode MatPermute(Mat mat, IS row, IS col, Mat* B);
PetscErrorCode MatInvertVariableBlockDiagonal(Mat A, PetscInt nblocks, const PetscInt* bsizes, PetscScalar* diag);

// Read-only CSR access used by tools built on this stand-in (not a PETSc name).
// Returns 0 and fills the pointers for a SeqAIJ matrix, 1 otherwise.
int slshim_mat_csr(Mat m, PetscInt* nrows, PetscInt* ncols, const PetscInt** rows, const PetscInt** cols, const PetscScalar** vals);

// ---- IS
PetscErrorCode ISCreateGeneral(MPI_Comm comm, PetscInt n, const PetscInt idx[], PetscCopyMode mode, IS* is);
PetscErrorCode ISDestroy(IS* is);
PetscErrorCode ISGetSize(IS is, PetscInt* size);
PetscErrorCode ISGetIndices(IS is, const PetscInt* ptr[]);
PetscErrorCode ISRestoreIndices(IS is, const PetscInt* ptr[]);
PetscErrorCode ISSetPermutation(IS is);

// ---- Viewer
PetscErrorCode PetscViewerDestroy(PetscViewer* v);
PetscErrorCode PetscViewerBinaryOpen(MPI_Comm comm, const char name[], PetscFileMode mode, PetscViewer* viewer);
PetscErrorCode PetscViewerASCIIOpen(MPI_Comm comm, const char name[], PetscViewer* lab);
PetscErrorCode PetscViewerPushFormat(PetscViewer viewer, PetscViewerFormat format);

// ---- KSP / PC (solvers are outside this stand-in: calls raise)
PetscErrorCode KSPCreate(MPI_Comm comm, KSP* ksp);
PetscErrorCode KSPDestroy(KSP* ksp);
PetscErrorCode KSPSetOperators(KSP ksp, Mat Amat, Mat Pmat);
PetscErrorCode KSPGetPC(KSP ksp, PC* pc);
PetscErrorCode KSPSetType(KSP ksp, KSPType type);
PetscErrorCode KSPSetFromOptions(KSP ksp);
PetscErrorCode KSPSolve(KSP ksp, Vec b, Vec x);
PetscErrorCode KSPSetDiagonalScale(KSP ksp, PetscBool scale);
PetscErrorCode KSPSetTolerances(KSP ksp, PetscReal rtol, PetscReal abstol, PetscReal dtol, PetscInt maxits);
PetscErrorCode KSPSetInitialGuessNonzero(KSP ksp, PetscBool flg);
PetscErrorCode KSPMonitorSet(KSP ksp, PetscErrorCode (*monitor)(KSP, PetscInt, PetscReal, void*), void* ctx, PetscErrorCode (*monitordestroy)(void**));
PetscErrorCode KSPGetResidualNorm(KSP ksp, PetscReal* rnorm);
PetscErrorCode KSPGetIterationNumber(KSP ksp, PetscInt* its);
PetscErrorCode PCSetType(PC pc, PCType type);
PetscErrorCode PCFactorSetMatSolverType(PC pc, MatSolverType stype);
PetscErrorCode PCSetUp(PC pc);
PetscErrorCode PCFactorGetMatrix(PC pc, Mat* mat);

// ---- DMPlex (PETSc mesh import is outside this stand-in: calls raise)
PetscErrorCode DMPlexCreateFromFile(MPI_Comm comm, const char filename[], PetscBool interpolate, DM* dm);
PetscErrorCode DMPlexCreateFromFile(MPI_Comm comm, const char filename[], const char plexname[], PetscBool interpolate, DM* dm);
PetscErrorCode DMDestroy(DM* dm);
PetscErrorCode DMView(DM dm, PetscViewer v);
PetscErrorCode DMGetDimension(DM dm, PetscInt* dim);
PetscErrorCode DMGetCoordinates(DM dm, Vec* c);
PetscErrorCode DMGetNumLabels(DM dm, PetscInt* numLabels);
PetscErrorCode DMGetLabelByNum(DM dm, PetscInt n, DMLabel* label);
PetscErrorCode DMLabelGetNumValues(DMLabel label, PetscInt* numValues);
PetscErrorCode DMLabelGetValueIS(DMLabel label, IS* values);
PetscErrorCode DMLabelGetStratumIS(DMLabel label, PetscInt value, IS* points);
PetscErrorCode DMPlexGetDepthStratum(DM dm, PetscInt depth, PetscInt* start, PetscInt* end);
PetscErrorCode DMPlexGetTransitiveClosure(DM dm, PetscInt p, PetscBool useCone, PetscInt* numPoints, PetscInt* points[]);
PetscErrorCode DMPlexRestoreTransitiveClosure(DM dm, PetscInt p, PetscBool useCone, PetscInt* numPoints, PetscInt* points[]);

// ---- SLEPc eigen solvers (outside this stand-in: calls raise)
PetscErrorCode EPSCreate(MPI_Comm comm, EPS* eps);
PetscErrorCode EPSDestroy(EPS* eps);
PetscErrorCode EPSSetOperators(EPS eps, Mat A, Mat B);
PetscErrorCode EPSSetProblemType(EPS eps, EPSProblemType type);
PetscErrorCode EPSSetType(EPS eps, EPSType type);
PetscErrorCode EPSSetWhichEigenpairs(EPS eps, EPSWhich which);
PetscErrorCode EPSSetTarget(EPS eps, PetscScalar target);
PetscErrorCode EPSSetDimensions(EPS eps, PetscInt nev, PetscInt ncv, PetscInt mpd);
PetscErrorCode EPSSetTolerances(EPS eps, PetscReal tol, PetscInt maxits);
PetscErrorCode EPSSetFromOptions(EPS eps);
PetscErrorCode EPSGetST(EPS eps, ST* st);
PetscErrorCode EPSSolve(EPS eps);
PetscErrorCode EPSGetConverged(EPS eps, PetscInt* nconv);
PetscErrorCode EPSGetEigenpair(EPS eps, PetscInt i, PetscScalar* eigr, PetscScalar* eigi, Vec Vr, Vec Vi);
PetscErrorCode PEPCreate(MPI_Comm comm, PEP* pep);
PetscErrorCode PEPDestroy(PEP* pep);
PetscErrorCode PEPSetOperators(PEP pep, PetscInt nmat, Mat A[]);
PetscErrorCode PEPSetProblemType(PEP pep, PEPProblemType type);
PetscErrorCode PEPSetType(PEP pep, PEPType type);
PetscErrorCode PEPSetWhichEigenpairs(PEP pep, PEPWhich which);
PetscErrorCode PEPSetTarget(PEP pep, PetscScalar target);
PetscErrorCode PEPSetDimensions(PEP pep, PetscInt nev, PetscInt ncv, PetscInt mpd);
PetscErrorCode PEPSetTolerances(PEP pep, PetscReal tol, PetscInt maxits);
PetscErrorCode PEPSetScale(PEP pep, PEPScale scale, PetscReal alpha, Vec Dl, Vec Dr, PetscInt its, PetscReal lambda);
PetscErrorCode PEPSTOARSetDetectZeros(PEP pep, PetscBool detect);
PetscErrorCode PEPSetFromOptions(PEP pep);
PetscErrorCode PEPSetUp(PEP pep);
PetscErrorCode PEPGetST(PEP pep, ST* st);
PetscErrorCode PEPSolve(PEP pep);
PetscErrorCode PEPGetConverged(PEP pep, PetscInt* nconv);
PetscErrorCode PEPGetEigenpair(PEP pep, PetscInt i, PetscScalar* eigr, PetscScalar* eigi, Vec Vr, Vec Vi);
PetscErrorCode STSetType(ST st, STType type);
PetscErrorCode STGetKSP(ST st, KSP* ksp);

#endif
