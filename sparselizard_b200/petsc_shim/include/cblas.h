// Stand-in CBLAS header for sparselizard's densemat::multiply
// (src/densemat.cpp:264-278).  cblas_dgemm forwards to the OpenBLAS build that
// ships with SciPy (symbol scipy_cblas_dgemm), loaded at run time.
#ifndef SLSHIM_CBLAS_H
#define SLSHIM_CBLAS_H

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE transa, enum CBLAS_TRANSPOSE transb,
                 int m, int n, int k, double alpha, const double* a, int lda, const double* b, int ldb,
                 double beta, double* c, int ldc);

#endif
