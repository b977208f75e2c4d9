/*
 * slref -- CPU restatement of sparselizard's assembly hot path, used only by
 * the tests and the CPU baseline as the checker for the GPU engine.
 *
 * Input is the engine's own lowered description (include/slgpu.h): element
 * groups with Gauss rules, form-function tables, a coefficient program and
 * dof/tf addresses, plus raw COO fragments.  Output is what
 * rawmat::process hands to PETSc.  Every step follows the reference:
 *   element matrices  src/formulation/contribution.cpp:144-210,
 *                     src/densemat.cpp:228-310 (multiply), :608-636
 *   Jacobian          src/field/jacobian.cpp:248-349, :396-504
 *   COO -> A/D CSR    src/formulation/rawmat.cpp:67-299
 *   right-hand side   src/formulation/contribution.cpp:293-300,
 *                     src/formulation/rawvec.cpp:216-254
 * This is test infrastructure, not part of the product.
 */
#ifndef SLREF_H
#define SLREF_H

#include "../include/slgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t ntr, ndr, nr;
    int64_t nc;
    const int32_t* rows;
    const int32_t* cols;
    const double* vals;
} slref_fragment;

typedef struct {
    int64_t nA, nD, nnzA, nnzD;
    int32_t *Arows, *Acols, *Drows, *Dcols; /* malloc'd; release with slref_free */
    double *Avals, *Dvals;
} slref_csr;

/* Element matrices of one group in the reference layout
 * K[((d*ntf + i)*ndof + j)*nelem + e] (d = destination, multiplier applied).
 * `xyz` [3*nnodes] and `conn` [nelem_type*ncurvednodes] are the mesh arrays
 * given to slgpu_mesh_set_nodes / slgpu_mesh_set_elements. */
int slref_element_matrices(const slgpu_group* g, const double* xyz, const int32_t* conn, double* K);

/* Full rawmat::process on the COO of the groups (in order, destinations in
 * order, entries (i*ndof+j)-major / element-minor) followed by the fragments. */
int slref_matrix(const slgpu_group* groups, int ngroups, const double* xyz, const int32_t* const* conn_per_group,
                 const slref_fragment* frags, int nfrags, int64_t ndofs, const uint8_t* isconstrained, slref_csr* out);

/* b[addr] += -(element vectors) of a right-hand-side group. */
int slref_rhs(const slgpu_group* g, const double* xyz, const int32_t* conn, int64_t ndofs, double* b);

void slref_free(slref_csr* c);

/* on != 0: the functions above return sum |terms| instead of sum terms (every
 * product, factor and summand taken in absolute value), the scale against
 * which rounding differences between two correct summation orders are
 * judged. */
void slref_set_absmode(int on);

#ifdef __cplusplus
}
#endif

#endif
