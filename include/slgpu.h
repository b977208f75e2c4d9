/*
 * slgpu.h -- C ABI of the B200 weak-form assembly engine.
 *
 * The engine replaces the compute inside sparselizard's
 *   contribution::generate  (src/formulation/contribution.cpp:20-308)
 *   rawmat::process         (src/formulation/rawmat.cpp:127-299)
 * Everything crossing this boundary is plain C: pointers, sizes and int status
 * codes.  Host arrays passed in are copied (or uploaded) before the call
 * returns; outputs are written to caller-owned host buffers, following
 * PETSc's MatCreateSeqAIJWithArrays ownership model that rawmat relies on
 * (src/formulation/rawmat.cpp:292-296).
 *
 * Error convention: every entry point returns SLGPU_OK (0) or a positive
 * SLGPU_E_* code; slgpu_last_error() gives the message.  sparselizard's
 * adapter turns a non-zero status into logs::error(), i.e. a thrown
 * std::runtime_error (src/logs.cpp:9-12).
 *
 * One context drives one device.  Calls on a context must be serialised by
 * the caller (sparselizard's assembly is single-threaded host code).
 */
#ifndef SLGPU_H
#define SLGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct slgpu_ctx slgpu_ctx;

enum {
    SLGPU_OK = 0,
    SLGPU_E_ARG = 1,          /* invalid argument or inconsistent sizes */
    SLGPU_E_CUDA = 2,         /* a CUDA call failed */
    SLGPU_E_UNSUPPORTED = 3,  /* input outside what the engine implements */
    SLGPU_E_BUDGET = 4,       /* request exceeds the context's HBM budget */
    SLGPU_E_STATE = 5,        /* call not valid in the current state */
    SLGPU_E_NODEVICE = 6,     /* no usable CUDA device / extension */
    SLGPU_E_TIMEOUT = 7       /* a bounded device wait gave up */
};

/* Context flags. */
#define SLGPU_CTX_RECORD_ONLY 1u /* no device: groups are recorded for inspection, never executed */

/* Contraction precision (slgpu_matrix_process / slgpu_rhs_assemble). */
enum {
    SLGPU_PREC_FP64 = 0,  /* plain FP64 */
    SLGPU_PREC_SPLIT = 1, /* FP64 operands split into 7 INT8 slices on the tensor cores (tcgen05 kind::i8), exact INT32
                             accumulation, FP64 recombination; <= 1e-10 relative per element matrix */
    SLGPU_PREC_FP32 = 2   /* same with 5 slices: FP32-level tier, <= 1e-6 */
};

/*
 * Context.  hbm_budget bounds the device memory the context may hold
 * (0 = 150 GB).  Replaces nothing in the reference: sparselizard has no
 * device; the adapter creates one context per process on first use.
 */
int slgpu_ctx_create(int device, size_t hbm_budget, unsigned flags, slgpu_ctx** out);
void slgpu_ctx_destroy(slgpu_ctx* ctx);
int slgpu_last_error(const slgpu_ctx* ctx, char* buf, size_t len);
/* Bytes of device memory currently held by the context. */
int64_t slgpu_bytes_in_use(const slgpu_ctx* ctx);
/* Host-to-device and device-to-host bytes the context's calls have copied so
 * far (uploads of meshes, groups, data and constraints; downloads of CSR
 * arrays and values).  No counterpart in the reference (no device there). */
int slgpu_transfer_bytes(const slgpu_ctx* ctx, int64_t* h2d, int64_t* d2h);
/* Page-locks [ptr, ptr + bytes) of host memory for the context's device, so
 * that downloads into it (slgpu_matrix_download*) and uploads from it go
 * straight over the link instead of through page-locked staging blocks.
 * Meant for buffers that receive many downloads; locking costs about as much
 * as touching the pages once.  slgpu_host_unregister(ptr) undoes it, and must
 * be called before the memory is freed.  No counterpart in the reference. */
int slgpu_host_register(slgpu_ctx* ctx, void* ptr, size_t bytes);
int slgpu_host_unregister(slgpu_ctx* ctx, void* ptr);
/* The tile shapes the first-use tuner picked (one line each: kind, choice,
 * group shape ntf/ndof/ngp) and the CSR value kernel of each resident
 * pattern, as text.  No counterpart in the reference (a single fixed BLAS
 * switch, src/densemat.cpp:264-306, picks between dgemm and a loop). */
int slgpu_tuned_tiles(slgpu_ctx* ctx, char* buf, size_t len);

/*
 * Mesh geometry, resident on the device.  Replaces the node-coordinate and
 * curved-node gathers of rawfield::getjacterms (src/field/rawfield.cpp:2442-2502).
 *   xyz   [3*nnodes]                  node coordinates (nodes::getcoordinates)
 *   conn  [nelem*ncurvednodes]        curved nodes of each element of `elemtype`
 *                                     (elements::getsubelement(0, type, e, n))
 */
int slgpu_mesh_set_nodes(slgpu_ctx* ctx, int mesh, int64_t nnodes, const double* xyz);
int slgpu_mesh_set_elements(slgpu_ctx* ctx, int mesh, int elemtype, int ncurvednodes, int64_t nelem, const int32_t* conn);

/*
 * Coefficient program: a DAG evaluated at every (element, Gauss point).  Node
 * k's value is computed from its operands (earlier nodes).  Lowered from
 * sparselizard's operation trees (opconstant, opjac, opinvjac, opdetjac,
 * opparameter, opfield, opsum, opproduct, opinversion, oppower;
 * src/expression/operation/op*.cpp).
 */
enum {
    SLGPU_OP_CONST = 0,  /* consts[a] */
    SLGPU_OP_JAC = 1,    /* J(a,b) = d x_b / d ref_a   (jacobian::getjac, src/field/jacobian.cpp:387) */
    SLGPU_OP_INVJAC = 2, /* inverse of J, entry (a,b)   (jacobian::getinvjac, src/field/jacobian.cpp:396-504) */
    SLGPU_OP_DETJAC = 3, /* det J (signed)               (src/field/jacobian.cpp:308-349) */
    SLGPU_OP_ELEM = 4,   /* elemdata[a][e]: one value per element (per-region parameters, ...) */
    SLGPU_OP_FIELD = 5,  /* sum_f fielddata[a][f*nelem+e] * table b [orient][f][g] (rawfield::interpolate, rawfield.cpp:2632-2686) */
    SLGPU_OP_COORD = 6,  /* coordinate a (0 x, 1 y, 2 z) interpolated with the Lagrange geometry */
    SLGPU_OP_ADD = 7,    /* v[a] + v[b] */
    SLGPU_OP_MUL = 8,    /* v[a] * v[b] */
    SLGPU_OP_INV = 9,    /* 1 / v[a] */
    SLGPU_OP_NEG = 10,   /* -v[a] */
    SLGPU_OP_POW = 11    /* pow(v[a], v[b]) */
};

typedef struct {
    int32_t op, a, b, c;
} slgpu_node;

/* Form-function table: [norient][rows][ngp] values at the Gauss points for one
 * (derivative, component); hierarchicalformfunctioncontainer::tomatrix
 * (src/shapefunction/hierarchical/hierarchicalformfunctioncontainer.cpp:78-113)
 * for each total orientation used by the group. */
typedef struct {
    int32_t rows;
    const double* vals;
} slgpu_table;

/* One coef*dof*tf term (contribution.cpp:155-249).  dof_table < 0 marks a
 * right-hand-side term (no dof).  scale is the harmonic product factor of
 * harmonic::getproduct (src/harmonic.cpp:86-108), relative to the group. */
typedef struct {
    int32_t tf_table;
    int32_t dof_table;
    int32_t coef_node;
    int32_t pad;
    double scale;
} slgpu_term;

/* Where a group's element matrices go: rows from tfaddr [ntf][nelem], columns
 * from dofaddr [ndof][nelem] (dofmanager::getaddresses, -1 = not a DOF here,
 * src/formulation/dofmanager.cpp:846-918), values times multiplier. */
typedef struct {
    const int32_t* tfaddr;
    const int32_t* dofaddr;
    double multiplier;
} slgpu_dest;

/* Element types follow sparselizard's numbering (src/element.h): 0 point,
 * 1 line, 2 triangle, 3 quadrangle, 4 tetrahedron, 5 hexahedron, 6 prism,
 * 7 pyramid. */
typedef struct {
    int32_t mesh, elemtype, elemdim, problemdim;
    int64_t nelem;
    const int32_t* elems;   /* [nelem] element numbers within the type */
    const int32_t* orient;  /* [nelem] orientation variant index in [0, norient) */
    int32_t norient;
    int32_t ngp;
    const double* weights;  /* [ngp] Gauss weights */
    int32_t ncurvednodes;
    const double* lagrange; /* [1+elemdim][ncurvednodes][ngp]: Lagrange geometry values then ki/eta/phi derivatives */
    int32_t ntf, ndof;      /* form functions of the tf and dof fields (ndof = 1 for rhs groups) */
    int32_t ntables;
    const slgpu_table* tables;
    int32_t nnodes;
    const slgpu_node* nodes;
    int32_t nconsts;
    const double* consts;
    int32_t nelemdata;
    const double* const* elemdata;  /* each [nelem] */
    int32_t nfielddata;
    const double* const* fielddata; /* each [fieldrows[k]][nelem] */
    const int32_t* fieldrows;
    int32_t nterms;
    const slgpu_term* terms;
    int32_t ndests;
    const slgpu_dest* dests;
} slgpu_group;

/*
 * Matrix assembly (one per sparselizard rawmat).  Groups and raw COO
 * fragments accumulate; process() builds the A/D CSR split of
 * rawmat::process (src/formulation/rawmat.cpp:127-299): rows of constrained
 * DOFs dropped, constrained columns routed to D, both renumbered locally,
 * duplicates summed in a fixed order.
 */
typedef struct {
    int64_t nA;    /* unconstrained DOFs (rows of A and D) */
    int64_t nD;    /* constrained DOFs (columns of D) */
    int64_t nnzA;
    int64_t nnzD;
    int64_t ncoo;  /* COO entries generated (before -1 / constrained-row drops) */
    int32_t pattern_reused; /* 1 if the CSR pattern came from the resident cache */
    int32_t pad;
} slgpu_csr_info;

int slgpu_matrix_create(slgpu_ctx* ctx, int64_t ndofs, int* handle);
int slgpu_matrix_destroy(slgpu_ctx* ctx, int handle);
/* New matrix sharing the groups and fragments added so far (copy-on-write
 * support for rawmat::extractaccumulated, src/formulation/rawmat.cpp:328-337). */
int slgpu_matrix_clone(slgpu_ctx* ctx, int handle, int* new_handle);
/* Adds a copy of `g`; returns its group index in *index (may be NULL). */
int slgpu_matrix_add_group(slgpu_ctx* ctx, int handle, const slgpu_group* g, int* index);
/* With `enable`, a destination address array (tfaddr or dofaddr) whose host
 * pointer and length equal one given to an earlier slgpu_matrix_add_group of
 * this matrix since its last process() is taken to hold the same values: its
 * device copy and hash are reused instead of uploaded again.  The caller then
 * keeps such arrays unchanged, and alive, until process().  The slices of a
 * vector field's formulation pass the same address arrays many times
 * (dofmanager::getaddresses per component, src/formulation/dofmanager.cpp:846);
 * off by default. */
int slgpu_matrix_share_addresses(slgpu_ctx* ctx, int handle, int enable);
/* Raw fragment as stored by rawmat::accumulate (src/formulation/rawmat.cpp:57-65):
 * rows [ntr][nc], cols [ndr][nc], vals [nr][nc]; row r of vals uses rows[r/ndr]
 * and cols[r%ndr] when ntr or ndr differ from nr, else rows[r] and cols[r]. */
int slgpu_matrix_add_fragment(slgpu_ctx* ctx, int handle, int32_t ntr, int32_t ndr, int32_t nr, int64_t nc,
                              const int32_t* rows, const int32_t* cols, const double* vals);
/* Replaces per-element data array `k` of group `gi` (new coefficients on a resident pattern). */
int slgpu_matrix_set_elemdata(slgpu_ctx* ctx, int handle, int gi, int k, const double* values);
/* Replaces field coefficient array `k` ([rows][nelem]) of group `gi`. */
int slgpu_matrix_set_fielddata(slgpu_ctx* ctx, int handle, int gi, int k, const double* values);
/* Shape of group `gi` of a matrix (what requests may update). */
typedef struct {
    int32_t mesh, elemtype, ntf, ndof, nterms, ngp, norient, ndests;
    int32_t nelemdata, nfielddata;
    int32_t fieldrows[8]; /* rows of the first 8 fielddata arrays */
    int64_t nelem;        /* elements of the group */
    int64_t mesh_nelem;   /* elements of the group's type in its mesh */
} slgpu_group_desc;
int slgpu_matrix_group_count(slgpu_ctx* ctx, int handle, int* ngroups);
int slgpu_matrix_group_desc(slgpu_ctx* ctx, int handle, int gi, slgpu_group_desc* out);
/* Replaces term scales and destination multipliers of group `gi` (e.g. a new frequency). */
int slgpu_matrix_set_scales(slgpu_ctx* ctx, int handle, int gi, const double* term_scales, const double* dest_multipliers);
/* Current term scales (nterms) and destination multipliers (ndests) of group `gi`. */
int slgpu_matrix_get_scales(slgpu_ctx* ctx, int handle, int gi, double* term_scales, double* dest_multipliers);
/* Symmetry of group `gi`'s element matrices.  mirror (nterms values, may be
 * NULL) receives each term's mirror term: the term whose test-function and
 * dof tables hold the values of this term's dof and test-function tables,
 * with a coefficient of the same expression; all -1 when some term has none.
 * Coefficients match up to the order of the factors of a product.
 * *symmetric (may be NULL) is nonzero when the split-precision contraction
 * currently computes only the upper triangle and mirrors it (mirror terms
 * with equal scales): 1 when every coefficient equals its mirror's bit for
 * bit (the mirrored result is then the unmirrored one bit for bit), 2 when
 * some differ in the order of their factors (a few units in the last place).
 * *partner (may be NULL) is the group whose element matrices are the
 * transposes of this group's (same elements and data, ntf and ndof swapped,
 * terms matched with tables swapped, coefficients of the same expression and
 * equal scales), so that one split-precision contraction writes both; -1
 * when there is none.  The reference computes full element matrices for
 * every group (src/formulation/contribution.cpp:155-249). */
int slgpu_matrix_group_symmetry(slgpu_ctx* ctx, int handle, int gi, int32_t* mirror, int32_t* symmetric, int32_t* partner);
/* isconstrained [ndofs] (dofmanager::isconstrained, src/formulation/dofmanager.cpp:366-382). */
int slgpu_matrix_process(slgpu_ctx* ctx, int handle, const uint8_t* isconstrained, int precision, slgpu_csr_info* info);
/* Copies the processed CSR blocks to host memory: Arows/Drows [nA+1], Acols/Avals [nnzA], Dcols/Dvals [nnzD]. */
int slgpu_matrix_download(slgpu_ctx* ctx, int handle, int32_t* Arows, int32_t* Acols, double* Avals,
                          int32_t* Drows, int32_t* Dcols, double* Dvals);
/* Copies only the values (pattern unchanged since the last download). */
int slgpu_matrix_download_values(slgpu_ctx* ctx, int handle, double* Avals, double* Dvals);
/* Serial number of the CSR pattern that the matrix's last process() used (0
 * before the first).  Every pattern the context builds gets a new serial, so
 * two process() calls that report the same serial produced the same
 * Arows/Acols/Drows/Dcols (rawmat.cpp:127-299 for the same addresses and
 * constraints): a caller that kept the host copies of those arrays can
 * download the values alone. */
int slgpu_matrix_pattern_serial(slgpu_ctx* ctx, int handle, uint64_t* serial);
/* Device pointers to the processed CSR arrays (valid until the next process/destroy). */
int slgpu_matrix_device_csr(slgpu_ctx* ctx, int handle, const int32_t** Arows, const int32_t** Acols, const double** Avals,
                            const int32_t** Drows, const int32_t** Dcols, const double** Dvals);
/* Elimination of the constrained DOFs from a right-hand side on the device,
 * for a solver that takes the CSR blocks without a download:
 *   out[r] = b[Ainds[r]] - sum_j D[r][j] * b[Dinds[j]]
 * (mat::eliminate, src/formulation/mat.cpp:78-103: ba - D*bd with the product
 * summed over each row of D in column order).  b [ndofs] and out [nA] are
 * device pointers on the context's device; returns when out is written. */
int slgpu_matrix_eliminate(slgpu_ctx* ctx, int handle, const double* b, double* out);

/*
 * Right-hand side (contribution.cpp:293-300 + rawvec::setvalues "add",
 * src/formulation/rawvec.cpp:216-254): b_accum[addr] += -sum of the group's
 * element vectors, negative addresses skipped, duplicates summed in a fixed
 * order.  b_accum is a host array of length ndofs.
 */
int slgpu_rhs_assemble(slgpu_ctx* ctx, const slgpu_group* g, int64_t ndofs, int precision, double* b_accum);
/* The same right-hand side, returned as the rows it reaches (ascending DOF
 * numbers) and their values instead of added into a dense array: *count rows,
 * at most `capacity` (ntf * nelem * ndests always suffices).  Rows it does not reach
 * hold zero in the dense form.  For callers that add the result into a vector
 * of their own (rawvec::setvalues with "add", src/formulation/rawvec.cpp:216-254). */
int slgpu_rhs_assemble_rows(slgpu_ctx* ctx, const slgpu_group* g, int64_t ndofs, int precision, int32_t* rows, double* vals,
                            int64_t capacity, int64_t* count);

/* Device time (ms) of the phases of the last process()/rhs call:
 * [0] geometry+coefficients, [1] contraction, [2] pattern (symbolic), [3] CSR values, [4] total. */
int slgpu_last_timings(const slgpu_ctx* ctx, double* ms5);
/* Compiles (host only, no device needed) the runtime-generated geometry and
 * coefficient kernels the matrix's groups would use, returning SLGPU_E_CUDA
 * with the compiler log in `log` if one does not compile. */
int slgpu_check_coefficient_kernels(slgpu_ctx* ctx, int handle, char* log, size_t len);
/* Per kernel family, for the last process(): summed device time in ms (CUDA
 * events around each launch on the context's stream), number of launches and
 * algorithmic work of those launches.  Families and work units:
 *   "coefficients"        bytes of coefficients written (8 per term, point, element)
 *   "contract_fp64"       FLOPs, 2*ntf*ndof*nterms*ngp per element
 *   "slice_cols"          bytes: coefficients read, slices and exponents written
 *   "contract_split"      INT8 tensor operations, 2*pairs*ntf*ndof*nterms*ngp per
 *   "contract_split_fp32" element (pairs = 28 for the split tier, 15 for FP32)
 *   "row_values"          bytes: kept element values + slots, incidences, row
 *                         pointers read; A and D values written
 * A family that did not run reports zeros.  No counterpart in the reference
 * (a measurement hook). */
int slgpu_kernel_stats(const slgpu_ctx* ctx, const char* family, double* total_ms, int64_t* launches, double* work);
/* Number of kernels this context has launched so far (kernels of replayed
 * graphs included). */
int64_t slgpu_kernel_launches(const slgpu_ctx* ctx);

/* CUDA graphs for the value path of process() on a resident pattern
 * (default on; SLGPU_GRAPHS=0 in the environment turns them off at context
 * creation).  The second process() of a matrix whose launches would be the
 * same as the first's (same pattern, buffers and kernels) captures the
 * coefficient, contraction and CSR value launches into one graph; later ones
 * replay it.  Per-element data, field data, term scales, destination
 * multipliers and node coordinates changed in place are seen by the replay.
 * No counterpart in the reference (rawmat::process runs on the host,
 * rawmat.cpp:127-299). */
int slgpu_ctx_set_graphs(slgpu_ctx* ctx, int enable);
/* Number of graph replays of process() so far. */
int64_t slgpu_graph_launches(const slgpu_ctx* ctx);
/* Per-kernel and per-phase CUDA events inside process() (default on;
 * SLGPU_KERNEL_TIMERS=0 in the environment turns them off at context
 * creation).  Off, slgpu_kernel_stats reports nothing and
 * slgpu_last_timings only the total, and a replayed graph holds no event
 * nodes between its kernels.  No counterpart in the reference. */
int slgpu_ctx_set_kernel_timers(slgpu_ctx* ctx, int enable);

/* Algorithmic work of one process() of a matrix, for roofline accounting:
 * contraction_flops = sum over groups of nelem * sum over terms of
 * 2*ntf*ndof*ngp (the reference's K = M * coef^T counted once per term);
 * coef_points = sum of nelem*ngp; ncoo / nvalid = COO entries generated / kept;
 * nnz = nnzA + nnzD. */
typedef struct {
    double contraction_flops;
    int64_t coef_points;
    int64_t ncoo;
    int64_t nvalid;
    int64_t nnz;
    int64_t nA;
    int32_t ngroups;
    int32_t pad;
} slgpu_work;
int slgpu_matrix_work(slgpu_ctx* ctx, int handle, slgpu_work* out);

/* Record-only contexts: inspect what was recorded for a matrix handle. */
int slgpu_record_count(const slgpu_ctx* ctx, int handle, int* ngroups, int* nfragments);
int slgpu_record_group(const slgpu_ctx* ctx, int handle, int gi, slgpu_group* out);
int slgpu_record_fragment(const slgpu_ctx* ctx, int handle, int fi, int32_t* ntr, int32_t* ndr, int32_t* nr, int64_t* nc,
                          const int32_t** rows, const int32_t** cols, const double** vals);
int slgpu_record_constraints(const slgpu_ctx* ctx, int handle, int64_t* ndofs, const uint8_t** isconstrained);
/* Right-hand-side groups passed to slgpu_rhs_assemble on a record-only context
 * (which returns SLGPU_E_NODEVICE after recording). */
int slgpu_record_rhs_count(const slgpu_ctx* ctx, int* ngroups);
int slgpu_record_rhs_group(const slgpu_ctx* ctx, int gi, slgpu_group* out, int64_t* ndofs);
/* Mesh arrays given to slgpu_mesh_set_nodes / slgpu_mesh_set_elements. */
int slgpu_record_mesh(const slgpu_ctx* ctx, int mesh, int elemtype, int64_t* nnodes, const double** xyz, int* ncurvednodes,
                      int64_t* nelem, const int32_t** conn);

/*
 * Serving: assembly requests on resident problems, run concurrently.
 * No counterpart in the reference, whose generate()/A() is one synchronous
 * assembly; this is the request loop around the same path.
 *
 * A template is a matrix handle that has been processed once (its pattern,
 * meshes, tables and addresses are resident).  A request recomputes its
 * values with new per-element coefficient data and downloads them:
 *   - updates replace per-element data arrays of the template's groups
 *     (SLGPU_UPDATE_ELEMDATA: elemdata array `index`, 1 row;
 *     SLGPU_UPDATE_FIELDDATA: fielddata array `index`, `rows` rows), given in
 *     mesh element order of the group's element type ([rows][count], count =
 *     elements of that type in the mesh) and gathered into each group's own
 *     element order on the device;
 *   - Avals / Dvals receive nnzA / nnzD values (the template's pattern);
 *     page-locked buffers (slgpu_host_alloc) are written by the copy engine
 *     directly, others through a staging copy.
 * A server thread admits queued requests in arrival order as soon as one of
 * `nslots` execution slots is free and the request's device memory fits the
 * context's HBM budget; each slot has its own stream, so admitted requests
 * overlap on the device.  Results are bit-identical to the same request run
 * alone (fixed summation order, no atomics in the values).
 * While a server exists, every other call on its context is serialised with
 * it (context lock); destroying the server waits for its requests.  A
 * template must not be changed (set_elemdata/fielddata/scales, destroy is
 * safe) while requests on it are queued or running.
 */
typedef struct slgpu_server slgpu_server;

/* SLGPU_UPDATE_SCALES: new term scales and destination multipliers of group
 * `group` for this request only (a frequency of a harmonic problem, as
 * slgpu_matrix_set_scales sets them on the template): values = [nterms] term
 * scales then [ndests] multipliers, rows = nterms + ndests, count = 1,
 * index unused.  On a group whose element matrices are contracted as
 * symmetric, mirror terms must keep equal scales (else SLGPU_E_ARG). */
enum { SLGPU_UPDATE_ELEMDATA = 0, SLGPU_UPDATE_FIELDDATA = 1, SLGPU_UPDATE_SCALES = 2 };

typedef struct {
    int32_t group; /* group index in the template */
    int32_t kind;  /* SLGPU_UPDATE_* */
    int32_t index; /* elemdata / fielddata array index in the group */
    int32_t rows;  /* rows of the array (1 for elemdata) */
    const double* values; /* [rows][count], mesh element order; copied at submit, unless
                             every array of the request is page-locked (slgpu_host_alloc):
                             then read in place and kept unchanged until the request is done */
    int64_t count;
} slgpu_update;

typedef struct {
    int32_t handle;    /* template matrix */
    int32_t precision; /* SLGPU_PREC_* */
    int32_t nupdates;
    int32_t pad;
    const slgpu_update* updates;
    double* Avals; /* host, nnzA values */
    double* Dvals; /* host, nnzD values (may be NULL when nnzD = 0) */
} slgpu_request;

typedef struct {
    double submit_s; /* host times (seconds since the server was created) */
    double start_s;  /* launched on a slot */
    double done_s;   /* results in host memory */
    double device_ms; /* event time from the first to the last operation on the slot */
    int32_t slot;
    int32_t status;  /* SLGPU_OK, or the request's error code */
    double launch_ms; /* host time the server thread spent issuing the request */
    double launch_parts_ms[3]; /* of which: inputs and gathers, contractions, values and copies */
} slgpu_request_stats;

int slgpu_server_create(slgpu_ctx* ctx, int nslots, slgpu_server** out);
/* Queues a request; returns its ticket.  Update values in pageable memory
 * are copied; page-locked ones are read in place (see slgpu_update). */
int slgpu_server_submit(slgpu_server* s, const slgpu_request* r, int64_t* ticket);
/* Waits up to timeout_s (< 0: no limit) for a request.  Returns SLGPU_OK when
 * it completed, SLGPU_E_TIMEOUT when still running, or the request's own
 * error code (message via slgpu_server_error).  stats may be NULL. */
/* Queues a new template: a matrix whose groups and fragments were added but
 * that was never processed (a new mesh, new orders, a new formulation).
 * When admitted -- in arrival order, against the HBM budget like any request
 * -- the server runs its first slgpu_matrix_process (pattern build and
 * values) with these constraint flags (ndofs bytes, copied at submit; NULL:
 * none constrained).  Once its ticket is done, requests may use the handle
 * as a template.  The pattern build synchronises the context's main stream;
 * requests already running on the slots continue meanwhile. */
int slgpu_server_submit_template(slgpu_server* s, int handle, const uint8_t* isconstrained, int precision, int64_t* ticket);
int slgpu_server_wait(slgpu_server* s, int64_t ticket, double timeout_s, slgpu_request_stats* stats);
int slgpu_server_error(slgpu_server* s, int64_t ticket, char* buf, size_t len);
/* Forgets a completed request. */
int slgpu_server_release(slgpu_server* s, int64_t ticket);
/* Requests queued or running. */
int64_t slgpu_server_pending(slgpu_server* s);
/* The server's clock: seconds since it was created (the time base of
 * slgpu_request_stats). */
double slgpu_server_clock(slgpu_server* s);
/* Readies every slot for requests of `precision` on a template: the slot's
 * request arena and split-precision scratch are grown to fit one request that
 * updates every per-element array, and the template's split operands are
 * built, so that the first requests allocate no device memory.  Only while
 * the server has no queued or running requests (else SLGPU_E_ARG).  No
 * counterpart in the reference. */
int slgpu_server_prepare(slgpu_server* s, int handle, int precision);
/* Waits for every request, stops the server thread and frees its slots. */
void slgpu_server_destroy(slgpu_server* s);
/* Page-locked host memory for request outputs (and inputs). */
int slgpu_host_alloc(slgpu_ctx* ctx, size_t bytes, void** out);
void slgpu_host_free(void* p);

/*
 * Element matrices of one group without allocating device memory.
 * This entry point has no counterpart in the reference: it exists for
 * callers that cannot allocate GPU memory themselves -- a host application
 * whose own allocator owns the whole device heap, or a latency-critical loop
 * that must not pay for cudaMalloc/cudaFree -- and already hold the mesh and
 * output buffers on the device.
 *   g          group description in host memory, as for slgpu_matrix_add_group
 *              (destinations are not used and may be absent: ndests = 0)
 *   xyz        device pointer, [3*nnodes] node coordinates
 *   nnodes     number of nodes in xyz; an element whose connectivity names a
 *              node outside [0, nnodes) is not read and its matrix is NaN
 *   conn       device pointer, [mesh_nelem*ncurvednodes] curved-node
 *              connectivity of g->elemtype
 *   K          device pointer, [nelem][ntf*ndof] output: K[e*ntf*ndof+i*ndof+j]
 *              = sum over terms of scale * element matrix entry (i, j) of
 *              element e (no destination multiplier)
 *   stream     cudaStream_t the work is queued on (0 = legacy default stream);
 *              the call returns once the work is queued
 *   err/errlen optional buffer for the error message
 * The group's host arrays (tables, per-element and field data, element
 * numbers, ...) are copied to the device on `stream`.  Arrays in pageable
 * memory may be reused as soon as the call returns; arrays in page-locked
 * memory are read when the stream reaches the copy, so they must stay
 * allocated and unchanged until then.  While `stream` is capturing, the call
 * returns SLGPU_E_UNSUPPORTED and queues nothing.
 * Working memory is a 32 MiB array compiled into this library's device image
 * (held on every GPU that loads the library until the process exits).
 * Groups needing more (program, tables, per-element data and
 * nterms*ngp*nelem doubles of coefficients) are rejected with SLGPU_E_BUDGET.
 * The first call on each device looks up the array's device address; make
 * that first call before any stream capture, and do not use the library
 * across a cudaDeviceReset.  All calls share the array: calls that may run
 * at the same time on the GPU race and must be ordered by the caller (same
 * stream, or events).
 */
int slgpu_element_matrices_noalloc(const slgpu_group* g, const double* xyz, int64_t nnodes, const int32_t* conn,
                                   int64_t mesh_nelem, double* K, void* stream, char* err, size_t errlen);

#ifdef __cplusplus
}
#endif

#endif
