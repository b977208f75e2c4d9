/*
 * slref.c -- CPU restatement of sparselizard's assembly hot path (test
 * oracle; see slref.h).  Plain C11, single-threaded, written for clarity and
 * for the reference's order of operations, not for speed.
 */
#include "slref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Jacobian of the mesh-dimension element at one Gauss point:
 * J[a][b] = sum_n dN_n/dref_a(g) * x_b(n)   (rawfield::getjacterms, src/field/rawfield.cpp:2442-2502)
 * det J and inverse by cofactors        (src/field/jacobian.cpp:308-349, :396-504). */
static void jacobian(const slgpu_group* g, const double* xyz, const int32_t* conn, int64_t e, int gp, double J[3][3], double inv[3][3],
                     double* det, double X[3])
{
    const int ncn = g->ncurvednodes, ngp = g->ngp, dim = g->problemdim;
    memset(J, 0, 9 * sizeof(double));
    memset(inv, 0, 9 * sizeof(double));
    X[0] = X[1] = X[2] = 0;
    const int32_t* cn = conn + (int64_t)g->elems[e] * ncn;
    for (int a = 0; a < dim; a++)
        for (int b = 0; b < dim; b++) {
            double s = 0;
            for (int n = 0; n < ncn; n++) s += xyz[3 * (int64_t)cn[n] + b] * g->lagrange[((int64_t)(1 + a) * ncn + n) * ngp + gp];
            J[a][b] = s;
        }
    for (int b = 0; b < 3; b++) {
        double s = 0;
        for (int n = 0; n < ncn; n++) s += xyz[3 * (int64_t)cn[n] + b] * g->lagrange[(int64_t)n * ngp + gp];
        X[b] = s;
    }
    if (dim == 1) {
        *det = J[0][0];
        inv[0][0] = 1.0 / J[0][0];
    } else if (dim == 2) {
        *det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        inv[0][0] = J[1][1] / *det;
        inv[0][1] = -J[0][1] / *det;
        inv[1][0] = -J[1][0] / *det;
        inv[1][1] = J[0][0] / *det;
    } else {
        *det = J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) - J[0][1] * (J[1][0] * J[2][2] - J[2][0] * J[1][2]) +
               J[0][2] * (J[1][0] * J[2][1] - J[2][0] * J[1][1]);
        inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / *det;
        inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / *det;
        inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / *det;
        inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / *det;
        inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / *det;
        inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / *det;
        inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / *det;
        inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / *det;
        inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / *det;
    }
}

/* Coefficient DAG at one (element, Gauss point): the values the reference's
 * operation::interpolate returns for that point. */
static void eval_nodes(const slgpu_group* g, int64_t e, int gp, int o, double J[3][3], double inv[3][3], double det, const double X[3],
                       double* v)
{
    for (int k = 0; k < g->nnodes; k++) {
        const slgpu_node nd = g->nodes[k];
        double r = 0;
        switch (nd.op) {
        case SLGPU_OP_CONST: r = g->consts[nd.a]; break;
        case SLGPU_OP_JAC: r = J[nd.a][nd.b]; break;
        case SLGPU_OP_INVJAC: r = inv[nd.a][nd.b]; break;
        case SLGPU_OP_DETJAC: r = det; break;
        case SLGPU_OP_ELEM: r = g->elemdata[nd.a][e]; break;
        case SLGPU_OP_FIELD: {
            const int rows = g->fieldrows[nd.a];
            const double* tb = g->tables[nd.b].vals + (int64_t)o * rows * g->ngp;
            for (int f = 0; f < rows; f++) r += g->fielddata[nd.a][(int64_t)f * g->nelem + e] * tb[(int64_t)f * g->ngp + gp];
            break;
        }
        case SLGPU_OP_COORD: r = X[nd.a]; break;
        case SLGPU_OP_ADD: r = v[nd.a] + v[nd.b]; break;
        case SLGPU_OP_MUL: r = v[nd.a] * v[nd.b]; break;
        case SLGPU_OP_INV: r = 1.0 / v[nd.a]; break;
        case SLGPU_OP_NEG: r = -v[nd.a]; break;
        case SLGPU_OP_POW: r = pow(v[nd.a], v[nd.b]); break;
        default: r = NAN;
        }
        v[k] = r;
    }
}

/* Magnitude mode: every product and every summand replaced by its absolute
 * value, giving sum |terms| for each entry -- the scale of the standard
 * floating-point error bound |fl(sum) - sum| <= gamma_n * sum |terms|. */
static int g_absmode = 0;

void slref_set_absmode(int on) { g_absmode = on; }

int slref_element_matrices(const slgpu_group* g, const double* xyz, const int32_t* conn, double* K)
{
    const int ngp = g->ngp, ntf = g->ntf, ndof = g->ndof, nterms = g->nterms, ndests = g->ndests;
    const int64_t nelem = g->nelem;
    const int64_t P = (int64_t)ntf * ndof;
    double* v = malloc(sizeof(double) * (g->nnodes > 0 ? g->nnodes : 1));
    double* coefdet = malloc(sizeof(double) * (size_t)nterms * ngp); /* coef * |detJ| (contribution.cpp:200) */
    double* Kt = malloc(sizeof(double) * (size_t)P);
    double* Kd = malloc(sizeof(double) * (size_t)P);
    if (!v || !coefdet || !Kt || !Kd) {
        free(v); free(coefdet); free(Kt); free(Kd);
        return 1;
    }
    for (int64_t e = 0; e < nelem; e++) {
        const int o = g->orient[e];
        for (int gp = 0; gp < ngp; gp++) {
            double J[3][3], inv[3][3], det, X[3];
            jacobian(g, xyz, conn, e, gp, J, inv, &det, X);
            eval_nodes(g, e, gp, o, J, inv, det, X, v);
            for (int t = 0; t < nterms; t++) coefdet[(int64_t)t * ngp + gp] = v[g->terms[t].coef_node] * fabs(det);
        }
        for (int d = 0; d < ndests; d++) {
            for (int64_t p = 0; p < P; p++) Kd[p] = 0;
            for (int t = 0; t < nterms; t++) {
                const slgpu_term tm = g->terms[t];
                const double* T = g->tables[tm.tf_table].vals + (int64_t)o * ntf * ngp;
                const double* D = tm.dof_table >= 0 ? g->tables[tm.dof_table].vals + (int64_t)o * ndof * ngp : NULL;
                /* M[(i,j)][g] = (tf[i][g] * w[g]) * dof[j][g]; K = M * coefdet^T
                 * (contribution.cpp:172-210, densemat.cpp:608-636). */
                for (int i = 0; i < ntf; i++)
                    for (int j = 0; j < ndof; j++) {
                        double s = 0;
                        for (int gp = 0; gp < ngp; gp++) {
                            double m = T[(int64_t)i * ngp + gp] * g->weights[gp];
                            if (D) m *= D[(int64_t)j * ngp + gp];
                            if (g_absmode)
                                s += fabs(m) * fabs(coefdet[(int64_t)t * ngp + gp]);
                            else
                                s += m * coefdet[(int64_t)t * ngp + gp];
                        }
                        Kt[(int64_t)i * ndof + j] = s;
                    }
                /* Harmonic folding: stiffness += factor * K_term (contribution.cpp:220-246). */
                const double factor = g_absmode ? fabs(tm.scale * g->dests[d].multiplier) : tm.scale * g->dests[d].multiplier;
                for (int64_t p = 0; p < P; p++) Kd[p] += factor * Kt[p];
            }
            for (int64_t p = 0; p < P; p++) K[((int64_t)d * P + p) * nelem + e] = Kd[p];
        }
    }
    free(v); free(coefdet); free(Kt); free(Kd);
    return 0;
}

typedef struct {
    int32_t col;
    int64_t idx;
    double val;
} entry;

static int cmp_entry(const void* a, const void* b)
{
    const entry* x = a;
    const entry* y = b;
    if (x->col != y->col)
        return x->col < y->col ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

int slref_matrix(const slgpu_group* groups, int ngroups, const double* xyz, const int32_t* const* conn_per_group, const slref_fragment* frags,
                 int nfrags, int64_t ndofs, const uint8_t* isconstrained, slref_csr* out)
{
    memset(out, 0, sizeof(*out));
    /* findtruefalse + renumtolocalindex (rawmat.cpp:133). */
    int32_t* renum = malloc(sizeof(int32_t) * (size_t)(ndofs > 0 ? ndofs : 1));
    int64_t nA = 0, nD = 0;
    for (int64_t i = 0; i < ndofs; i++) renum[i] = isconstrained[i] ? (int32_t)nD++ : (int32_t)nA++;
    /* Element matrices of every group. */
    double** K = calloc((size_t)(ngroups > 0 ? ngroups : 1), sizeof(double*));
    for (int gi = 0; gi < ngroups; gi++) {
        const slgpu_group* g = &groups[gi];
        K[gi] = malloc(sizeof(double) * (size_t)g->ndests * g->ntf * g->ndof * (g->nelem > 0 ? g->nelem : 1));
        if (!K[gi] || slref_element_matrices(g, xyz, conn_per_group[gi], K[gi]))
            return 1;
    }
    /* Pass 1: per-row counts (rawmat.cpp:136-169). */
    int64_t* rowcount = calloc((size_t)(ndofs + 1), sizeof(int64_t));
    int64_t total = 0;
#define VISIT(BODY)                                                                                                 \
    do {                                                                                                            \
        int64_t idx = 0;                                                                                            \
        for (int gi = 0; gi < ngroups; gi++) {                                                                      \
            const slgpu_group* g = &groups[gi];                                                                     \
            const int64_t P = (int64_t)g->ntf * g->ndof;                                                            \
            for (int d = 0; d < g->ndests; d++)                                                                     \
                for (int64_t p = 0; p < P; p++)                                                                     \
                    for (int64_t e = 0; e < g->nelem; e++, idx++) {                                                 \
                        const int64_t i = p / g->ndof, j = p % g->ndof;                                             \
                        const int32_t cr = g->dests[d].tfaddr[i * g->nelem + e];                                    \
                        const int32_t cc = g->dests[d].dofaddr[j * g->nelem + e];                                   \
                        const double cv = K[gi][((int64_t)d * P + p) * g->nelem + e];                               \
                        BODY                                                                                        \
                    }                                                                                               \
        }                                                                                                           \
        for (int fi = 0; fi < nfrags; fi++) {                                                                       \
            const slref_fragment* f = &frags[fi];                                                                   \
            for (int64_t r = 0; r < f->nr; r++) {                                                                   \
                int64_t ctr = r, cdr = r;                                                                           \
                if (f->ntr != f->nr || f->ndr != f->nr) {                                                           \
                    ctr = r / f->ndr;                                                                               \
                    cdr = r % f->ndr;                                                                               \
                }                                                                                                   \
                for (int64_t c = 0; c < f->nc; c++, idx++) {                                                        \
                    const int32_t cr = f->rows[ctr * f->nc + c];                                                    \
                    const int32_t cc = f->cols[cdr * f->nc + c];                                                    \
                    const double cv = g_absmode ? fabs(f->vals[r * f->nc + c]) : f->vals[r * f->nc + c];            \
                    BODY                                                                                            \
                }                                                                                                   \
            }                                                                                                       \
        }                                                                                                           \
    } while (0)

    VISIT({
        (void)cv;
        if (cr >= 0 && cc >= 0 && !isconstrained[cr]) {
            rowcount[cr]++;
            total++;
        }
    });
    int64_t* ads = malloc(sizeof(int64_t) * (size_t)(ndofs + 1));
    ads[0] = 0;
    for (int64_t i = 0; i < ndofs; i++) ads[i + 1] = ads[i] + rowcount[i];
    entry* ent = malloc(sizeof(entry) * (size_t)(total > 0 ? total : 1));
    int64_t* fill = calloc((size_t)(ndofs + 1), sizeof(int64_t));
    /* Pass 2: scatter (col, val) in insertion order (rawmat.cpp:177-218). */
    VISIT({
        if (cr >= 0 && cc >= 0 && !isconstrained[cr]) {
            entry* en = &ent[ads[cr] + fill[cr]++];
            en->col = cc;
            en->idx = idx;
            en->val = cv;
        }
    });
#undef VISIT
    /* Per-row stable sort by (col, index) and duplicate sums (rawmat.cpp:67-125). */
    int64_t nnzA = 0, nnzD = 0;
    int64_t* uniq = calloc((size_t)(ndofs + 1), sizeof(int64_t));
    for (int64_t r = 0; r < ndofs; r++) {
        entry* row = ent + ads[r];
        const int64_t n = rowcount[r];
        qsort(row, (size_t)n, sizeof(entry), cmp_entry);
        int64_t w = -1;
        for (int64_t k = 0; k < n; k++) {
            if (w >= 0 && row[w].col == row[k].col)
                row[w].val += row[k].val;
            else {
                row[++w] = row[k];
                if (isconstrained[row[w].col]) nnzD++;
                else nnzA++;
            }
        }
        uniq[r] = w + 1;
    }
    /* A (unconstrained x unconstrained) and D (unconstrained x constrained) (rawmat.cpp:241-289). */
    out->nA = nA;
    out->nD = nD;
    out->nnzA = nnzA;
    out->nnzD = nnzD;
    out->Arows = calloc((size_t)(nA + 1), sizeof(int32_t));
    out->Drows = calloc((size_t)(nA + 1), sizeof(int32_t));
    out->Acols = malloc(sizeof(int32_t) * (size_t)(nnzA > 0 ? nnzA : 1));
    out->Dcols = malloc(sizeof(int32_t) * (size_t)(nnzD > 0 ? nnzD : 1));
    out->Avals = malloc(sizeof(double) * (size_t)(nnzA > 0 ? nnzA : 1));
    out->Dvals = malloc(sizeof(double) * (size_t)(nnzD > 0 ? nnzD : 1));
    int64_t index = 0;
    for (int64_t r = 0; r < ndofs; r++) {
        if (isconstrained[r])
            continue;
        out->Arows[index + 1] = out->Arows[index];
        out->Drows[index + 1] = out->Drows[index];
        const entry* row = ent + ads[r];
        for (int64_t k = 0; k < uniq[r]; k++) {
            if (isconstrained[row[k].col]) {
                out->Dcols[out->Drows[index + 1]] = renum[row[k].col];
                out->Dvals[out->Drows[index + 1]] = row[k].val;
                out->Drows[index + 1]++;
            } else {
                out->Acols[out->Arows[index + 1]] = renum[row[k].col];
                out->Avals[out->Arows[index + 1]] = row[k].val;
                out->Arows[index + 1]++;
            }
        }
        index++;
    }
    for (int gi = 0; gi < ngroups; gi++) free(K[gi]);
    free(K); free(renum); free(rowcount); free(ads); free(ent); free(fill); free(uniq);
    return 0;
}

int slref_rhs(const slgpu_group* g, const double* xyz, const int32_t* conn, int64_t ndofs, double* b)
{
    const int64_t P = g->ntf;
    double* K = malloc(sizeof(double) * (size_t)g->ndests * P * (g->nelem > 0 ? g->nelem : 1));
    if (!K || slref_element_matrices(g, xyz, conn, K)) {
        free(K);
        return 1;
    }
    /* stiffnesses.minus(); rawvec::setvalues(addresses, values, "add"), negative addresses skipped. */
    for (int d = 0; d < g->ndests; d++)
        for (int64_t i = 0; i < P; i++)
            for (int64_t e = 0; e < g->nelem; e++) {
                const int32_t a = g->dests[d].tfaddr[i * g->nelem + e];
                if (a >= 0 && a < ndofs)
                    b[a] += -K[((int64_t)d * P + i) * g->nelem + e];
            }
    free(K);
    return 0;
}

void slref_free(slref_csr* c)
{
    free(c->Arows); free(c->Acols); free(c->Avals);
    free(c->Drows); free(c->Dcols); free(c->Dvals);
    memset(c, 0, sizeof(*c));
}
