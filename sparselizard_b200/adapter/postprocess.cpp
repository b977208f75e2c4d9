// Post-processing on the GPU through the same lowering as the assembly.
//
// expression::integrate (src/expression/expression.cpp:808-889) sums, per
// element, the expression at the Gauss points times the weights and |det J|.
// The element-wise right-hand side of a "one" field (one form function of
// value 1 per element) holds exactly those per-element integrals, negated
// (contribution.cpp:293-300): b_e = -sum_g w_g |det J| expr(e, g).  So the
// integral is the negated sum of that right-hand side, which the GPU
// contribution::generate and slgpu_rhs_assemble compute: coefficient program
// at the Gauss points (field values interpolated on the device), contraction
// with the constant form function and the deterministic scatter.
#include "sparselizard.h"
#include "slgpu_adapter.h"

namespace slgpu_adapter {

double integrate(expression e, int physreg, int integrationorder)
{
    if (!e.isscalar()) {
        logs log;
        log.msg() << "Error in slgpu_adapter::integrate: cannot integrate a nonscalar expression" << std::endl;
        log.error();
    }
    field one("one");
    formulation f;
    // Integration order of a contribution: dof order + tf order + 2 + delta,
    // with both orders 0 for a "one" field without dof.
    f += sl::integral(physreg, e * sl::tf(one), integrationorder - 2);
    f.generaterhs();
    vec b = f.rhs(false, false);
    densemat v = b.getallvalues();
    const double* bv = v.getvalues();
    double s = 0;
    for (long long i = 0; i < v.count(); i++) s += bv[i];
    return -s;
}

}  // namespace slgpu_adapter
