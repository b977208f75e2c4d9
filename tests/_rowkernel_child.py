"""Child process for tests that compare engine variants chosen by environment
(SLGPU_ROW_KERNEL, SLGPU_FUSED_SPLIT): assembles synthetic matrices in FP64
and split precision and saves the values (argv[1])."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from sparselizard_b200 import abi  # noqa: E402

import test_gpu_graphs as T  # noqa: E402

ctx = abi.Context(0)
out = {}
for name, (grid, ntf, ndof, nterms, ngp1, ndofs) in {"narrow": (60, 9, 9, 4, 3, 3000), "wide": (30, 20, 40, 3, 3, 4000),
                                                      "small": (80, 4, 4, 3, 2, 5000), "short": (40, 4, 4, 2, 2, 20000)}.items():
    rng = np.random.Generator(np.random.PCG64(31))
    t = T._setup(ctx, rng, 20 + len(out), grid, ntf, ndof, nterms, ngp1, ndofs)
    for prec in (abi.PREC_FP64, abi.PREC_SPLIT):
        A, D = T._process(ctx, t, prec)
        out[f"{name}_{prec}_A"], out[f"{name}_{prec}_D"] = A, D
ctx.close()
np.savez(sys.argv[1], **out)
