"""se_b200 -- B200-native semi-Lagrangian advection and spectral-element
Helmholtz/Poisson solves for SE (davelee2804/SE).

The product is ``libsegpu.so`` (C-ABI declared in ``include/segpu.h``),
built in-tree by :mod:`se_b200.build`. :mod:`se_b200.segpu` mirrors the
reference's classes (Mesh, BCs, Field, Advector, HelmholtzEqn, PoissonEqn)
over that C-ABI.
"""
from .segpu import (BCs, Advector, Server, REQ_ADVECT, REQ_HELMHOLTZ, CalcTimeStep, Field, FieldError, GenVel, HelmholtzEqn, Mesh, NavierStokesEqn,  # noqa: F401
                    TwoLayerQGEqn, WriteXDMF, WriteXDMFHeader, WriteXDMFFooter, WriteXDMFTemporal,
                    PoissonEqn, SEError, load_library, set_stream, solver_opts, synchronize, solve_batch,
                    MODE_EXACT, MODE_REFERENCE, PREC_FP64, PREC_MIXED, PREC_BF16, PREC_FP16, PREC_FP64_TC,
                    METHOD_CG,
                    METHOD_FDM, NORM_NATURAL,
                    NORM_PRECONDITIONED, NORM_UNPRECONDITIONED)

__all__ = ["Mesh", "BCs", "Field", "Advector", "HelmholtzEqn", "PoissonEqn", "NavierStokesEqn",
           "TwoLayerQGEqn", "GenVel", "CalcTimeStep",
           "FieldError", "SEError", "load_library", "set_stream", "synchronize", "solver_opts"]
