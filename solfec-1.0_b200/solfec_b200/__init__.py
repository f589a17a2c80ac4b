"""B200-native contact-solve path of Solfec-1.0 (local dynamics assembly,
colour-by-colour block Gauss-Seidel with the Signorini-Coulomb diagonal
solvers, merit function) behind the reference's GAUSS_SEIDEL_SOLVER interface.

The compute path is libsolfec_b200.so (sm_100a CUDA kernels, host code in C);
this package binds it and provides the seeded synthetic scenes."""
from .solver import GAUSS_SEIDEL_SOLVER, LOCDYN, SolfecError, DeviceError  # noqa: F401
from . import scenes  # noqa: F401
from . import dynamics  # noqa: F401
from . import detect  # noqa: F401
