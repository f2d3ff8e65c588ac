"""hedge_b200: a B200-native (sm_100a) backend for hedge's DG right-hand side.

Host set-up (reference element, mesh, connectivity) is FP64 numpy; every
right-hand-side evaluation and LSRK stage runs in hand-written CUDA kernels
(libhedge_b200.so) behind a C ABI (include/hedge_b200.h).
"""

from .mesh import (Mesh, TAG_ALL, TAG_NONE, make_regular_rect_mesh,
                   make_box_tet_mesh, check_bc_coverage)
from .refelem import TriangleElement, TetrahedronElement, make_element
from .models import (StrongAdvectionOperator, WeakAdvectionOperator, StrongWaveOperator,
                     VariableVelocityStrongWaveOperator, MaxwellOperator,
                     TMMaxwellOperator, TEMaxwellOperator,
                     VariableCoefficientAdvectionOperator, make_tdep_constant, TimeConstantGivenFunction,
                     TimeDependentGivenFunction)
from .discretization import Discretization, CompiledOperator, BoundRHS
from .timestep import GraphedLSRK4, LSRK4TimeStepper, RK4TimeStepper
from .nd_calculus import GradientOperator, DivergenceOperator
from .visualization import VtkVisualizer, LegacyVtkVisualizer

__all__ = [
    "Mesh", "TAG_ALL", "TAG_NONE", "make_regular_rect_mesh", "make_box_tet_mesh",
    "check_bc_coverage", "TriangleElement", "TetrahedronElement", "make_element",
    "StrongAdvectionOperator", "WeakAdvectionOperator", "StrongWaveOperator",
    "VariableVelocityStrongWaveOperator", "MaxwellOperator", "TMMaxwellOperator",
    "TEMaxwellOperator", "VariableCoefficientAdvectionOperator", "make_tdep_constant",
    "TimeConstantGivenFunction", "TimeDependentGivenFunction", "Discretization", "CompiledOperator", "BoundRHS",
    "LSRK4TimeStepper", "RK4TimeStepper", "GraphedLSRK4", "GradientOperator", "DivergenceOperator",
    "VtkVisualizer", "LegacyVtkVisualizer",
]
