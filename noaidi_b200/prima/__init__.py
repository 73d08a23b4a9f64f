"""Host-side mirror of prima-core for the device backend."""
from .model import Direct, LpBuilder, LpProblem, Negated, Range, RowTranslation, SparseMatrix
from .types import (Convergence, KktError, LpSolution, MixedPrecisionParams, MixedPrecisionResult,
                    PdhgParams, ScalingParams, SolveStatus, WarmStart, convergence)
