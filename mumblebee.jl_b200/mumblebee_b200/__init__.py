"""B200-native interior-point hot path of Mumblebee.jl (see ipm.py for the API)."""
from .ipm import (IPMProblem, IPMSettings, IPMSolver, IPMResult, IPMHistory, IPMStatus, KKTStatus, Batch,
                  AbstractCone, CofreeCone, PositiveCone, SecondOrderCone, SemidefiniteCone, ExponentialCone,
                  PowerCone, Context, init, reinit, step, solve, solve_, print_timers, frule, frule2, rrule,
                  batch_solve,
                  batch_solve_static, Server)
from .comp import BlockSparseMatrix, blocksparse, extmul, twomul
from . import autotune, moi

__all__ = ["IPMProblem", "IPMSettings", "IPMSolver", "IPMResult", "IPMHistory", "IPMStatus", "KKTStatus", "Batch",
           "AbstractCone", "CofreeCone", "PositiveCone", "SecondOrderCone", "SemidefiniteCone", "ExponentialCone",
           "PowerCone", "Context", "init", "reinit", "step", "solve", "solve_", "print_timers", "frule", "frule2", "rrule",
           "batch_solve",
           "batch_solve_static", "Server", "BlockSparseMatrix", "blocksparse", "extmul", "twomul", "autotune", "moi"]
