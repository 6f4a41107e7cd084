"""B200-native interior-point hot path of Mumblebee.jl (see ipm.py for the API)."""
from .ipm import (IPMProblem, IPMSettings, IPMSolver, IPMResult, IPMHistory, IPMStatus, KKTStatus, Batch,
                  AbstractCone, CofreeCone, PositiveCone, SecondOrderCone, SemidefiniteCone, ExponentialCone,
                  PowerCone, Context, init, reinit, step, solve, solve_, print_timers, frule, frule2, rrule,
                  batch_solve,
                  batch_solve_static, Server)

__all__ = ["IPMProblem", "IPMSettings", "IPMSolver", "IPMResult", "IPMHistory", "IPMStatus", "KKTStatus", "Batch",
           "AbstractCone", "CofreeCone", "PositiveCone", "SecondOrderCone", "SemidefiniteCone", "ExponentialCone",
           "PowerCone", "Context", "init", "reinit", "step", "solve", "solve_", "print_timers", "frule", "frule2", "rrule",
           "batch_solve",
           "batch_solve_static", "Server"]
