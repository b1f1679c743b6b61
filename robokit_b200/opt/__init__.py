from .lm_optimizer import LMOptimizer, LMOptimizerConfig, OptimizerConfig
from .population_solver import PopulationSolver, PopulationSolverConfig, Stage
from .var_values import Var, VarKey, VarValues

__all__ = ["LMOptimizer", "LMOptimizerConfig", "OptimizerConfig", "PopulationSolver", "PopulationSolverConfig",
           "Stage", "Var", "VarKey", "VarValues"]
