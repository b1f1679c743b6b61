from .lm_optimizer import LMOptimizer, LMOptimizerConfig, OptimizerConfig
from .var_values import Var, VarKey, VarValues

__all__ = ["LMOptimizer", "LMOptimizerConfig", "OptimizerConfig", "Var", "VarKey", "VarValues"]
