"""TBPM API of the reference (`tbplas.tbpm`): Config, Solver, Analyzer."""
from .analysis import Analyzer, window_exp, window_exp_ten, window_hanning
from .config import Config, read_config
from .solver import Solver

__all__ = ["Config", "read_config", "Solver", "Analyzer", "window_hanning", "window_exp",
           "window_exp_ten"]
