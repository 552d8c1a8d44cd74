"""gridsim_b200 — B200-native AC load flow and N-1 contingency screen behind GridSim's solver seams."""
from .model import GridModel, load_case_dir, load_matpower, parse_matpower, save_case_dir  # noqa: F401
