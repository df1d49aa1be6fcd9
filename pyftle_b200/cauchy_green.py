"""Flow-map Jacobians (pyFTLE ``cauchy_green.py`` names); implemented in ``pyftle_b200.ftle``."""

from pyftle_b200.ftle import compute_flow_map_jacobian_2x2, compute_flow_map_jacobian_3x3

__all__ = ["compute_flow_map_jacobian_2x2", "compute_flow_map_jacobian_3x3"]
