"""Output bundle of the theory in the reference's ``.dat`` format (skyrmion_solver th/lightly_bound_skyrme/io.py)."""
from ...core.io import make_output_data_bundle

output_data_bundle = make_output_data_bundle("lightly_bound")
