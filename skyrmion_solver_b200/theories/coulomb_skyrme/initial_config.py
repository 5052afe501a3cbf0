"""Initial configurations of the Coulomb Skyrme model (host-built FP64 fields uploaded to ``Field``)."""
from .._init_common import make_initialize

initialize = make_initialize("coulomb")
