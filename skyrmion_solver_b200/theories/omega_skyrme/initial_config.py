"""Initial configurations of the Omega Skyrme model (host-built FP64 fields uploaded to ``Field``)."""
from .._init_common import make_initialize

initialize = make_initialize("omega")
