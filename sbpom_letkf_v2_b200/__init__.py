"""B200 (sm_100a) implementation of the sbPOM-LETKF analysis step."""
from .params import LETKFParams  # noqa: F401
