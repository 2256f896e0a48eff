"""Alias of fan_equiangluar (the reference numpy module name is misspelt)."""
from .fan_equiangluar import *  # noqa: F401,F403
from .fan_equiangluar import distance_driven_bp, distance_driven_fp, fbp_bp, ramp_filter, siddon_bp, siddon_fp  # noqa: F401,E501
