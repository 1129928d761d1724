"""Physical constants shared by the solver front end.

Values follow ``hornlab_metal_bem/_constants.py:3-5`` of the reference.
"""
from __future__ import annotations

SPEED_OF_SOUND: float = 343.0
AIR_DENSITY: float = 1.2041
REFERENCE_PRESSURE: float = 20e-6
