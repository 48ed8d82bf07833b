"""nuvort_b200 -- B200-native filament-velocity path of the NuVort vortex-filament code."""
from .abi import State, make_params, default_params  # noqa: F401

__version__ = "0.1.0"
