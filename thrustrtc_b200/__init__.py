"""thrustrtc_b200 -- B200-native data-parallel core with the ThrustRTC interface."""
from . import _native  # noqa: F401  (fails loudly when the CUDA library is missing)
