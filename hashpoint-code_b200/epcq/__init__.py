"""B200 drop-in for the reference's `epcq` package (point searching and sampling)."""
from .epcq import *  # noqa: F401,F403
from .epcq import CameraSpec, NeuralPoints, NeuralPointsGrads, RenderOptions  # noqa: F401

__version__ = "1.0.0"
