"""B200-native fixed-background Valencia GRHD operator (GRDzhadzha's
Source/Matter/GRHD fixed-background path) over a C ABI."""
from .operator import (  # noqa: F401
    AtmosphereOptions,
    CircularBinaryPN,
    FixedBGLevelDataFiniteVolumeOperator,
    IdealGasEOS,
    KerrSchild,
    LevelBox,
    LevelDataFiniteVolumeOperator,
    RecoveryOptions,
    TimeDependentFixedBGLevelDataFiniteVolumeOperator,
    level_exchange,
)
from ._lib import GRHDError, InvalidArgument  # noqa: F401
from .ensemble import Ensemble  # noqa: F401
