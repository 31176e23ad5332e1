"""B200 photon-mapping core: host side (Python) over the C ABI in include/pm_api.h."""
from .core import (PM_MAP_CAUSTIC, PM_MAP_GLOBAL, Batch, Camera, Context, PMError, camera_setup, library,  # noqa: F401
                   load_obj, write_pfm, write_ppm)
from . import scenes  # noqa: F401
