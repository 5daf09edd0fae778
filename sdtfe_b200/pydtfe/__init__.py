"""pydtfe: the reference's Python interface (python/pydtfe/__init__.py), backed
by the B200 library.  Put the directory holding this package on sys.path (or
import it as sdtfe_b200.pydtfe) and use it exactly like the reference's module:
compute_surface_density, compute_3d_density, interpolate_field2grid,
compute_particle_density.  Extra: set_seed, set_precision."""
from ._pydtfe import *  # noqa: F401,F403
