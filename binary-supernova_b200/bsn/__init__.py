"""bsn -- host-side mirror of Binary-Supernova's hot-path API on libbsn (B200).

Function names, argument order and meaning follow the reference Julia
package (src/euler3d.jl, src/gravity_bh.jl, src/sinks.jl, src/nbody.jl,
src/kepler_orbit.jl, src/self_gravity.jl, src/fmr3d.jl, src/fmr_gravity.jl),
with Julia's `!` dropped.  Device arrays are torch CUDA float64 tensors in the
reference layout U[q,i,j,k] (see `state`); every call runs hand-written
sm_100a kernels through the C ABI of include/bsn.h.  There is no CPU path.
"""
from .api import *  # noqa: F401,F403
from .api import __all__  # noqa: F401
from .h5io import *  # noqa: F401,F403,E402
from .h5io import __all__ as _h5io_all  # noqa: E402

__all__ = list(__all__) + list(_h5io_all)
