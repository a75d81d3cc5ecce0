"""ripple_b200: Ripple.jl's SSP-RK3 time-step path on one NVIDIA B200.

The public names mirror Ripple.jl's (set! -> set_, run! -> run_, time_step! ->
time_step). All compute runs in librpl.so (hand-written sm_100a kernels behind
the C-ABI of include/rpl.h); there is no CPU fallback.
"""
from ._lib import ArgumentError, RplError, load as load_library, LIB_PATH
from .grids import (Bounded, Flat, InfiniteDepth, Periodic, PolarWaveVectorGrid, RectilinearGrid,
                    centers_to_faces, lower_bounded_centers_to_faces)
from .sources import (BulkWindDrag, Clockwise, Counterclockwise, HollandHurricaneWind, LinearStormTrack,
                      LocalSaturationDissipation, PrecomputedSources, PressureCorrelationInput,
                      ExponentialWindInput, WaveAgeWindInput, WhitecappingDissipation, MeanSpectrumWhitecapping,
                      SourceTermSet)
from .model import (Clock, ProductField, PseudomomentumVelocities, Simulation, SpatialAveraging, SpectralWaveModel, WENO, WaveActionField,
                    compute_tendencies, interior, run_, set_, time_step, update_coupling)
from .ensemble import Ensemble
from . import decomposition
from .output import (HostBuffer, SnapshotWriter, diagnostics_device, fetch_output, snapshot_async,
                     snapshot_wait)
from . import learned
from .diagnostics import (diagnostics, m0, mean_direction, mean_period, root_mean_square_wavenumber,
                          significant_wave_height, total_action)

__all__ = [n for n in dir() if not n.startswith("_")]
