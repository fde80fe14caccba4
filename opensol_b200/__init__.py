"""opensol_b200: a B200-native FDTD time-stepping engine behind open_sol's solver contract.

The FDTD path of open_sol (Simulation.run -> EMPhysics.step -> FDTDEngine2D_Ez.advance in 2D, EMPhysics3D.step ->
FDTDEngine3D.advance in 3D) with the field updates, CPML, source injection and DFT monitors in hand-written sm_100a CUDA (libopensol_fdtd.so, C ABI in include/opensol_fdtd.h),
called through ctypes.  There is no CPU fallback: without the built library or a CUDA device the engines raise.
"""
from .boundaries import BCType, BoundaryConfig
from .domain import Domain
from .domain3d import BoundaryConfig3D, Domain3D
from .grid import Grid2D, courant_time_step
from .monitors import DFTMonitor, FluxMonitor, dft_sample_interval
from .physics import EMPhysics
from .physics3d import EMPhysics3D
from .simulation import MultiphysicsRunner, Simulation
from .poles import DrudePole, LorentzPole
from .sources import ContinuousWave, GaussianPulse, LineSource, RickerWavelet

__all__ = ['BCType', 'BoundaryConfig', 'BoundaryConfig3D', 'Domain', 'Domain3D', 'EMPhysics3D', 'Grid2D', 'courant_time_step', 'DFTMonitor', 'DrudePole', 'FluxMonitor', 'LorentzPole',
           'dft_sample_interval', 'EMPhysics', 'MultiphysicsRunner', 'Simulation', 'ContinuousWave',
           'GaussianPulse', 'LineSource', 'RickerWavelet']
__version__ = '0.1.0'
