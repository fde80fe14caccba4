"""Physical constants and the float32 field type, as open_sol defines them (open_sol/core/constants.py:5-18)."""
import numpy as np

DTYPE = np.float32
C0 = 299792458.0
EPS0 = 8.8541878128e-12
MU0 = 1.2566370614e-6
ETA0 = np.sqrt(MU0 / EPS0)
FACES = ('x_lo', 'x_hi', 'y_lo', 'y_hi')
FACES_3D = FACES + ('z_lo', 'z_hi')
