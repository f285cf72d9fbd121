"""Physical constants, identical to src/constants.rs:8-18 of the reference."""
import math

C0 = 299_792_458.0          # speed of light in vacuum (m/s)
EPS0 = 8.854_187_817e-12    # permittivity of free space (F/m)
MU0 = 1.256_637_062e-6      # permeability of free space (H/m)
Z0 = 376.730_313_668        # impedance of free space (Ohm)
PI = math.pi
