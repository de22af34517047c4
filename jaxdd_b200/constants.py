"""Physical constants of SIMsalabim 5.36 (its `DDTypesAndConstants` unit), which jaxdd takes over
unchanged (jaxdd src/jaxdd/constants.py:1-12).

They are not CODATA's values: the reference solution is SIMsalabim's, and a change in the fifth
digit of `K_B/Q` moves the thermal voltage and every exponential after it.
"""

#: Elementary charge, C.
Q = 1.6022e-19
#: Boltzmann's constant, J/K.
K_B = 1.3807e-23
#: Vacuum permittivity, F/m.
EPS_0 = 8.8542e-12
