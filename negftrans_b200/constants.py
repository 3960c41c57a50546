"""Physical constants and unit conversions of src/global.f90:24-28."""
HARTREE = 27.211386245988          # eV, global.f90:24
K_B = 8.617333262e-5 / HARTREE     # Hartree / K, global.f90:26
A_0 = 0.529177210903               # Angstrom, global.f90:27
PI = 3.141592653589793             # global.f90:28
