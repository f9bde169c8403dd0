"""B200 backend for the viscoelastic time step of VILMA v2 (fesmc/FastEarth3D)."""
