"""Finite-element side of the hot path: matrix-free K(rho) and the PCG solve."""
