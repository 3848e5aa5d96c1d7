"""Optimiser side of the hot path: filters, OC update and the SIMP driver."""
