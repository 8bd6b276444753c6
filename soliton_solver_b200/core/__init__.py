"""Core of the B200 backend: parameters, the native solver handle, hook adapters
and the Simulation driver (mirrors soliton_solver/core)."""
