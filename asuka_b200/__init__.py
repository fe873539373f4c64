"""B200-native density-fitted two-electron engine (DF 3c/2c Rys integrals, DF-J/K, DF gradient)."""

__version__ = "0.1.0"
