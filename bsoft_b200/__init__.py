"""bsoft_b200: B200-native single-particle Fourier reconstruction and
projection matching with the reference's (Bsoft) parameter-file and library
call surface."""
__version__ = "0.1.0"
