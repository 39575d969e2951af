from .relaxation import (
    matrix_diagonal,
    inverse_diagonal,
    jacobi,
    approximate_spectral_radius,
    none,
)
