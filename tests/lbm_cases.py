"""Shared case definitions for the parity tests (no GPU, no oracle imports)."""
import numpy as np

# lattice weights in the reference's direction order
W = np.array([1 / 18] * 4 + [1 / 36] * 4 + [1 / 18] + [1 / 36] * 4 + [1 / 18] + [1 / 36] * 4 + [1 / 3])
CX = np.array([0, 0, 1, -1, 1, 1, -1, -1, 0, 0, 1, -1, 0, 0, 0, 0, -1, 1, 0])
CY = np.array([1, -1, 0, 0, 1, -1, 1, -1, 0, 1, 0, 0, -1, 0, -1, 1, 0, 0, 0])
CZ = np.array([0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, 0])
INV = np.array([1, 0, 3, 2, 7, 6, 5, 4, 13, 14, 16, 17, 15, 8, 9, 12, 10, 11, 18])


def random_pdfs(ncells, seed, amp=0.05):
    """Equilibrium-like start with seeded perturbations: w_i * (1 + amp*U(-1,1))."""
    rng = np.random.default_rng(seed)
    return (W[None, :] * (1.0 + amp * (2.0 * rng.random((ncells, 19)) - 1.0))).astype(np.float64)


# (geometry, dims, periodic flags given on the command line)
FIELD_CASES = [
    ("box", (16, 16, 16), (1, 1, 0)),      # the -verify preset
    ("channel", (12, 10, 9), (0, 0, 0)),   # x faces fluid but not periodic for the kernels (open)
    ("channel", (12, 10, 9), (1, 0, 0)),
    ("fluid", (9, 8, 7), (0, 0, 0)),       # all faces open
    ("fluid", (9, 8, 7), (1, 1, 1)),       # fully periodic
    ("fluid", (9, 8, 7), (1, 0, 1)),       # mixed: corner links wrap on every crossed axis
    ("pipe", (10, 12, 11), (0, 0, 0)),
    ("blocks-2", (13, 11, 12), (0, 1, 0)),
    ("box", (5, 7, 9), (0, 1, 1)),
]
