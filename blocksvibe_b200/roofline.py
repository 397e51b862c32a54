"""Algorithmic work of the hot path, for the roofline: bytes each kernel must move at least (every distinct
input number read once, every output written once; a number is 4 L + 8 bytes: L limbs and an exponent) and
multiprecision multiply-accumulates, from the plan of one operator.  Per right-hand side counts scale with
the batch B through N = Smax^2 B."""


def number_bytes(L):
    return 4 * L + 8


def cauchy_level_bytes(lev, N, L):
    """b3d_cauchy_level: the level's gathered residues (columns in use) and h_inf rows read, H written"""
    cols = int(sum(int(x) for x in lev["ncol"]))
    return (cols + lev["nb"] + lev["nb"] * lev["Mr"]) * N * number_bytes(L)


def pole_level_bytes(lev, N, S, L):
    """b3d_pole_level: each task's H row read, its R and q L matrices read, its residues written, and the
    intermediate (scratch) written and read back"""
    T = len(lev["t_slot"])
    return (T * N * 4 + 2 * T * S * S) * number_bytes(L)


def cauchy_level_macs(lev, N):
    """multiprecision MACs of the Cauchy step (one-limb divisions by 2 / (D' - D_i)), padded rows excluded"""
    return sum(int(r) * int(c) for r, c in zip(lev["nrow"], lev["ncol"])) * N


def pole_level_macs(lev, N, S):
    return len(lev["t_slot"]) * 2 * S * N
