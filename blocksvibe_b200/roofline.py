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


def pole_mma_geometry(L):
    """(U, MT): digits per entry along K and 128-position tiles of the tensor-core pole step (pole_mma.cuh)"""
    NB, D = 32 * L - 2, 4 * L
    U = 32 * (-(-D // 32))

    def p0(mt):
        top = 8 * L - 1 - 128 * mt
        return 0 if top <= 0 else 16 * (-(-top // 16))
    return U, (1 if 8 * p0(1) + 17 <= NB - 160 else 2)


def pole_mma_macs(lev, N, S, L):
    """int8 MACs of both stages of b3d_pole_level_mma on one level, N = S^2 B numbers per task as in
    pole_level_bytes: (issued by the MMAs, digit products of the exact sums).  A task has S B columns; per task
    and stage: S rows x S entries x U / 32 K steps x MT tiles of 128 x NC x 32 MACs per column chunk; the exact
    sums need S^2 (S B) (4 L)^2 digit products."""
    U, MT = pole_mma_geometry(L)
    T = len(lev["t_slot"])
    cols = N // S
    nc = 32 if cols >= 32 else 16 * (-(-cols // 16))
    chunks = -(-cols // nc)
    issued = 2 * T * chunks * S * S * (U // 32) * MT * 128 * nc * 32
    useful = 2 * T * S * S * cols * (4 * L) ** 2
    return issued, useful
