"""blocks_3d's drop-in hot path on one B200 (sm_100a): multiprecision radial recursion, derivative moments,
numerators with pole shifting and the xt / xt_radial write_output maps, behind the host interface of
BlocksviBe (recursion_gpu.Plan / Recursion, derivatives.Derivs, output.Output).  Kernels live in
libb3dgpu.so (csrc/, C ABI in include/b3dgpu.h); python -m blocksvibe_b200.build compiles it."""
__version__ = "0.1.0"
