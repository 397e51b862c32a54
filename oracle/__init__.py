"""Oracle: a CPU restatement (pure Python + mpmath) of the reference's algorithms for the blocks_3d hot
path.  TEST INFRASTRUCTURE ONLY: it is imported by tests/, by __graft_entry__.smoke() and by bench.py's
CPU-baseline leg as the checker, never by the product package.

Pinned against golden vectors produced by the reference's own code (tests/golden/make_golden.py imports
the reference's recursion_ref / recursion_gpu.Plan / output / test ports and writes the fixtures; the
CPU tests check this oracle against them).

Modules:
  blocks       pole / spin bookkeeping (blocks_3d Pole.hxx etc.; reference structure.py:16-84)
  recursion    fill_residues (reference recursion_ref.py:11-44)
  derivatives  residues_to_derivatives, restore_r_delta, shift_fraction, together_with_factors
               (reference tests/test_blocks_derivatives.py:36-80) and blocks_3d's pole shifting by a
               linear solve (reference derivatives.py:27-33 describes it)
  output       lambda_lr_to_lrho_lrhob, congruence transforms, zzb_to_xt, lrho_to_xt_radial
               (reference output.py:1-21, 58-95; tests/test_blocks_output.py:13-47)
"""
