"""CPU oracle for the memetic-GA hot path of lucasgaldinos/tsp_gpu_clean.

TEST INFRASTRUCTURE ONLY. This package is a plain NumPy restatement of the
reference's CPU strategies (2-opt, tour cost, tournament selection, PMX,
inversion mutation, survival, elite selection, nearest-neighbour init and the
`GeneticAlgorithm.evolve` loop). Every function cites the reference file and
lines it follows (paths relative to the reference project root).

Only `tests/`, `__graft_entry__.smoke()` and the CPU-baseline legs of
`bench.py` may import it, and there only as the checker or as the timed CPU
baseline. The product package `tsp_gpu_clean_b200` never imports it; its GPU
path fails loudly when the CUDA library is missing.

Pinning: the oracle is checked against golden vectors produced by running the
reference itself (`tests/golden/make_golden.py`, committed with its outputs; the
checks are `tests/test_oracle_golden.py`). `three_opt_kernel.py` restates two
parts of the reference's 3-opt that exist only as CUDA kernels; it is pinned to
outputs of those kernels, compiled from the reference's sources by
`oracle/build_ref.py` and run by `tests/golden/make_three_opt_kernel_golden.py`.
Or-opt has no reference counterpart (`or_opt.py` pins itself two ways).
"""
