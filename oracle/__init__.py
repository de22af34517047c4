"""TEST INFRASTRUCTURE ONLY — the CPU oracle that the CUDA path is checked against.

`oracle.dd` restates, in NumPy FP64 and vectorised over a batch of devices, the reference's
steady-state path: jaxdd's `solve_batch` (src/jaxdd/batch.py) and `solve_jv`
(src/jaxdd/solver.py), each function citing the lines it follows. Only `tests/`,
`__graft_entry__.smoke()` and `bench.py`'s CPU-baseline / reference arm may import it; the
product (`jaxdd_b200`) never does, and fails loudly without its CUDA library.

Pinning: the reference itself cannot run here (it needs JAX, which is not installed). The oracle
is pinned against the reference's own golden J-V curves (SimSS 5.36 runs committed under the
reference's tests/data, copied to tests/golden/inputs) at the reference's own tolerances, and
against its known-answer invariants (B(−x) = B(x) + x, sweep = dense solve, |J_sc| ≤ generation).
"""
