"""CPU oracle for the sweep hot path -- TEST INFRASTRUCTURE ONLY.

A plain-numpy restatement of the Renormalizer reference's algorithm for the
MPS sweep path (hop_expr, contract_one_site, expm_krylov, svd_qn,
select_basis, TDVP-PS / TDVP-PS2 sweeps, Davidson DMRG).  It is pinned
against golden fixtures produced by the reference itself (tests/golden).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
arm may import this package, and only as the checker / the timed CPU
baseline.  The product (``renormalizer_b200``) never imports it.
"""
