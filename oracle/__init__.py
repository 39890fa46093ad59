"""CPU oracle for the TT contraction-and-rounding path (TEST INFRASTRUCTURE ONLY).

This package restates, in FP64 numpy/scipy, the algorithms of the Julia package
TensorTrains (rodrigofj99/Tensor-Train-Julia) that the CUDA library replaces.
It is the checker: only the tests, ``__graft_entry__.smoke()`` and the CPU legs of
``bench.py`` may import it.  Nothing in the shipped ``ttcuda`` package imports it.

Parity status: the reference ships no golden vectors or seeded known answers for
this path, and Julia is not available to run it.  The oracle is pinned by the
reference's own property tests (dense equality, exact reconstruction,
partial_contraction == dot), re-expressed in ``tests/test_oracle_reference_props.py``.
"""
