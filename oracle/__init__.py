"""FP64 CPU oracle for the Hopkins/SOCS aerial-image path.

TEST INFRASTRUCTURE ONLY. This package restates, in numpy and plain C, the
reference's CPU algorithm for the imaging path (highuvlith-core: aerial.rs,
mask.rs, optics/, source.rs, ilt.rs, opc.rs, metrics.rs). It is the checker:
only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import or run it. The product (``highuvlith_b200``) never
imports anything from here and never falls back to it.

Pinning: the restatement is checked against the reference's own known-answer
tests (SOCS == direct Abbe sum, clear field == 1, coherent three-beam closed
form, mask-spectrum DC and pixel-transfer identities, ILT adjoint vs finite
differences, CD/NILS closed-form fixtures, and the published end-to-end
contrast / printed-CD numbers).
"""
