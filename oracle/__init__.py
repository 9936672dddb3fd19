"""FP64 CPU oracle for the Faceted HyperSARA primal-dual iteration.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` as the
checker and the timed CPU baseline.  The product (``faceted-hypersara_b200``)
never imports it.

Parity status: the reference (basp-group/Faceted-HyperSARA) is MATLAB whose
NUFFT and SARA primitives live in two un-vendored submodules and which ships no
tests or golden vectors, so this restatement is *parity unpinned* against the
MATLAB code.  It is pinned instead against mathematical known answers (exact
NUDFT, closed-form db2 filter, adjointness, perfect reconstruction, Moreau /
projection identities) and committed golden fixtures generated from it
(``tests/golden/make_golden.py``).
"""
