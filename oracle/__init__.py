"""Oracle package — TEST INFRASTRUCTURE ONLY.

CPU restatement of the cuEV reference solver used to check the CUDA library
(``cuev_oracle``).  Imported only by ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py``; the product (``cuev_b200``) never imports it.
"""
