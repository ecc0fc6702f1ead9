"""desi_b200 -- grid-node pair and triplet counting on NVIDIA B200 (sm_100a).

The compute path is ``libpcf.so`` (hand-written CUDA, C ABI in
``include/pcf.h``), built in tree by ``python -m desi_b200.build``.  This
package only binds it (``_lib``, ``api``) and provides catalog helpers
(``catalog``).  Importing :mod:`desi_b200.api` fails loudly when the library
is missing; there is no CPU fallback.
"""
__all__ = ["api", "catalog", "build"]
