"""B200-native fused lattice-Boltzmann stream-collide step, as a pylbm backend.

* ``pylbm_b200.backend``  solver classes (pylbm's Solver contract) and ``register()``;
* ``pylbm_b200.problem``  a stand-alone mirror of pylbm's ``Problem``;
* ``pylbm_b200._lib``     the ctypes binding of the C ABI (include/pylbm_b200.h);
* ``pylbm_b200.build``    builds ``_lib/libpylbm_b200.so`` for sm_100a.
"""

__version__ = "0.1.0"
