"""B200-native drop-in for SDDC's residual-and-time-step hot path.

The package replaces the reference's ``compresid`` (and everything under it)
plus the RK stage update with CUDA kernels built for sm_100a, behind the
C ABI declared in ``include/sddc.h``.  Python modules:

* ``mesh``, ``cases``, ``deck``: synthetic meshes, cases and the reference's
  file formats (input tooling);
* ``host``: the host-side set-up (connectivity, operators, metrics) through
  ``libsddc_host.so``;
* ``solver``: the drop-in itself, a ctypes binding of ``libsddc_b200.so``.
"""

__all__ = ["mesh", "cases", "deck", "host", "solver"]
