"""B200-native CM1 large-step dynamics (WENO5 advection + split-explicit acoustic step)
behind ThunderEngine's tape-player interface.

* ``timestep`` - the step encoder (command tape of one large step)
* ``scenario`` - synthetic CM1 inputs (grid, base state, bubble)
* ``replayer`` - the ``Replayer``-shaped host class over the CUDA C-ABI library
"""
