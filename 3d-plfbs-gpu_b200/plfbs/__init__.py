"""plfbs-b200: the LBFS explicit time step of 3D-PLFBS on B200 (sm_100a) behind
a C ABI (include/plfbs.h, include/plfbs_gnn.h; library plfbs/_lib/libplfbs.so).

Modules:
  build      compiles every csrc/ source for sm_100a into plfbs/_lib/libplfbs.so
  capi       ctypes binding of include/plfbs.h and a Solver class over it
  cases      synthetic cases: polyMesh generators, the reference's XML and
             polyMesh writers, the pre-processed mesh arrays in numpy
  gnn        ctypes binding of include/plfbs_gnn.h (the warm-start network)
  warmstart  solver-generated training data, training and inference of the
             warm start

Importing the package loads nothing; capi.lib() loads the library.
"""
