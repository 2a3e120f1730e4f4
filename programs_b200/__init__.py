"""B200-native face-addressed Krylov solvers (the spray-simulation
``solv_cg`` / ``solv_bicg`` / ``solv_precond`` / ``solv_direct`` /
``solv_res`` hot path) with a C-ABI in ``include/solv_gpu.h``.

``programs_b200.solver`` mirrors the reference subroutines on top of the
C-ABI; ``programs_b200.mesh`` generates and renumbers the face-addressed
matrices they solve.
"""
