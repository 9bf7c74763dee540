"""TEST INFRASTRUCTURE ONLY -- the parity oracle for slChannel's SL-BDF2 step.

A CPU restatement of the reference's float64 algorithm (gmcavallazzi/SLchannel
v1.0.1): the semi-Lagrangian trace and gather in plain C (``sl_oracle.c``,
built by ``oracle/Makefile`` into ``oracle/_build``), everything else of the
step in numpy (``slbdf2.py``).  Each function cites the reference file:line it
follows.

Pinned by ``tests/golden/*.npz``: outputs of the reference itself, run in the
development container by ``tests/golden/make_golden.py``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its
``cpu_baseline`` leg and ``--impl reference`` arm) may import this package, and
only as the reference answer that results are compared against, or as the
timed CPU baseline.  The product package
``slchannel_b200`` never imports it.
"""

from .slbdf2 import (  # noqa: F401
    OracleAdvector,
    OracleChannel,
    apply_bc_all,
    compute_bulk_velocity,
    compute_divergence,
    diffusion_xy,
    generate_grid,
    initialize_fft_solver,
    project_velocity,
    solve_implicit_diffusion,
    solve_poisson_fft,
)
