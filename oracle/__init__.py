"""CPU oracle for the photonfdtd time-stepping hot path (test infrastructure).

This package is the checker, not the product. Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its ``cpu_baseline`` leg and its
``--impl reference`` arm) may import it. The shipped engine in
``photonfdtd_b200`` never calls into it.

``fdtd_oracle`` restates, in NumPy, the reference's vectorised stepping loop
(``src/photonfdtd/simulation.py:910-1436`` of ngpaladi/photonfdtd v0.12.0),
together with the host-side tables the loop consumes. The parity pin is
``tests/golden/*.npz``: outputs of the reference itself on small scenes,
written by ``tests/golden/make_golden.py``. ``tests/test_oracle_golden.py``
checks the oracle against every one of them.
"""
from .fdtd_oracle import OracleRun, run_oracle, scene_tables  # noqa: F401
