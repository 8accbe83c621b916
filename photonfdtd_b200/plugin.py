"""Register ``backend="b200"`` on the reference ``photonfdtd.Simulation``.

    import photonfdtd, photonfdtd_b200.plugin as p
    p.install()
    sim = photonfdtd.Simulation(..., backend="b200")
    result = sim.run()          # stepped on the B200 engine

The reference validates backend names in ``Simulation.__init__``
(src/photonfdtd/simulation.py:412-415) and dispatches in ``run()``
(:896-904). ``install`` wraps both: the constructor accepts "b200" (stored
after the reference's own checks ran with a name it knows), and ``run``
routes "b200" simulations to ``photonfdtd_b200.engine.run_b200`` before the
reference's own branches. The reference's Grid, structures, sources,
monitors and Result objects are used unchanged.
"""
from __future__ import annotations

_installed = False


def install(module=None) -> None:
    """Patch ``module`` (default: the importable ``photonfdtd``) once."""
    global _installed
    if module is None:
        import photonfdtd as module
    Sim = module.Simulation
    if getattr(Sim, "_b200_installed", False):
        return
    orig_init = Sim.__init__
    orig_run = Sim.run

    def __init__(self, *args, backend="auto", **kw):
        want = backend
        orig_init(self, *args, backend="numpy" if want == "b200" else want, **kw)
        self.backend = want

    def run(self, *args, **kw):
        if getattr(self, "backend", None) == "b200":
            if args or kw.get("out_of_core"):
                raise NotImplementedError("out_of_core is not used by the b200 backend")
            from .engine import run_b200
            return run_b200(self)
        return orig_run(self, *args, **kw)

    Sim.__init__ = __init__
    Sim.run = run
    Sim._b200_installed = True
    _installed = True
