"""Register this package as a backend of PriNCe's own solver factories.

PriNCe picks the implementation of ``UHECRPropagationSolverETD2`` and
``MultiRHSPropagationSolverETD2`` in their ``__new__`` from
``prince_run.backend.linear_algebra_backend``
(``src/prince_cr/solvers/propagation.py:398-404, 2400-2409``).  ``register``
adds one more value, ``"b200"`` by default, without editing PriNCe's files:
constructing either reference class with a run whose backend is set to that
value returns this package's solver (same constructor, flags, ``solve``,
``state``, ``res`` and multi-RHS views); every other backend value keeps
PriNCe's own dispatch.

    import prince_cr.solvers.propagation as P
    from prince_b200 import plugin
    plugin.register(P)
    run.backend.linear_algebra_backend = "b200"
    solver = P.UHECRPropagationSolverETD2(initial_z=1.0, final_z=0.0, prince_run=run)
"""

from __future__ import annotations

_PAIRS = (("UHECRPropagationSolverETD2", "UHECRPropagationSolverETD2"),
          ("MultiRHSPropagationSolverETD2", "MultiRHSPropagationSolverETD2"))


def _run_of(args, kwargs):
    """The ``prince_run`` argument: keyword, or the third positional (initial_z, final_z, prince_run)."""
    if "prince_run" in kwargs:
        return kwargs["prince_run"]
    return args[2] if len(args) > 2 else None


def register(propagation_module, name="b200", solvers=None):
    """Route the reference solver classes of ``propagation_module`` to this package for backend ``name``.

    ``solvers`` maps the reference class names to replacement classes
    (default: ``prince_b200.solvers``).  Registering twice is harmless.
    """
    if solvers is None:
        from . import solvers as _s

        solvers = {ref: getattr(_s, ours) for ref, ours in _PAIRS}
    key = name.lower()
    for ref_name, ours in solvers.items():
        ref_cls = getattr(propagation_module, ref_name)
        table = ref_cls.__dict__.get("_b200_backends")
        if table is None:
            table = {}
            original = ref_cls.__dict__.get("__new__")

            def __new__(cls, *args, _ref=ref_cls, _orig=original, _table=table, **kwargs):
                if cls is _ref:
                    run = _run_of(args, kwargs)
                    backend = getattr(getattr(run, "backend", None), "linear_algebra_backend", "")
                    target = _table.get(str(backend).lower())
                    if target is not None:
                        return target(*args, **kwargs)
                if _orig is None:
                    return object.__new__(cls)
                return _orig(cls, *args, **kwargs)

            ref_cls.__new__ = __new__
            ref_cls._b200_backends = table
        table[key] = ours
    return propagation_module
