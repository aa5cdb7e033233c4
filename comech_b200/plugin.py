"""Install the device solver into an imported CoMech code base, the way the reference installs its own
GPU solver: by swapping module attributes that the engine looks up at call time (rb/rbfe.py:21-27 swaps
``fe.gmg.pcg_gmg``; rb/splitfe.py:125,153 and fe/solver.py:234-236 look it up at call time).

    import fe.gmg, fe.solver, splitfe          # the reference's modules
    from comech_b200 import plugin
    plugin.install(gmg=fe.gmg, solver=fe.solver, splitfe=splitfe)

Each replaced attribute keeps the original as ``_<name>_cpu`` on its module (as rb/rbfe.py keeps
``fe.gmg._pcg_gmg_cpu``) and ``uninstall`` puts it back.  Nothing here runs the original functions: the
device solver has no CPU fallback.
"""
from . import engine

_SWAPS = {
    "gmg": ("pcg_gmg",),
    "solver": ("solve", "cell_stress"),
    "splitfe": ("solve_cn", "cell_stress_cn", "element_forces_cn", "split_connectivity", "split_connectivity_fast"),
}


def _wrap(name, precision):
    if name.startswith("split_connectivity"):
        from .split import split_connectivity_device
        return split_connectivity_device
    fn = getattr(engine, name)
    if precision is None or name not in ("pcg_gmg", "solve", "solve_cn"):
        return fn

    def call(*a, **k):
        k.setdefault("precision", precision)
        return fn(*a, **k)
    call.__name__ = fn.__name__
    call.__doc__ = fn.__doc__
    return call


def install(gmg=None, solver=None, splitfe=None, precision=None):
    """Replace the solve entry points of the given reference modules (those the module has); ``precision``
    ('fp64', 'mixed', 'refine') becomes the default of the replaced solves."""
    mods = {"gmg": gmg, "solver": solver, "splitfe": splitfe}
    for key, mod in mods.items():
        if mod is None:
            continue
        for name in _SWAPS[key]:
            if not hasattr(mod, name):           # an older module without this entry point
                continue
            if not hasattr(mod, "_%s_cpu" % name):
                setattr(mod, "_%s_cpu" % name, getattr(mod, name))
            setattr(mod, name, _wrap(name, precision))


def uninstall(gmg=None, solver=None, splitfe=None):
    """Put back the functions ``install`` replaced."""
    mods = {"gmg": gmg, "solver": solver, "splitfe": splitfe}
    for key, mod in mods.items():
        if mod is None:
            continue
        for name in _SWAPS[key]:
            orig = getattr(mod, "_%s_cpu" % name, None)
            if orig is not None:
                setattr(mod, name, orig)
                delattr(mod, "_%s_cpu" % name)
