"""Per-shape choice among the library's runtime variants, by timing them.

For one run configuration (grid, precision, modules) every candidate combination of the options
below is timed on a scratch context loaded with the run's own inputs (a few steps after `initial`,
CUDA events on the context's stream), and the fastest is kept in a cache keyed by the shape, so an
ensemble with several members of one shape tunes it once.  The members' own contexts are never
stepped by the tuner.

    KMM_OPT_ZTMA            z transforms with TMA tile copies, or plain loads       (fused step)
    KMM_OPT_COLUMN_BLOCKED  column kernels on 16 lanes per column, or a warp each   (fused step)
    KMM_OPT_GRAPH           the step replayed from captured CUDA graphs, or launched kernel by kernel
    KMM_OPT_TC_DCT          y transforms as tensor-core GEMMs, or FFTs             (routine path, mixed)

The candidate set is the product of the values that apply to the configuration; at most eight
combinations are timed.
"""
import itertools

from . import abi

_CACHE = {}


def shape_key(p, ib=False):
    return (p.nx, p.ny, p.nz, p.precision, p.scalar_on, p.polymer_on, p.npart > 0, bool(ib), p.particle_flag > 0)


def candidates(p, ib=False):
    """Option combinations that make a difference for this configuration: a list of dicts."""
    routine = p.polymer_on or ib or (p.particle_flag > 0 and p.npart > 0) or (p.scalar_on and p.scl_flag >= 2)
    axes = []
    if not routine:
        axes.append((abi.OPT_ZTMA, (1, 0)))
        if p.ny in (32, 64, 96, 128) and p.precision == 0:
            axes.append((abi.OPT_COLUMN_BLOCKED, (1, 0)))
        axes.append((abi.OPT_GRAPH, (1, 0)))
    elif p.precision == 1:
        axes.append((abi.OPT_TC_DCT, (0, 1)))
    if not axes:
        return [{}]
    keys = [k for k, _ in axes]
    return [dict(zip(keys, vals)) for vals in itertools.product(*[v for _, v in axes])][:8]


def time_options(runtime, p, load, options, steps=4, warmup=3, device=0):
    """ms per step of a scratch context with `options` set, loaded by `load(ctx)`; None if the
    combination does not run (an option unsupported for the configuration)."""
    ctx = runtime.KmmContext(p, device=device)
    try:
        for k, v in options.items():
            ctx.call("set_option", k, v)
        load(ctx)
        if ctx.call("initial", allow=(abi.ERR_UNSUPPORTED,)):
            return None
        for _ in range(warmup):
            if ctx.call("step", allow=(abi.ERR_UNSUPPORTED, abi.ERR_CFL)):
                return None
        ctx.call("sync")
        ctx.event_record(0)
        for _ in range(steps):
            ctx.call("step", allow=(abi.ERR_CFL,))
        ctx.event_record(1)
        return ctx.event_elapsed(0, 1) / steps
    finally:
        ctx.close()


def tune(runtime, p, load, ib=False, device=0, steps=4):
    """(best options, {options-as-text: ms}) for the configuration, from the cache when the shape
    has been tuned before."""
    key = shape_key(p, ib)
    if key in _CACHE:
        return _CACHE[key]
    timings = {}
    best, best_ms = {}, None
    for opts in candidates(p, ib):
        ms = time_options(runtime, p, load, opts, steps=steps, device=device)
        timings[describe(opts)] = None if ms is None else round(ms, 4)
        if ms is not None and (best_ms is None or ms < best_ms):
            best, best_ms = opts, ms
    _CACHE[key] = (best, timings)
    return _CACHE[key]


def apply(ctx, options):
    for k, v in options.items():
        ctx.call("set_option", k, v)


_NAMES = {abi.OPT_ZTMA: "ztma", abi.OPT_COLUMN_BLOCKED: "column_blocked", abi.OPT_GRAPH: "graph",
          abi.OPT_TC_DCT: "tc_dct"}


def describe(options):
    return ",".join("%s=%d" % (_NAMES.get(k, str(k)), v) for k, v in sorted(options.items())) or "defaults"
